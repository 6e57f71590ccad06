"""sailfish_b200: the reference's ROMS-style time step on NVIDIA B200 (sm_100a).

Host set-up (sailfish_b200.host), the C-ABI library binding (sailfish_b200._lib), the
reference-facing entry points (sailfish_b200.dropin), the device model driver
(sailfish_b200.model), the learned closure (sailfish_b200.closure) and the ensemble driver
(sailfish_b200.ensemble).
"""
__version__ = "0.2.0"
