"""sailfish_b200: the reference's ROMS-style time step on NVIDIA B200 (sm_100a).

Host set-up (sailfish_b200.host), the C-ABI library binding (sailfish_b200._lib), the
reference-facing entry points (sailfish_b200.api) and the device model driver
(sailfish_b200.model).
"""
__version__ = "0.1.0"
