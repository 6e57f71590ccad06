"""Config 0: the flat closed 130 x 66 basin (dx = dy = 5 km, h = 4000 m, beta-plane f, dt = 30 s)
in the reference's main2d order (nonlinear/main2d.py:9-88: next2DTimeStep, cycleTimes2D,
step2dPredictor, step2dCorrector per 2D step).

The reference's runnable 2D step has no wind stress, bottom drag or 2D Coriolis (they exist only
in its untranslated pseudo-code), so a basin at rest stays at rest; the runs start from a 1 cm
Gaussian surface bump instead.  On this non-square grid the reference's flat-index semantics
(the momentum predictor's guard against the row count, mod_cppkernels.cpp:162) make the
solution non-finite within a few steps; the comparison is bit for bit through that, against the
reference's own kernels compiled for the host (oracle/_ref), for the oracle restatement (CPU)
and for the drop-in entry points in FP64 (GPU).  The fast-time weights are zero-padded past the
reference's 257 entries (main2d's counter passes them; they only feed the accumulators, which do
not enter zeta, ubar or vbar)."""
import numpy as np
import pytest

import oracle as O
import ref_driver as RD

NSTEPS = 8
NAMES2 = ("zeta", "ubar", "vbar")
BKEYS = ("zetaClosedOrGradientBCIdx1", "zetaClosedOrGradientBCIdx2", "ubarClosedBCIdx1",
         "vbarClosedBCIdx1", "ubarClampedBCIdx1", "ubarGradientBCIdx1", "ubarGradientBCIdx2",
         "vbarGradientBCIdx1")


def case():
    from sailfish_b200 import configs
    cfg = configs.basin0()
    g, B = cfg["grid"], cfg["boundary"]
    bump = 0.01 * np.exp(-((g.x - g.x.max() / 2) ** 2 + (g.y - g.y.max() / 2) ** 2) / 50.0e3 ** 2)
    return cfg, g, B, bump


def oracle_state(g, B, bump):
    og = O.Grid(g.L, g.M, g.N, g.h, g.pm, g.pn, g.on_u, g.om_v, g.fomn, g.sc_r, g.sc_w, g.Cs_r,
                g.Cs_w, g.hc, g.Vtransform)
    ob = O.Boundary({k: np.ascontiguousarray(getattr(B, k), np.int32) for k in BKEYS})
    oc = O.Ocean(og)
    for k in range(3):
        oc.zeta[k][...] = bump
    ct = O.CompTimes(30.0, 1, 1, np.zeros(4 * NSTEPS + 257), np.zeros(4 * NSTEPS + 257))
    return og, ob, oc, ct


def slots(oc, n):
    return np.stack([oc.t(n, k) for k in range(3)])


def reference_run(g, B, bump):
    og, ob, oc, ct = oracle_state(g, B, bump)
    RD.main2d(og, ob, oc, ct, NSTEPS)
    return {n: slots(oc, n) for n in NAMES2}


@pytest.mark.skipif(not RD.available(), reason="oracle/_ref not built")
def test_oracle_main2d_matches_the_reference_on_config0():
    cfg, g, B, bump = case()
    ref = reference_run(g, B, bump)
    og, ob, oc, ct = oracle_state(g, B, bump)
    O.main2d(og, ob, oc, ct, NSTEPS)
    for n in NAMES2:
        np.testing.assert_array_equal(slots(oc, n), ref[n], err_msg=n)
    # the reference's semantics on this non-square grid: non-finite within the run
    assert not np.isfinite(ref["zeta"]).all()


class _Ocean:
    """The 2D part of T_OCEAN (modules/mod_ocean.py:14-154) on torch CUDA arrays."""

    def __init__(self, J, I, bump, torch):
        for n in NAMES2 + ("rzeta", "rubar", "rvbar"):
            a = torch.zeros((3, J, I), dtype=torch.float64, device="cuda")
            if n == "zeta":
                a[:] = torch.from_numpy(bump)
            setattr(self, n, a)
            for k in range(3):
                setattr(self, "%s_t%d" % (n, k), a[k].view(-1))
        for n in ("Zt_avg1", "DU_avg1", "DV_avg1"):
            setattr(self, n, torch.zeros(J * I, dtype=torch.float64, device="cuda"))

    def cycleTimes2D(self):
        for n in NAMES2 + ("rzeta", "rubar", "rvbar"):
            a, b, c = (getattr(self, "%s_t%d" % (n, k)) for k in range(3))
            setattr(self, n + "_t0", b)
            setattr(self, n + "_t1", c)
            setattr(self, n + "_t2", a)


class _Times:
    def __init__(self, dt):
        self.dtfast = dt
        self.iif = 0
        self.time2D = 0.0
        self.weight1 = np.zeros(4 * NSTEPS + 257)

    def isFirst2DStep(self):
        return self.iif == 0

    def next2DTimeStep(self):
        self.iif += 1
        self.time2D += self.dtfast


@pytest.mark.gpu
def test_dropin_main2d_is_bit_exact_on_config0():
    import torch
    from sailfish_b200 import dropin
    cfg, g, B, bump = case()
    ref = reference_run(g, B, bump)
    dropin.initModule(g, B, precision="fp64")
    OC = _Ocean(g.J, g.I, bump, torch)
    ct = _Times(cfg["dt"] / cfg["ndtfast"])
    for _ in range(NSTEPS):   # nonlinear/main2d.py:43-80
        ct.next2DTimeStep()
        OC.cycleTimes2D()
        dropin.step2dPredictor(ct, g, OC, B)
        dropin.step2dCorrector(ct, g, OC, B)
    torch.cuda.synchronize()
    for n in NAMES2:
        got = np.stack([getattr(OC, "%s_t%d" % (n, k)).cpu().numpy() for k in range(3)])
        np.testing.assert_array_equal(got, ref[n], err_msg=n)


# ---- config 0 with its forcing, in the ROMS form -------------------------------------------------
# Config 0 asks for wind stress tau_x = 0.1 cos(pi y/Ly) N/m2, quadratic bottom drag 3e-3 and
# Coriolis from rest for 2000 steps of 30 s.  Those terms exist in the ROMS-form step
# (oracle/roms_oracle.py, Model(semantics="roms")); at h = 4000 m and dx = 5 km its time step of
# 30 s is c dt / dx = 1.2, beyond the scheme's 2D stability limit of 0.757 (von Neumann, tested
# in tests/test_roms.py), so the same 16.7 simulated hours run as 4000 steps of 15 s (0.6).
DT0, NSTEPS0 = 15.0, 4000


def _roms_case():
    import roms_oracle as ro
    from sailfish_b200 import configs
    cfg = configs.basin0()
    g = cfg["grid"]
    G = dict(h=g.h, pm=g.pm, pn=g.pn, on_u=g.on_u, om_v=g.om_v, fomn=g.fomn)
    Ly = (g.M - 1) / g.pn.flat[0]
    su = 0.1 * np.cos(np.pi * g.y / Ly) / 1025.0
    return cfg, g, G, su, np.zeros_like(su), ro


def test_roms_form_config0_forced_from_rest():
    """2000 x 30 s of config 0's forcing from rest (as 4000 x 15 s): finite, volume conserved to
    rounding, and a wind-driven flow: eastward depth-mean flow under the eastward wind of the
    southern half, westward in the north, with sea level set up against the walls."""
    cfg, g, G, su, sv, ro = _roms_case()
    S = ro.State(g.J, g.I)
    with np.errstate(all="raise"):
        ro.main2d(G, S, NSTEPS0, DT0, su, sv, 3e-3)
    z, u = S.zeta[1], S.ubar[1]
    assert np.isfinite(z).all() and np.isfinite(u).all()
    area = 1.0 / (g.pm * g.pn)
    assert abs(ro.volume(G, z)) <= 1e-12 * np.abs(z).max() * area.sum()
    J = g.J
    south, north = u[2:J // 4, 3:-3].mean(), u[3 * J // 4:J - 2, 3:-3].mean()
    assert south > 1e-4 and north < -1e-4
    assert 1e-4 < np.abs(z).max() < 1e-2     # set-up ~ tau L / (rho g h) = 1.6 mm


@pytest.mark.gpu
def test_roms_form_config0_forced_cuda_bit_exact():
    """The same run through the FP64 CUDA kernels (sf_roms_step2d), bit for bit."""
    import torch
    from sailfish_b200.model import Model
    cfg, g, G, su, sv, ro = _roms_case()
    m = Model(g, cfg["boundary"], cfg["dt"], 1, precision="fp64", semantics="roms")
    m.set_forcing(su, sv, 3e-3)
    m.dtfast = DT0
    m.step2d(NSTEPS0)
    torch.cuda.synchronize()
    S = ro.State(g.J, g.I)
    ro.main2d(G, S, NSTEPS0, DT0, su, sv, 3e-3)
    sh = (g.J, g.I)
    for n in ("zeta", "ubar", "vbar"):
        buf = getattr(m, n).cpu().numpy()
        for k in range(2):
            np.testing.assert_array_equal(buf[m.slots[k]].reshape(sh), getattr(S, n)[k],
                                          err_msg="%s[%d]" % (n, k))
