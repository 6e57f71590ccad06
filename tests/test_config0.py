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
