"""The drop-in Python entry points (sailfish_b200.dropin) driven exactly as the reference's
nonlinear/main3d.py:118-324 drives its own, on reference-shaped state objects whose arrays
are CUDA arrays (torch tensors through __cuda_array_interface__), against the reference's own
main3d runs: bit-exact in FP64."""
import numpy as np
import pytest

from golden_io import load, boundary_dict

NAMES2 = ("zeta", "ubar", "vbar", "rzeta", "rubar", "rvbar")


class RefGrid:
    pass


class RefOcean:
    """The attribute layout of T_OCEAN (modules/mod_ocean.py:14-154): three-slot parents,
    flat _t0/_t1/_t2 views rotated by cycleTimes2D, 3D fields used through slot 2."""

    def __init__(self, d, N, J, I, torch):
        t = lambda a, shape: torch.tensor(np.asarray(a, np.float64).reshape(shape), device="cuda")
        for n in NAMES2:
            setattr(self, n, t(d["in_" + n], (3, J, I)))
            for k in range(3):
                setattr(self, "%s_t%d" % (n, k), getattr(self, n)[k].view(-1))
        for n in ("u", "v", "ru", "rv"):
            setattr(self, n, t(d["in_" + n], (3, N + 1, J, I)))
            setattr(self, n + "_t2", getattr(self, n)[2].view(-1))
        for n in ("W", "Huon", "Hvom", "AKv"):
            setattr(self, n, t(d["in_" + n], (N + 1, J, I)))
        for n in ("Zt_avg1", "DU_avg1", "DV_avg1"):
            setattr(self, n, t(d["in_" + n], (J * I,)))

    def cycleTimes2D(self):
        for n in NAMES2:
            a, b, c = (getattr(self, "%s_t%d" % (n, k)) for k in range(3))
            setattr(self, n + "_t0", b)
            setattr(self, n + "_t1", c)
            setattr(self, n + "_t2", a)


class RefCompTimes:
    """The counters of modules/mod_comptimes.py:7-100 used on the step path."""

    def __init__(self, dt, ndtfast, nfast, weight1):
        self.dt, self.ndtfast, self.nfast = dt, ndtfast, nfast
        self.dtfast = dt / ndtfast
        self.weight1 = weight1
        self.iic = self.iif = self.ntfirst = 0
        self.time = self.time2D = 0.0

    def isFirst2DStep(self):
        return self.iif == 0

    def first2DTimeStep(self):
        self.iif = 0

    def next2DTimeStep(self):
        self.iif += 1
        self.time2D += self.dtfast

    def nextTimeStep(self):
        self.iic += 1
        self.time += self.dt
        self.time2D = self.time


@pytest.mark.gpu
@pytest.mark.parametrize("tag", ["square", "vt1"])
def test_reference_main3d_through_dropin_is_bit_exact(tag):
    import torch
    from sailfish_b200 import dropin, host
    d = load("main3d_%s.npz" % tag)
    L, M, N = int(d["in_L"]), int(d["in_M"]), int(d["in_N"])
    J, I = M + 1, L + 1
    GRID = RefGrid()
    GRID.L, GRID.M, GRID.N = L, M, N
    for k in ("h", "pm", "pn", "on_u", "om_v", "fomn", "sc_r", "sc_w", "Cs_r", "Cs_w"):
        a = np.asarray(d["in_grid_" + k], np.float64)
        setattr(GRID, k, torch.tensor(a.reshape((J, I)) if a.size == J * I else a, device="cuda"))
    GRID.hc, GRID.Vtransform = float(d["in_grid_hc"]), int(d["in_Vtransform"])
    GRID.Hz = torch.zeros((N, J, I), dtype=torch.float64, device="cuda")
    GRID.z_r = torch.zeros((N, J, I), dtype=torch.float64, device="cuda")
    GRID.z_w = torch.zeros((N + 1, J, I), dtype=torch.float64, device="cuda")
    BOUNDARY = host.Boundary(L, M)
    ref_b = boundary_dict(d, "in_bnd_")
    np.testing.assert_array_equal(BOUNDARY.ubarGradientBCIdx2, ref_b["ubarGradientBCIdx2"])
    OCEAN = RefOcean(d, N, J, I, torch)
    nfast, w1, _ = host.set_weights(int(d["in_ndtfast"]))
    ct = RefCompTimes(float(d["in_dt"]), int(d["in_ndtfast"]), nfast, w1)
    dropin.initModule(GRID, BOUNDARY, precision="fp64")
    BC = torch.tensor(BOUNDARY.zetaBC.bcIdxFieldIdx2, dtype=torch.int32, device="cuda")
    tmpU = torch.zeros_like(OCEAN.u_t2)
    tmpV = torch.zeros_like(OCEAN.v_t2)
    g, b = (1,), (1,)

    # main3d.py:62, then the step loop (main3d.py:118-324)
    dropin.set_depth(g, b, (GRID.Vtransform, OCEAN.Zt_avg1, GRID.z_w, GRID.z_r, GRID.h, GRID.hc,
                            GRID.Hz, GRID.sc_r, GRID.sc_w, GRID.Cs_r, GRID.Cs_w))
    for _ in range(int(d["in_nsteps"])):
        dropin.set_maxflux(g, b, (OCEAN.u_t2, OCEAN.v_t2, OCEAN.Huon, OCEAN.Hvom, GRID.Hz))
        dropin.omega(g, b, (OCEAN.W, OCEAN.u_t2, OCEAN.v_t2, OCEAN.Huon, OCEAN.Hvom, GRID.z_w, BC))
        dropin.set_zeta(g, b, (OCEAN.zeta_t1, OCEAN.zeta_t2, OCEAN.Zt_avg1))
        dropin.rhs3d(GRID, OCEAN, BOUNDARY)
        ct.first2DTimeStep()
        for _ in range(ct.nfast + 1):
            if ct.isFirst2DStep():
                OCEAN.Zt_avg1.zero_()
                OCEAN.DU_avg1.zero_()
                OCEAN.DV_avg1.zero_()
            ct.next2DTimeStep()
            OCEAN.cycleTimes2D()
            dropin.step2dPredictor(ct, GRID, OCEAN, BOUNDARY)
            dropin.step2dCorrector(ct, GRID, OCEAN, BOUNDARY)
            OCEAN.vbar_t2.zero_()
        dropin.set_depth(g, b, (GRID.Vtransform, OCEAN.Zt_avg1, GRID.z_w, GRID.z_r, GRID.h,
                                GRID.hc, GRID.Hz, GRID.sc_r, GRID.sc_w, GRID.Cs_r, GRID.Cs_w))
        tmpU.copy_(OCEAN.u_t2)
        tmpV.copy_(OCEAN.v_t2)
        dropin.step3d_UV(g, b, (OCEAN.u_t2, OCEAN.v_t2, OCEAN.ru_t2, OCEAN.rv_t2, OCEAN.ubar_t1,
                                OCEAN.vbar_t1, OCEAN.ubar_t2, OCEAN.vbar_t2, GRID.Hz, OCEAN.AKv,
                                GRID.z_r, OCEAN.DU_avg1, OCEAN.DV_avg1, tmpU, tmpV, GRID.h,
                                ct.iic, ct.ntfirst, 1.0, 1e-5, ct.dt))
        dropin.setLateralUVBCs(g, b, (ct.time, OCEAN.u_t2, OCEAN.v_t2, None, None, None, None))
        dropin.omega(g, b, (OCEAN.W, OCEAN.u_t2, OCEAN.v_t2, OCEAN.Huon, OCEAN.Hvom, GRID.z_w, BC))
        ct.nextTimeStep()
    torch.cuda.synchronize()

    for n in NAMES2:
        slots = list(d["out_slots_" + n])
        ref = d["out_" + n].reshape(3, -1)
        for k in range(3):
            np.testing.assert_array_equal(getattr(OCEAN, "%s_t%d" % (n, k)).cpu().numpy(),
                                          ref[slots[k]], err_msg="%s_t%d" % (n, k))
    for n in ("u", "v", "ru", "rv"):
        np.testing.assert_array_equal(getattr(OCEAN, n)[2].cpu().numpy().ravel(),
                                      d["out_" + n][2].ravel(), err_msg=n)
    for n in ("W", "Huon", "Hvom", "Zt_avg1", "DU_avg1", "DV_avg1"):
        np.testing.assert_array_equal(getattr(OCEAN, n).cpu().numpy().ravel(),
                                      d["out_" + n].ravel(), err_msg=n)
    for n in ("z_w", "z_r", "Hz"):
        np.testing.assert_array_equal(getattr(GRID, n).cpu().numpy().ravel(),
                                      d["out_" + n].ravel(), err_msg=n)


@pytest.mark.gpu
def test_dropin_rejects_wrong_arrays():
    import torch
    from sailfish_b200 import dropin
    from sailfish_b200._lib import SailfishError
    from sailfish_b200 import configs
    cfg = configs.small(16, 12, 6)
    g = cfg["grid"]
    dropin.initModule(g, cfg["boundary"], precision="fp64")
    J, I, N = g.J, g.I, g.N
    f32 = torch.zeros((N + 1, J, I), dtype=torch.float32, device="cuda")
    f64 = torch.zeros((N + 1, J, I), dtype=torch.float64, device="cuda")
    with pytest.raises(SailfishError, match="element type"):
        dropin.set_maxflux((1,), (1,), (f32, f64, f64, f64, f64[:N]))
    with pytest.raises(SailfishError, match="C-contiguous"):
        dropin.set_maxflux((1,), (1,), (f64.transpose(1, 2), f64, f64, f64, f64[:N]))
    with pytest.raises(SailfishError, match="CUDA array"):
        dropin.set_maxflux((1,), (1,), (np.zeros(3), f64, f64, f64, f64[:N]))


def test_dropin_needs_initmodule():
    from sailfish_b200 import dropin
    from sailfish_b200._lib import SailfishError
    saved = dropin._ctx
    dropin._ctx = None
    try:
        with pytest.raises(SailfishError, match="initModule"):
            dropin._need()
    finally:
        dropin._ctx = saved
