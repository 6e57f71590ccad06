"""The whole time step on the GPU against the reference's own main3d runs.

FP64: bit-exact (the FP64 kernels are built without FMA contraction and evaluate every
expression as the reference does).  FP32: stencils in FP32 with FP64 accumulators; the
error is stated against the reference run.
"""
import numpy as np
import pytest

from golden_io import load, boundary_dict
from sailfish_b200 import host

NAMES = ("zeta", "ubar", "vbar", "rzeta", "rubar", "rvbar", "u", "v", "ru", "rv", "W", "Huon",
         "Hvom", "Zt_avg1", "DU_avg1", "DV_avg1", "AKv")


def golden_model(tag, precision):
    from sailfish_b200.model import Grid, Model
    d = load("main3d_%s.npz" % tag)
    L, M, N = int(d["in_L"]), int(d["in_M"]), int(d["in_N"])
    g = lambda k: d["in_grid_" + k]
    grid = Grid(L, M, N, g("h"), g("pm"), g("pn"), g("on_u"), g("om_v"), g("fomn"), g("sc_r"),
                g("sc_w"), g("Cs_r"), g("Cs_w"), float(g("hc")), int(d["in_Vtransform"]))
    B = host.Boundary(L, M)
    ref_b = boundary_dict(d, "in_bnd_")
    np.testing.assert_array_equal(B.zetaClosedOrGradientBCIdx1, ref_b["zetaClosedOrGradientBCIdx1"])
    np.testing.assert_array_equal(B.uvelBC.bcIdxFieldType, ref_b["uvelBC_bcIdxFieldType"])
    m = Model(grid, B, float(d["in_dt"]), int(d["in_ndtfast"]), precision=precision)
    assert m.nfast == int(d["in_nfast"])
    m.load({n: d["in_" + n] for n in NAMES})
    return m, d


def out_of(d, n, slots=None):
    a = d["out_" + n]
    if n in ("u", "v", "ru", "rv"):
        a = a[2]
    return a


@pytest.mark.gpu
@pytest.mark.parametrize("tag", ["square", "nonsquare", "vt1"])
def test_main3d_fp64_bit_exact(tag):
    m, d = golden_model(tag, "fp64")
    m.step(int(d["in_nsteps"]))
    s = m.state()
    for n in ("zeta", "ubar", "vbar", "rzeta", "rubar", "rvbar"):
        assert s["slots"] == list(d["out_slots_" + n])
    for n in NAMES + ("z_w", "z_r", "Hz"):
        np.testing.assert_array_equal(s[n].reshape(-1), out_of(d, n).reshape(-1), err_msg=n)
    assert m.iic == int(d["out_iic"]) and m.time == float(d["out_time"])


@pytest.mark.gpu
def test_main3d_fp32_error_stated():
    m, d = golden_model("square", "fp32")
    m.step(int(d["in_nsteps"]))
    s = m.state()
    # Relative to each field's largest magnitude: FP32 stencils with FP64 accumulators.
    tol = {"zeta": 2e-5, "ubar": 2e-5, "vbar": 2e-5, "u": 2e-4, "v": 2e-4, "Zt_avg1": 2e-5,
           "DU_avg1": 2e-5, "DV_avg1": 2e-5, "z_w": 1e-6, "Hz": 1e-5}
    for n, t in tol.items():
        ref = out_of(d, n).reshape(-1)
        got = s[n].reshape(-1)
        scale = max(np.abs(ref).max(), 1e-30)
        err = np.abs(got - ref).max() / scale
        assert err <= t, "%s: max error %.3g of field scale (tolerance %.1g)" % (n, err, t)


@pytest.mark.gpu
@pytest.mark.parametrize("ndtfast,precision,L,M", [(4, "fp64", 24, 24), (5, "fp64", 24, 24),
                                                   (7, "fp64", 24, 24), (30, "fp64", 24, 24),
                                                   (30, "fp32", 24, 24), (5, "fp64", 100, 60)])
def test_graph_replay_of_the_barotropic_loop_is_identical(ndtfast, precision, L, M):
    """sf_barotropic_loop replayed from captured CUDA graphs (the default) against plain
    launches, with and without programmatic dependent launch and the fused predictor, over
    steps whose slot rotation cycles through all three phases: bit-identical in FP64.  The
    100 x 60 basin has fused-predictor tiles wholly inside the deep region (which leave before
    the count that orders the corner chains' writes) as well as edge tiles."""
    import numpy as np
    import torch
    from sailfish_b200 import configs
    from sailfish_b200._lib import lib
    from sailfish_b200.model import Model
    cfg = configs.basin(L, M, 6, 2.0e4, [(0.5, 0.5)], dt=240.0, ndtfast=ndtfast)
    g = cfg["grid"]
    bump = 1e-3 * np.exp(-((g.x - g.x.max() / 2) ** 2 + (g.y - g.y.max() / 2) ** 2) / (1e5) ** 2)
    out = []
    for graphs, pdl, fused in ((0, 0, 0), (1, 1, 1), (0, 1, 1), (1, 0, 0), (0, 0, 1)):
        m = Model(g, cfg["boundary"], cfg["dt"], cfg["ndtfast"], precision=precision)
        assert lib.sf_ctx_fused_available(m.ctx.ptr) == 1
        assert lib.sf_ctx_set_graphs(m.ctx.ptr, graphs) == 0
        assert lib.sf_ctx_set_pdl(m.ctx.ptr, pdl) == 0
        assert lib.sf_ctx_set_fused(m.ctx.ptr, fused) == 0
        m.Zt_avg1.copy_(torch.from_numpy(bump.ravel()))
        m.step(4)
        torch.cuda.synchronize()
        out.append(m.state())
    for o in out[1:]:
        for k in ("zeta", "ubar", "vbar", "u", "v", "Zt_avg1", "DU_avg1", "W"):
            if precision == "fp64":
                np.testing.assert_array_equal(o[k], out[0][k], err_msg=k)
            else:   # the fused predictor's FP32 contractions may differ from the unfused ones
                scale = max(np.abs(out[0][k]).max(), 1e-30)
                assert np.abs(o[k] - out[0][k]).max() <= 1e-5 * scale, k
        assert o["slots"] == out[0]["slots"]


@pytest.mark.gpu
@pytest.mark.parametrize("precision,mode", [("fp64", "gls"), ("fp32", "gls")])
def test_overlapped_phases_give_the_same_step(precision, mode):
    """Model.step with rhs3d beside the barotropic loop and the closure beside the next step's
    first phases (the default) against the phases one after another: identical fields after
    several steps, including the mixing's own."""
    import numpy as np
    import torch
    from sailfish_b200 import closure, configs
    from sailfish_b200.model import Model
    cfg = configs.basin(40, 24, 8, 2.0e3, [(0.5, 0.5)], dt=120.0, ndtfast=10)
    g = cfg["grid"]
    bump = 1e-3 * np.exp(-((g.x - g.x.max() / 2) ** 2 + (g.y - g.y.max() / 2) ** 2) / (2e4) ** 2)
    out = []
    for overlap in (False, True):
        m = Model(g, cfg["boundary"], cfg["dt"], cfg["ndtfast"], precision=precision)
        m.overlap = overlap
        m.Zt_avg1.copy_(torch.from_numpy(bump.ravel()))
        m.mixing = closure.Closure(m, mode)
        closure.wind_driven_state(m, m.mixing.cols, 0.1, 0.3, 500.0, np.random.default_rng(2))
        m.step(3)
        torch.cuda.synchronize()
        st = m.state()
        st["tke"] = m.mixing.cols.tke.cpu().numpy()
        st["AKv"] = m.AKv.cpu().numpy()
        out.append(st)
    for k in ("zeta", "ubar", "vbar", "u", "v", "W", "Zt_avg1", "AKv", "tke"):
        np.testing.assert_array_equal(out[1][k], out[0][k], err_msg=k)


@pytest.mark.gpu
@pytest.mark.parametrize("Lm", [70, 69])
def test_rhs3d_tile_variants_agree_on_one_grid(Lm):
    """sf_rhs3d on one square grid with every tile variant and every marching form
    (SF_TUNE_RHS_MARCH), bit-identical in FP64: an even row length (Lm = 70, I = 72) takes the
    paired staging, an odd one (I = 71) the element staging; both leave partial tiles on the
    east and north edges."""
    import numpy as np
    import torch
    from sailfish_b200 import configs
    from sailfish_b200._lib import lib
    from sailfish_b200.model import Model, stream_handle
    cfg = configs.basin(Lm, Lm, 8, 2.0e3, [(0.5, 0.5)], dt=120.0, ndtfast=10)
    g = cfg["grid"]
    bump = 1e-3 * np.exp(-((g.x - g.x.max() / 2) ** 2 + (g.y - g.y.max() / 2) ** 2) / (2e4) ** 2)
    m = Model(g, cfg["boundary"], cfg["dt"], cfg["ndtfast"], precision="fp64")
    m.Zt_avg1.copy_(torch.from_numpy(bump.ravel()))
    m.step(2)
    p = m._p
    out = []
    for v in (0, 1, 2, 3, 4, 5, 6):
        assert lib.sf_ctx_set_tile(m.ctx.ptr, v if v < 4 else 0) == 0
        assert lib.sf_ctx_tune(m.ctx.ptr, 3, v - 3 if v >= 4 else 0) == 0
        m.ru.zero_()
        m.rv.zero_()
        assert lib.sf_rhs3d(m.ctx.ptr, p(m.u), p(m.v), p(m.Huon), p(m.Hvom), p(m.W), p(m.Hz),
                            p(m.ru), p(m.rv), stream_handle()) == 0
        torch.cuda.synchronize()
        out.append((m.ru.cpu().numpy(), m.rv.cpu().numpy()))
    assert np.isfinite(out[0][0]).all() and np.abs(out[0][0]).max() > 0
    for o in out[1:]:
        np.testing.assert_array_equal(o[0], out[0][0])
        np.testing.assert_array_equal(o[1], out[0][1])
