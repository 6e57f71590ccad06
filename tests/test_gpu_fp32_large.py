"""The FP32 production form at sizes where every tiled kernel runs interior tiles.

Each FP32-only kernel (the fused predictor k_pred2d, the corrector's kernels, the paired-
staging k_rhs3d, the reciprocal-depth k_set_depth, k_maxflux_omega, the pipelined column solve
k_step3d_uv_pipe) runs on the same inputs as the FP64 path, whose results are bit-identical to
the reference's own kernels (tests/test_gpu_main3d.py, and the oracle comparison at this size
below).  Inputs are smooth fields of realistic magnitude rounded to FP32, so that both paths
start from identical values and the difference is the FP32 arithmetic alone.

Tolerances are relative to the largest magnitude of each FP64 output field (stated per
kernel in TOL); the measured errors are printed (pytest -s).  Grids: 200 x 200 x 32
(I = 202, an even row length: rhs3d's paired staging) and 199 x 199 x 32 (I = 201, odd: its
element staging), square because the reference's flat-index guards (the szJ guard of
computeMomentumPred) leave the interior on non-square grids.
"""
import ctypes

import numpy as np
import pytest

from golden_io import BND_KEYS

CASES = [200, 199]
N = 32

# max |FP32 - FP64| / max |FP64| per output, per kernel
TOL = {
    "set_depth": {"z_w": 2e-7, "z_r": 2e-7, "Hz": 5e-7},
    "maxflux_omega": {"Huon": 1e-6, "Hvom": 1e-6, "W": 2e-5},
    "rhs3d": {"ru": 2e-5, "rv": 2e-5},
    # the pressure-gradient tendencies difference FP32 surface elevations of neighbouring
    # nodes (cancellation: ~3e-5 of their scale on these smooth fields)
    "predictor": {"zeta2": 5e-6, "ubar2": 2e-5, "vbar2": 2e-5, "rzeta1": 1e-5, "rubar1": 1e-4,
                  "rvbar1": 1e-4},
    # vbar is reset to 0 after every substep (main3d.py:189), so DV_avg1 sums single-substep
    # increments of it and carries their FP32 relative error (3e-4 measured)
    "loop": {"zeta": 1e-4, "ubar": 5e-5, "Zt_avg1": 5e-5, "DU_avg1": 5e-5,
             "DV_avg1": 1e-3},
    "step3d_uv": {"u": 2e-5, "v": 2e-5, "ubar1": 2e-5, "vbar1": 2e-5},
    "step": {"zeta": 1e-4, "ubar": 1e-4, "u": 2e-4, "v": 2e-4, "W": 2e-4, "Zt_avg1": 1e-4},
}
MEASURED = {}


def _smooth(rng, shape, amp, levels=None):
    """A sum of a few random sinusoids over (j, i) (and a level profile), amplitude amp."""
    J, I = shape[-2], shape[-1]
    jj, ii = np.meshgrid(np.arange(J), np.arange(I), indexing="ij")
    f = np.zeros((J, I))
    for _ in range(4):
        kx, ky = rng.uniform(0.5, 4.0, 2) * 2 * np.pi / np.array([I, J])
        f += rng.uniform(-1, 1) * np.sin(kx * ii + ky * jj + rng.uniform(0, 2 * np.pi))
    f *= amp / max(np.abs(f).max(), 1e-30)
    if len(shape) == 2:
        return f
    k = np.arange(shape[0])[:, None, None]
    return f[None] * (0.6 + 0.4 * np.cos(np.pi * k / shape[0]))


def _f32(a):
    return np.asarray(a, np.float32).astype(np.float64)


def _inputs(Lm):
    from sailfish_b200 import configs
    cfg = configs.basin(Lm, Lm, N, 2.0e3, [(0.5, 0.6)], dt=240.0, ndtfast=30)
    g = cfg["grid"]
    rng = np.random.default_rng(Lm)
    J, I = g.J, g.I
    st = {}
    for n, amp in (("zeta", 0.05), ("ubar", 0.05), ("vbar", 0.05), ("rzeta", 1e-6),
                   ("rubar", 1e-2), ("rvbar", 1e-2)):
        st[n] = np.stack([_smooth(rng, (J, I), amp) for _ in range(3)])
    for n, amp in (("u", 0.1), ("v", 0.1), ("ru", 1e-2), ("rv", 1e-2)):
        st[n] = _smooth(rng, (N + 1, J, I), amp)
    st["AKv"] = 1e-3 + np.abs(_smooth(rng, (N + 1, J, I), 5e-3))
    st["Zt_avg1"] = _smooth(rng, (J, I), 0.05).ravel()
    st["DU_avg1"] = _smooth(rng, (J, I), 50.0 * 2e3).ravel()
    st["DV_avg1"] = _smooth(rng, (J, I), 50.0 * 2e3).ravel()
    return cfg, {k: _f32(v) for k, v in st.items()}


def _models(Lm):
    from sailfish_b200.model import Model
    cfg, st = _inputs(Lm)
    out = []
    for prec in ("fp64", "fp32"):
        m = Model(cfg["grid"], cfg["boundary"], cfg["dt"], cfg["ndtfast"], precision=prec)
        m.load(st)
        m.start()
        out.append(m)
    return out


def _sync(m64, m32, names):
    """The FP64 model takes the FP32 model's values of `names`, so that the next kernel starts
    from identical inputs."""
    for n in names:
        getattr(m64, n).copy_(getattr(m32, n).double())


def _compare(kernel, pairs, case):
    errs = {}
    for name, (a64, a32) in pairs.items():
        a64 = a64.double().cpu().numpy()
        a32 = a32.double().cpu().numpy()
        assert np.isfinite(a32).all(), "%s/%s: non-finite FP32 values" % (kernel, name)
        scale = np.abs(a64).max()
        assert scale > 0, "%s/%s: the FP64 field is zero (nothing compared)" % (kernel, name)
        errs[name] = float(np.abs(a32 - a64).max() / scale)
    MEASURED.setdefault(case, {})[kernel] = errs
    print("\n%s [%d]: %s" % (kernel, case, ", ".join("%s %.2e" % kv for kv in errs.items())))
    for name, e in errs.items():
        assert e <= TOL[kernel][name], "%s/%s: %.3g of field scale > %.1g" % (
            kernel, name, e, TOL[kernel][name])


@pytest.mark.gpu
@pytest.mark.parametrize("Lm", CASES)
def test_fp32_kernels_against_fp64_on_interior_tiles(Lm):
    import torch
    from sailfish_b200._lib import lib, check
    m64, m32 = _models(Lm)
    p = m64._p
    st = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    torch.cuda.synchronize()
    _compare("set_depth", {k: (getattr(m64, k), getattr(m32, k)) for k in ("z_w", "z_r", "Hz")}, Lm)

    _sync(m64, m32, ("z_w", "z_r", "Hz"))
    for m in (m64, m32):
        check(lib.sf_maxflux_omega(m.ctx.ptr, p(m.u), p(m.v), p(m.Huon), p(m.Hvom), p(m.Hz),
                                   p(m.W), p(m.z_w), None, None, None, st), "sf_maxflux_omega")
    torch.cuda.synchronize()
    _compare("maxflux_omega", {k: (getattr(m64, k), getattr(m32, k)) for k in ("Huon", "Hvom", "W")},
             Lm)

    _sync(m64, m32, ("Huon", "Hvom", "W"))
    for m in (m64, m32):
        check(lib.sf_rhs3d(m.ctx.ptr, p(m.u), p(m.v), p(m.Huon), p(m.Hvom), p(m.W), p(m.Hz),
                           p(m.ru), p(m.rv), st), "sf_rhs3d")
    torch.cuda.synchronize()
    _compare("rhs3d", {k: (getattr(m64, k), getattr(m32, k)) for k in ("ru", "rv")}, Lm)

    # one fused predictor (k_pred2d in FP32) from identical slots
    _sync(m64, m32, ("ru", "rv"))
    for m in (m64, m32):
        s = m.state2d()
        check(lib.sf_step2d_predictor(m.ctx.ptr, ctypes.byref(s), m.dtfast, 0.0, 0, st),
              "sf_step2d_predictor")
    torch.cuda.synchronize()
    assert lib.sf_ctx_fused_available(m32.ctx.ptr) == 1
    sl = lambda m, n, k: getattr(m, n)[m.slots[k]]
    _compare("predictor", {"zeta2": (sl(m64, "zeta", 2), sl(m32, "zeta", 2)),
                           "ubar2": (sl(m64, "ubar", 2), sl(m32, "ubar", 2)),
                           "vbar2": (sl(m64, "vbar", 2), sl(m32, "vbar", 2)),
                           "rzeta1": (sl(m64, "rzeta", 1), sl(m32, "rzeta", 1)),
                           "rubar1": (sl(m64, "rubar", 1), sl(m32, "rubar", 1)),
                           "rvbar1": (sl(m64, "rvbar", 1), sl(m32, "rvbar", 1))}, Lm)

    # the whole barotropic loop (graph replay: predictor, corrector kernels, boundary programs)
    _sync(m64, m32, m64.NAMES2)
    for m in (m64, m32):
        s = m.state2d()
        t2 = ctypes.c_double(0.0)
        check(lib.sf_barotropic_loop(m.ctx.ptr, ctypes.byref(s), m.nfast + 1,
                                     m._w1.ctypes.data_as(ctypes.POINTER(ctypes.c_double)),
                                     m.dtfast, ctypes.byref(t2), st), "sf_barotropic_loop")
        m._sync_slots(s)
    torch.cuda.synchronize()
    _compare("loop", {"zeta": (sl(m64, "zeta", 2), sl(m32, "zeta", 2)),
                      "ubar": (sl(m64, "ubar", 2), sl(m32, "ubar", 2)),
                      "Zt_avg1": (m64.Zt_avg1, m32.Zt_avg1), "DU_avg1": (m64.DU_avg1, m32.DU_avg1),
                      "DV_avg1": (m64.DV_avg1, m32.DV_avg1)}, Lm)

    # the column solve with the barotropic coupling and lateral BCs (k_step3d_uv_pipe in FP32)
    _sync(m64, m32, m64.NAMES2 + ("Zt_avg1", "DU_avg1", "DV_avg1"))
    for m in (m64, m32):
        m.set_depth()
    torch.cuda.synchronize()
    _sync(m64, m32, ("z_w", "z_r", "Hz"))
    for m in (m64, m32):
        check(lib.sf_step3d_uv_bc(m.ctx.ptr, p(m.u), p(m.v), p(m.ru), p(m.rv),
                                  p(sl(m, "ubar", 1)), p(sl(m, "vbar", 1)), p(sl(m, "ubar", 2)),
                                  p(sl(m, "vbar", 2)), p(m.Hz), p(m.AKv), p(m.z_r),
                                  p(m.DU_avg1), p(m.DV_avg1), 3, 0, 1.0, m.dt, 0.0, st),
              "sf_step3d_uv_bc")
    torch.cuda.synchronize()
    _compare("step3d_uv", {"u": (m64.u, m32.u), "v": (m64.v, m32.v),
                           "ubar1": (sl(m64, "ubar", 1), sl(m32, "ubar", 1)),
                           "vbar1": (sl(m64, "vbar", 1), sl(m32, "vbar", 1))}, Lm)


@pytest.mark.gpu
@pytest.mark.parametrize("Lm", CASES)
def test_fp32_step_against_fp64(Lm):
    """One whole baroclinic step (all phases in the production order) from identical inputs."""
    import torch
    m64, m32 = _models(Lm)
    for m in (m64, m32):
        m.step(1)
    torch.cuda.synchronize()
    sl = lambda m, n: getattr(m, n)[m.slots[2]]
    _compare("step", {"zeta": (sl(m64, "zeta"), sl(m32, "zeta")),
                      "ubar": (sl(m64, "ubar"), sl(m32, "ubar")),
                      "u": (m64.u, m32.u), "v": (m64.v, m32.v), "W": (m64.W, m32.W),
                      "Zt_avg1": (m64.Zt_avg1, m32.Zt_avg1)}, Lm)


@pytest.mark.gpu
def test_fp64_step_bit_exact_against_the_oracle_at_size():
    """The FP64 path at 200 x 200 x 32 (interior tiles everywhere) against the oracle's
    restatement of the reference, one whole step from the same smooth state, bit for bit."""
    import torch
    import oracle as orc
    from sailfish_b200 import host
    from sailfish_b200.model import Model
    cfg, st = _inputs(200)
    g = cfg["grid"]
    m = Model(g, cfg["boundary"], cfg["dt"], cfg["ndtfast"], precision="fp64")
    m.load(st)
    m.step(1)
    torch.cuda.synchronize()
    s = m.state()

    og = orc.Grid(g.L, g.M, g.N, g.h, g.pm, g.pn, g.on_u, g.om_v, g.fomn, g.sc_r, g.sc_w,
                  g.Cs_r, g.Cs_w, g.hc, g.Vtransform)
    init = dict(st)
    for n in ("u", "v", "ru", "rv"):
        parent = np.zeros((3,) + st[n].shape)
        parent[2] = st[n]
        init[n] = parent
    O = orc.Ocean(og, init)
    B = cfg["boundary"]
    bd = {}
    for name in ("zetaBC", "ubarBC", "vbarBC", "uvelBC", "vvelBC"):
        for f in ("bcIdx", "bcIdx1", "bcIdx2", "bcIdxFieldIdx2", "bcIdxFieldType", "LBC"):
            bd["%s_%s" % (name, f)] = getattr(getattr(B, name), f)
    for f in BND_KEYS:
        bd[f] = getattr(B, f)
    nfast, w1, w2 = host.set_weights(cfg["ndtfast"])
    ct = orc.CompTimes(cfg["dt"], cfg["ndtfast"], nfast, w1, w2)
    orc.main3d(og, orc.Boundary(bd), O, ct, 1)
    for n in ("zeta", "ubar", "vbar", "Zt_avg1", "DU_avg1", "DV_avg1", "W", "AKv"):
        a = getattr(O, n)
        if n in O.NAMES2:
            a = np.stack([a[O.slots[n][k]] for k in range(3)])
            b = np.stack([s[n][s["slots"][k]] for k in range(3)])
        else:
            b = s[n]
        np.testing.assert_array_equal(b.reshape(-1), a.reshape(-1), err_msg=n)
    for n in ("u", "v", "ru", "rv"):
        np.testing.assert_array_equal(s[n].reshape(-1), O.t3(n), err_msg=n)
    for n in ("z_w", "z_r", "Hz"):
        np.testing.assert_array_equal(s[n].reshape(-1), getattr(og, n).reshape(-1), err_msg=n)


@pytest.mark.gpu
@pytest.mark.parametrize("Lm", CASES)
def test_column_solve_bulk_and_element_staging_agree(Lm):
    """The FP32 column solve with its levels staged by bulk copies (cp.async.bulk, interior
    tiles), by 16-byte cp.async of the same spans (the default) and by per-element cp.async:
    identical results."""
    import torch
    from sailfish_b200._lib import lib, check
    out = []
    for bulk, vec in ((1, 0), (0, 1), (0, 0)):
        _, m = _models(Lm)
        assert lib.sf_ctx_set_bulk(m.ctx.ptr, bulk) == 0
        assert lib.sf_ctx_tune(m.ctx.ptr, 2, vec) == 0
        p = m._p
        st = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
        sl = lambda n, k: getattr(m, n)[m.slots[k]]
        check(lib.sf_step3d_uv_bc(m.ctx.ptr, p(m.u), p(m.v), p(m.ru), p(m.rv), p(sl("ubar", 1)),
                                  p(sl("vbar", 1)), p(sl("ubar", 2)), p(sl("vbar", 2)), p(m.Hz),
                                  p(m.AKv), p(m.z_r), p(m.DU_avg1), p(m.DV_avg1), 3, 0, 1.0, m.dt,
                                  0.0, st), "sf_step3d_uv_bc")
        m.check_state()            # also reports a bounded wait that gave up
        torch.cuda.synchronize()
        out.append([t.cpu().numpy() for t in (m.u, m.v, sl("ubar", 1), sl("vbar", 1))])
    for o in out[1:]:
        for a, b in zip(out[0], o):
            np.testing.assert_array_equal(a, b)


@pytest.mark.gpu
@pytest.mark.parametrize("precision", ["fp64", "fp32"])
@pytest.mark.parametrize("Lm", CASES)
def test_rhs3d_marching_and_tiled_forms_agree(precision, Lm):
    """sf_rhs3d in its tiled form and its three marching forms (SF_TUNE_RHS_MARCH) on grids
    with interior tiles on every side (I = 202: 16-byte chunk staging in FP32, else pairs;
    I = 201: element staging; SF_TUNE_RHS_CHUNKS switches the chunks off), the
    fluxes and W from sf_maxflux_omega: identical ru and rv in FP64 (built without FMA
    contraction); in FP32 the forms may contract different products into FMAs, so they agree
    to a few units of FP32 rounding of each field's scale."""
    import torch
    from sailfish_b200._lib import lib, check
    m64, m32 = _models(Lm)
    m = m64 if precision == "fp64" else m32
    p = m._p
    st = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    check(lib.sf_maxflux_omega(m.ctx.ptr, p(m.u), p(m.v), p(m.Huon), p(m.Hvom), p(m.Hz),
                               p(m.W), p(m.z_w), None, None, None, st), "sf_maxflux_omega")
    out, staged = [], {}
    for mv, ch in ((0, 1), (1, 1), (2, 1), (3, 1), (1, 0), (2, 0), (3, 0)):
        assert lib.sf_ctx_tune(m.ctx.ptr, 3, mv) == 0
        assert lib.sf_ctx_tune(m.ctx.ptr, 4, ch) == 0
        for t in (m.ru, m.rv):
            t.fill_(7.0)
        check(lib.sf_rhs3d(m.ctx.ptr, p(m.u), p(m.v), p(m.Huon), p(m.Hvom), p(m.W), p(m.Hz),
                           p(m.ru), p(m.rv), st), "sf_rhs3d")
        torch.cuda.synchronize()
        out.append([t.cpu().numpy() for t in (m.ru, m.rv)])
        staged[mv, ch] = out[-1]
    assert lib.sf_ctx_tune(m.ctx.ptr, 3, 0) == 0
    assert lib.sf_ctx_tune(m.ctx.ptr, 4, 1) == 0
    assert lib.sf_ctx_tune(m.ctx.ptr, 4, 2) != 0
    # the staging (16-byte chunks in FP32 where aligned, else pairs or elements) moves the same
    # values: the marching forms' results do not depend on it
    for mv in (1, 2, 3):
        for a, b in zip(staged[mv, 1], staged[mv, 0]):
            np.testing.assert_array_equal(a, b)
    assert np.abs(m.W.cpu().numpy()).max() > 0
    assert np.abs(out[0][0]).max() > 0 and np.abs(out[0][1]).max() > 0
    for o in out[1:]:
        for a, b in zip(out[0], o):
            if precision == "fp64":
                np.testing.assert_array_equal(a, b)
            else:
                assert np.abs(b - a).max() <= 4e-6 * np.abs(a).max()
    assert lib.sf_ctx_tune(m.ctx.ptr, 3, 4) != 0


@pytest.mark.gpu
@pytest.mark.parametrize("precision", ["fp64", "fp32"])
def test_maxflux_omega_chunk_variants_agree(precision):
    """The fused set_maxflux/omega kernel with its interior columns' loads issued one level at a
    time and in chunks of 4, 5 and 8 levels (sf_ctx_tune): identical fluxes and W in FP64 (built
    without FMA contraction); in FP32 the variants' code may contract different products into
    FMAs, so they agree to a few units of FP32 rounding of each field's scale."""
    import torch
    from sailfish_b200._lib import lib, check
    m64, m32 = _models(199)
    m = m64 if precision == "fp64" else m32
    p = m._p
    st = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    out = []
    for ch in (0, 4, 5, 8):
        assert lib.sf_ctx_tune(m.ctx.ptr, 0, ch) == 0
        for t in (m.Huon, m.Hvom, m.W):
            t.zero_()
        check(lib.sf_maxflux_omega(m.ctx.ptr, p(m.u), p(m.v), p(m.Huon), p(m.Hvom), p(m.Hz),
                                   p(m.W), p(m.z_w), None, None, None, st), "sf_maxflux_omega")
        torch.cuda.synchronize()
        out.append([t.cpu().numpy() for t in (m.Huon, m.Hvom, m.W)])
    assert np.abs(out[0][2]).max() > 0
    for o in out[1:]:
        for a, b in zip(out[0], o):
            if precision == "fp64":
                np.testing.assert_array_equal(a, b)
            else:
                assert np.abs(b - a).max() <= 4e-6 * np.abs(a).max()
    assert lib.sf_ctx_tune(m.ctx.ptr, 0, 3) != 0


@pytest.mark.gpu
@pytest.mark.parametrize("precision", ["fp64", "fp32"])
def test_fused_predictor_pair_and_scalar_forms_agree(precision):
    """The fused barotropic predictor's paired form (two nodes per thread, vector loads; taken
    on grids with an even row length, 202 here) and its scalar form, through one whole step
    from the same smooth state: identical in FP64; in FP32 the two forms' code may contract
    products into FMAs differently, so they agree to FP32 rounding of each field's scale
    (measured: rzeta 4.4e-5 and rvbar 2.3e-4, differences of nearly equal terms)."""
    import torch
    from sailfish_b200._lib import lib
    from sailfish_b200.model import Model
    cfg, st = _inputs(200)
    out = []
    for pair in (0, 1, 2):      # scalar, paired (16-row and 8-row blocks)
        m = Model(cfg["grid"], cfg["boundary"], cfg["dt"], cfg["ndtfast"], precision=precision)
        assert lib.sf_ctx_tune(m.ctx.ptr, 1, pair) == 0
        m.load(st)
        m.step(1)
        torch.cuda.synchronize()
        out.append(m.state())
        del m
    names = ("zeta", "ubar", "vbar", "rzeta", "rubar", "rvbar", "Zt_avg1", "DU_avg1", "DV_avg1",
             "u", "v", "W")
    for o in out[1:]:
        assert out[0]["slots"] == o["slots"]
        for n in names:
            a, b = out[0][n], o[n]
            assert np.isfinite(b).all(), n
            if precision == "fp64":
                np.testing.assert_array_equal(b, a, err_msg=n)
            else:
                # the right-hand sides difference nearly equal fluxes and pressure terms;
                # DV_avg1 sums single-substep vbar increments (as in the loop's tolerance)
                tol = {"rzeta": 5e-4, "rubar": 5e-4, "rvbar": 5e-4, "DV_avg1": 1e-3}.get(n, 1e-4)
                err = np.abs(b - a).max() / np.abs(a).max()
                assert err <= tol, (n, err)
