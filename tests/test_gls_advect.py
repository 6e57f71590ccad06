"""GLS corrector's advective terms (nonlinear/gls_corrector_step.py:172-388) and the corrector
started from the advected new level: oracle properties on the CPU, CUDA against the oracle on
the GPU (FP64 within 1e-12 relative, the chain through the corrector within 1e-9 as the
corrector's own test; FP32 within the stated tolerances)."""
import ctypes

import numpy as np
import pytest

import gls_oracle as go
from gls_case import make

FIELDS = ("tke", "gls", "Akv", "Akt", "Akk", "Akp", "Lscale")


def fluxes(c, seed=11):
    """W-level-compatible U/V fluxes (rho levels, N+1 allocated) and W for the gls_case basin
    (pm = pn = 1e-3): Huon ~ u Hz dy, Hvom ~ v Hz dx, W of either sign."""
    rng = np.random.default_rng(seed)
    N, s2 = c["N"], c["I"] * c["J"]
    Huon = np.zeros((N + 1, s2))
    Hvom = np.zeros((N + 1, s2))
    Huon[:N] = c["u"][:N] * c["Hz"] * 1.0e3
    Hvom[:N] = c["v"][:N] * c["Hz"] * 1.0e3
    W = 30.0 * rng.standard_normal((N + 1, s2))
    W[0] = 0.0
    W[N] = 0.0
    return Huon, Hvom, W


def interior_mask(I, J):
    idx = np.arange(I * J)
    i, j = idx % I, idx // I
    return (i != 0) & (i != I - 1) & (j != 0) & (j != J - 1)


def test_advect_oracle_keeps_a_constant_in_a_nondivergent_flow():
    c = make()
    I, J, N = c["I"], c["J"], c["N"]
    s2 = I * J
    q = np.full((N + 1, s2), 3e-4)
    Huon = np.tile(np.linspace(-2.0, 3.0, N + 1)[:, None], (1, s2))   # uniform along i and j
    Hvom = np.tile(np.linspace(1.0, -1.0, N + 1)[:, None], (1, s2))
    W = np.full((N + 1, s2), 5.0)                                      # uniform in k
    new = np.full((N + 1, s2), 7e-4)
    pm = np.full(s2, 1e-3)
    t, g = go.gls_advect(240.0, I, J, N, pm, pm, Huon, Hvom, W, q, q, new, new, 1e-9, 1e-12)
    np.testing.assert_allclose(t, new, rtol=1e-12)
    np.testing.assert_allclose(g, new, rtol=1e-12)


def test_advect_oracle_linear_field_is_exact():
    """Third-order upstream fluxes of a field linear in i under a uniform eastward flux: the
    curvature vanishes (edge differences repeated), so the divergence is XF * slope."""
    I, J, N = 12, 7, 5
    s2 = I * J
    ii = np.arange(s2) % I
    q = np.tile((1e-4 + 2e-6 * ii)[None, :], (N + 1, 1))
    XF = 40.0
    Huon = np.full((N + 1, s2), XF)
    Hvom = np.zeros((N + 1, s2))
    W = np.zeros((N + 1, s2))
    new = np.full((N + 1, s2), 5e-3)
    pm = np.full(s2, 1e-3)
    dt = 100.0
    t, _ = go.gls_advect(dt, I, J, N, pm, pm, Huon, Hvom, W, q, q, new, new, 1e-9, 1e-12)
    m = interior_mask(I, J)
    np.testing.assert_allclose(t[1:N][:, m], 5e-3 - dt * 1e-6 * XF * 2e-6, rtol=1e-12)
    np.testing.assert_array_equal(t[:, ~m], new[:, ~m])     # edges untouched
    np.testing.assert_array_equal(t[0], new[0])             # bottom and surface untouched
    np.testing.assert_array_equal(t[N], new[N])


def test_advect_oracle_floors():
    c = make()
    I, J, N = c["I"], c["J"], c["N"]
    s2 = I * J
    Huon, Hvom, W = fluxes(c)
    pm = np.full(s2, 1e-3)
    tiny = np.full((N + 1, s2), 1e-12)
    t, g = go.gls_advect(240.0, I, J, N, pm, pm, 1e3 * Huon, 1e3 * Hvom, 1e3 * W, c["tke"],
                         c["gls"], tiny, tiny, 7.6e-6, 1e-12)
    m = interior_mask(I, J)
    assert np.all(t[1:N][:, m] >= 7.6e-6) and np.any(t[1:N][:, m] == 7.6e-6)
    assert np.all(g[1:N][:, m] >= 1e-12)


def test_corrector_oracle_default_start_is_hz_times_nstp():
    c = make()
    N = c["N"]
    Hzw = np.zeros_like(c["tke"])
    Hzw[1:N] = 0.5 * (c["Hz"][:-1] + c["Hz"][1:])
    base = go.gls_corrector(go.DEFAULT, 240.0, c["I"], c["J"], N, c["u"], c["v"], c["z_r"],
                            c["Hz"], c["bvf"], c["sustr"], c["svstr"], c["tke"], c["gls"],
                            c["Akv"], c["Akt"], c["Akk"], c["Akp"], c["Lscale"])
    same = go.gls_corrector(go.DEFAULT, 240.0, c["I"], c["J"], N, c["u"], c["v"], c["z_r"],
                            c["Hz"], c["bvf"], c["sustr"], c["svstr"], c["tke"], c["gls"],
                            c["Akv"], c["Akt"], c["Akk"], c["Akp"], c["Lscale"],
                            tke_nnew=Hzw * c["tke"], gls_nnew=Hzw * c["gls"])
    for a, b in zip(base, same):
        np.testing.assert_array_equal(a, b)


# ---- on the GPU -------------------------------------------------------------------------------
class Gpu:
    """The gls_case basin on a context of the given precision, with device copies of fields."""

    def __init__(self, c, precision):
        import torch
        from sailfish_b200 import host as H
        from sailfish_b200._lib import GlsParams
        from sailfish_b200.model import Context, Grid
        self.torch = torch
        I, J, N = c["I"], c["J"], c["N"]
        L, M = I - 1, J - 1
        z = np.zeros(I * J)
        grid = Grid(L, M, N, c["h"], z + 1e-3, z + 1e-3, z + 1.0, z + 1.0, z, c["sc_r"],
                    c["sc_w"], c["Cs_r"], c["Cs_w"], c["hc"], 2)
        self.ctx = Context(grid, H.Boundary(L, M), precision)
        self.dt_ = torch.float64 if precision == "fp64" else torch.float32
        self.P = GlsParams(**{k: go.DEFAULT[k] for k, _ in GlsParams._fields_})
        self.shape = (N + 1, I * J)

    def t(self, a):
        return self.torch.tensor(np.ascontiguousarray(a), dtype=self.dt_, device="cuda")

    def zeros(self):
        return self.torch.zeros(self.shape, dtype=self.dt_, device="cuda")

    @staticmethod
    def p(t):
        return ctypes.c_void_p(t.data_ptr())

    def stream(self):
        return ctypes.c_void_p(self.torch.cuda.current_stream().cuda_stream)

    @staticmethod
    def host(t):
        return t.double().cpu().numpy()


def gpu_advect(g, dt, Huon, Hvom, W, t3, g3, tn, gn):
    from sailfish_b200._lib import lib, check
    check(lib.sf_gls_advect(g.ctx.ptr, ctypes.byref(g.P), dt, go.GADV, g.p(Huon), g.p(Hvom),
                            g.p(W), g.p(t3), g.p(g3), g.p(tn), g.p(gn), g.stream()),
          "sf_gls_advect")


@pytest.mark.gpu
@pytest.mark.parametrize("precision,rtol", [("fp64", 1e-12), ("fp32", 2e-4)])
def test_gls_advect_matches_oracle(precision, rtol):
    c = make()
    I, J, N = c["I"], c["J"], c["N"]
    Huon, Hvom, W = fluxes(c)
    Hzw = np.ones_like(c["tke"])
    Hzw[1:N] = 0.5 * (c["Hz"][:-1] + c["Hz"][1:])
    tn0, gn0 = Hzw * c["tke"], Hzw * c["gls"]
    t3 = c["tke"] * (1.0 + 0.3 * np.sin(np.arange(c["tke"].size)).reshape(c["tke"].shape))
    g3 = c["gls"] * (1.0 + 0.3 * np.cos(np.arange(c["gls"].size)).reshape(c["gls"].shape))
    pm = np.full(I * J, 1e-3)
    ref = go.gls_advect(240.0, I, J, N, pm, pm, Huon, Hvom, W, t3, g3, tn0, gn0,
                        go.DEFAULT["Kmin"], go.DEFAULT["Pmin"])
    g = Gpu(c, precision)
    d = {k: g.t(a) for k, a in dict(Huon=Huon, Hvom=Hvom, W=W, t3=t3, g3=g3, tn=tn0,
                                    gn=gn0).items()}
    gpu_advect(g, 240.0, d["Huon"], d["Hvom"], d["W"], d["t3"], d["g3"], d["tn"], d["gn"])
    g.torch.cuda.synchronize()
    for name, r in zip(("tn", "gn"), ref):
        got = g.host(d[name])
        np.testing.assert_allclose(got, r, rtol=rtol, atol=rtol * np.abs(r[1:N]).max() * 1e-2,
                                   err_msg=name)
    # the advection moved something: the result is not the start
    assert np.abs(ref[0] - tn0).max() > 1e-3 * np.abs(tn0[1:N]).max()


def gpu_chain(c, precision, dt=240.0, advect=True):
    """sf_gls_predictor (first step) -> sf_gls_advect -> sf_gls_corrector_nnew."""
    from sailfish_b200._lib import lib, check
    g = Gpu(c, precision)
    Huon, Hvom, W = fluxes(c)
    d = {k: g.t(c[k]) for k in ("u", "v", "z_r", "Hz", "bvf", "sustr", "svstr") + FIELDS}
    d.update(Huon=g.t(Huon), Hvom=g.t(Hvom), W=g.t(W))
    t3, g3, tn, gn, hh = (g.zeros() for _ in range(5))
    check(lib.sf_gls_predictor(g.ctx.ptr, dt, 1, g.p(d["Huon"]), g.p(d["Hvom"]), g.p(d["W"]),
                               g.p(d["Hz"]), g.p(d["tke"]), g.p(d["tke"]), g.p(t3), g.p(tn),
                               g.p(d["gls"]), g.p(d["gls"]), g.p(g3), g.p(gn), g.p(hh),
                               g.stream()), "sf_gls_predictor")
    if advect:
        gpu_advect(g, dt, d["Huon"], d["Hvom"], d["W"], t3, g3, tn, gn)
    check(lib.sf_gls_corrector_nnew(
        g.ctx.ptr, ctypes.byref(g.P), dt, *[g.p(d[k]) for k in
                                            ("u", "v", "z_r", "Hz", "bvf", "sustr", "svstr")],
        g.p(tn), g.p(gn), *[g.p(d[k]) for k in FIELDS], g.stream()), "sf_gls_corrector_nnew")
    g.torch.cuda.synchronize()
    return {k: g.host(d[k]) for k in FIELDS}


def oracle_chain(c, dt=240.0):
    I, J, N = c["I"], c["J"], c["N"]
    Huon, Hvom, W = fluxes(c)
    pm = np.full(I * J, 1e-3)
    t3, g3, tn, gn, _ = go.gls_prestep(dt, True, I, J, N, pm, pm, Huon, Hvom, W, c["Hz"],
                                       c["tke"], c["tke"], c["gls"], c["gls"])
    tn, gn = go.gls_advect(dt, I, J, N, pm, pm, Huon, Hvom, W, t3, g3, tn, gn,
                           go.DEFAULT["Kmin"], go.DEFAULT["Pmin"])
    out = go.gls_corrector(go.DEFAULT, dt, I, J, N, c["u"], c["v"], c["z_r"], c["Hz"], c["bvf"],
                           c["sustr"], c["svstr"], c["tke"], c["gls"], c["Akv"], c["Akt"],
                           c["Akk"], c["Akp"], c["Lscale"], tke_nnew=tn, gls_nnew=gn)
    return dict(zip(FIELDS, out))


@pytest.mark.gpu
def test_gls_chain_fp64_matches_oracle():
    c = make()
    ref = oracle_chain(c)
    got = gpu_chain(c, "fp64")
    for k in FIELDS:
        np.testing.assert_allclose(got[k], ref[k], rtol=1e-9, atol=0, err_msg=k)


@pytest.mark.gpu
def test_gls_chain_fp32_within_tolerance():
    c = make()
    ref = oracle_chain(c)
    got = gpu_chain(c, "fp32")
    m = interior_mask(c["I"], c["J"])
    for k in ("Akv", "Akt", "tke"):
        rel = np.abs(got[k][:, m] - ref[k][:, m]) / np.abs(ref[k][:, m])
        assert rel.max() < 2e-3, (k, rel.max())


@pytest.mark.gpu
def test_corrector_from_unadvected_level_is_the_plain_corrector():
    """sf_gls_corrector_nnew started from the predictor's Hz_w * tke (no advection) gives
    sf_gls_corrector's result bit for bit in FP64."""
    from test_gls import gpu_run
    c = make()
    plain = gpu_run(c, "fp64")
    got = gpu_chain(c, "fp64", advect=False)
    for k in FIELDS:
        np.testing.assert_array_equal(got[k], plain[k], err_msg=k)


def test_aliasing_is_refused():
    """The new level may not alias the old one (CPU: the check runs before any launch)."""
    from sailfish_b200._lib import lib, GlsParams
    P = GlsParams(**{k: go.DEFAULT[k] for k, _ in GlsParams._fields_})
    a = ctypes.c_void_p(0x1000)
    rc = lib.sf_gls_corrector_nnew(None, ctypes.byref(P), 1.0, *([None] * 7), a, a, a, a,
                                   *([None] * 5), None)
    assert rc != 0 and b"alias" in lib.sf_last_error()
    rc = lib.sf_gls_advect(None, ctypes.byref(P), 1.0, 1.0 / 3.0, None, None, None, a, a, a, a,
                           None)
    assert rc != 0 and b"distinct" in lib.sf_last_error()


@pytest.mark.gpu
def test_dropin_gls_predictor_then_corrector_matches_oracle():
    """dropin.gls_predictor_step then dropin.gls_corrector_step on reference-shaped state
    objects (torch CUDA arrays) run the advected chain."""
    import types

    import torch
    from sailfish_b200 import dropin
    c = make()
    I, J, N = c["I"], c["J"], c["N"]
    z = np.zeros(I * J)
    t = lambda a: torch.tensor(np.ascontiguousarray(a, np.float64), device="cuda")
    GRID = types.SimpleNamespace(L=I - 1, M=J - 1, N=N, h=c["h"], pm=z + 1e-3, pn=z + 1e-3,
                                 on_u=z + 1.0, om_v=z + 1.0, fomn=z, sc_r=c["sc_r"],
                                 sc_w=c["sc_w"], Cs_r=c["Cs_r"], Cs_w=c["Cs_w"], hc=c["hc"],
                                 Vtransform=2, z_r=t(c["z_r"]), Hz=t(c["Hz"]))
    dropin.initModule(GRID, None, precision="fp64")
    Huon, Hvom, W = fluxes(c)
    OCEAN = types.SimpleNamespace(Huon=t(Huon), Hvom=t(Hvom), W=t(W), u_t2=t(c["u"]),
                                  v_t2=t(c["v"]), AKv=t(c["Akv"]))
    MIXING = types.SimpleNamespace(**{k: t(c[k]) for k in ("tke", "gls", "Akt", "Akk", "Akp",
                                                           "Lscale", "bvf")})
    for k in ("tke_aux", "gls_aux", "tke_nnew", "gls_nnew", "Hz_half"):
        setattr(MIXING, k, torch.zeros((N + 1, I * J), dtype=torch.float64, device="cuda"))
    FORCES = types.SimpleNamespace(sustr=t(c["sustr"]), svstr=t(c["svstr"]))
    comp = types.SimpleNamespace(dt=240.0, iic=0, ntfirst=0)
    dropin.gls_predictor_step(comp, GRID, OCEAN, MIXING)
    dropin.gls_corrector_step(comp, GRID, OCEAN, MIXING, FORCES)
    torch.cuda.synchronize()
    ref = oracle_chain(c)
    got = dict(tke=MIXING.tke, gls=MIXING.gls, Akv=OCEAN.AKv, Akt=MIXING.Akt, Akk=MIXING.Akk,
               Akp=MIXING.Akp, Lscale=MIXING.Lscale)
    for k in FIELDS:
        np.testing.assert_allclose(got[k].cpu().numpy(), ref[k], rtol=1e-9, atol=0, err_msg=k)
