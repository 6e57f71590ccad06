"""GLS vertical-mixing corrector: oracle sanity on the CPU, CUDA against the oracle on the GPU.

The reference has no runnable GLS (its closure is untranslated ROMS Fortran), so the oracle
(oracle/gls_oracle.py) is a restatement of that pseudo-code: parity unpinned by reference
outputs, checked here for the properties the closure guarantees and used as the checker of
the CUDA kernel (FP64 within 1e-9 relative: pow/sqrt may differ in the last bit; FP32 within
the stated tolerance)."""
import numpy as np
import pytest

import gls_oracle as go
from gls_case import make

FIELDS = ("tke", "gls", "Akv", "Akt", "Akk", "Akp", "Lscale")


def run_oracle(c, dt=240.0, P=go.DEFAULT):
    return go.gls_corrector(P, dt, c["I"], c["J"], c["N"], c["u"], c["v"], c["z_r"], c["Hz"],
                            c["bvf"], c["sustr"], c["svstr"], c["tke"], c["gls"], c["Akv"], c["Akt"],
                            c["Akk"], c["Akp"], c["Lscale"])


def interior(c):
    I, J = c["I"], c["J"]
    idx = np.arange(I * J)
    i, j = idx % I, idx // I
    return idx[(i != 0) & (i != I - 1) & (j != 0) & (j != J - 1)]


def test_oracle_floors_and_boundaries():
    c = make()
    out = dict(zip(FIELDS, run_oracle(c)))
    col = interior(c)
    assert np.all(out["tke"][:, col] >= go.DEFAULT["Kmin"])
    assert np.all(out["gls"][:, col] >= go.DEFAULT["Pmin"])
    assert np.all(out["Akv"][:, col] >= go.DEFAULT["Akv_bak"])
    assert np.all(out["Akt"][:, col] >= go.DEFAULT["Akt_bak"])
    assert np.all(np.isfinite(out["Akv"]))
    # surface tke from the wind stress u*^2/cmu0^2 (gls_corrector_step.py:541-544)
    ustar2 = np.hypot(2 * c["sustr"][col], 2 * c["svstr"][col]) * 0.5
    np.testing.assert_allclose(out["tke"][-1, col], ustar2 / 0.5477 ** 2, rtol=1e-12)
    # columns outside the interior are untouched
    edge = np.setdiff1d(np.arange(c["I"] * c["J"]), col)
    np.testing.assert_array_equal(out["Akv"][:, edge], c["Akv"][:, edge])


def test_oracle_stronger_shear_mixes_more():
    c = make()
    base = dict(zip(FIELDS, run_oracle(c)))
    c2 = dict(c)
    c2["u"] = c["u"] * 3.0
    more = dict(zip(FIELDS, run_oracle(c2)))
    col = interior(c)
    assert np.mean(more["tke"][1:-1, col]) > np.mean(base["tke"][1:-1, col])


def gpu_run(c, precision, dt=240.0, preset=go.DEFAULT):
    import ctypes
    import torch
    from sailfish_b200 import host as H
    from sailfish_b200._lib import lib, check, GlsParams
    from sailfish_b200.model import Context, Grid
    I, J, N = c["I"], c["J"], c["N"]
    L, M = I - 1, J - 1
    z = np.zeros(I * J)
    grid = Grid(L, M, N, c["h"], z + 1e-3, z + 1e-3, z + 1.0, z + 1.0, z, c["sc_r"], c["sc_w"],
                c["Cs_r"], c["Cs_w"], c["hc"], 2)
    ctx = Context(grid, H.Boundary(L, M), precision)
    dt_ = torch.float64 if precision == "fp64" else torch.float32
    T = {k: torch.tensor(np.ascontiguousarray(c[k]), dtype=dt_, device="cuda")
         for k in ("u", "v", "z_r", "Hz", "bvf", "sustr", "svstr") + FIELDS}
    P = GlsParams(**{k: preset[k] for k, _ in GlsParams._fields_})
    ptr = lambda t: ctypes.c_void_p(t.data_ptr())
    check(lib.sf_gls_corrector(ctx.ptr, ctypes.byref(P), dt, *[ptr(T[k]) for k in
                               ("u", "v", "z_r", "Hz", "bvf", "sustr", "svstr") + FIELDS],
                               ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)),
          "sf_gls_corrector")
    torch.cuda.synchronize()
    return {k: T[k].double().cpu().numpy() for k in FIELDS}


def test_presets_match_between_library_and_oracle():
    """The library's named GLS models carry the oracle's constants."""
    from sailfish_b200 import closure
    for name in ("k-epsilon", "k-omega", "gen", "k-psi"):
        P = closure.gls_preset(name)
        for k, _ in type(P)._fields_:
            assert getattr(P, k) == go.PRESETS[name][k], (name, k)


@pytest.mark.parametrize("name", ["k-omega", "gen"])
def test_oracle_other_models_floors_and_surface(name):
    """Other GLS models in the oracle: finite coefficients above their backgrounds and floors,
    and the surface tke u*^2/cmu0^2 of each model's cmu0 (gls_corrector_step.py:541-544)."""
    P = go.PRESETS[name]
    c = make()
    out = dict(zip(FIELDS, run_oracle(c, P=P)))
    col = interior(c)
    assert np.all(np.isfinite(out["Akv"][:, col])) and np.all(np.isfinite(out["gls"][:, col]))
    assert np.all(out["tke"][:, col] >= P["Kmin"]) and np.all(out["gls"][:, col] >= P["Pmin"])
    assert np.all(out["Akv"][:, col] >= P["Akv_bak"]) and np.all(out["Akt"][:, col] >= P["Akt_bak"])
    ustar2 = np.hypot(2 * c["sustr"][col], 2 * c["svstr"][col]) * 0.5
    np.testing.assert_allclose(out["tke"][-1, col], ustar2 / P["cmu0"] ** 2, rtol=1e-12)


@pytest.mark.gpu
@pytest.mark.parametrize("name", ["k-omega", "gen"])
def test_gls_other_models_fp64_match_oracle(name):
    """The corrector kernel with the k-omega and generic (k-psi) constants: FP64 within 1e-9."""
    c = make()
    ref = dict(zip(FIELDS, run_oracle(c, P=go.PRESETS[name])))
    got = gpu_run(c, "fp64", preset=go.PRESETS[name])
    for k in FIELDS:
        np.testing.assert_allclose(got[k], ref[k], rtol=1e-9, atol=0, err_msg=k)


@pytest.mark.gpu
def test_gls_fp64_matches_oracle():
    c = make()
    ref = dict(zip(FIELDS, run_oracle(c)))
    got = gpu_run(c, "fp64")
    for k in FIELDS:
        np.testing.assert_allclose(got[k], ref[k], rtol=1e-9, atol=0, err_msg=k)


@pytest.mark.gpu
def test_gls_fp32_within_tolerance():
    c = make()
    ref = dict(zip(FIELDS, run_oracle(c)))
    got = gpu_run(c, "fp32")
    col = interior(c)
    for k in ("Akv", "Akt", "tke"):
        rel = np.abs(got[k][:, col] - ref[k][:, col]) / np.abs(ref[k][:, col])
        assert rel.max() < 2e-3, (k, rel.max())


# ---- GLS predictor (gls_predictor_step.py:18-216) -------------------------------------------
def predictor_case(I=13, J=9, N=8, seed=3):
    rng = np.random.default_rng(seed)
    s2 = I * J
    pm = 1.0 / (1000.0 * (1.0 + 0.2 * rng.random(s2)))
    pn = 1.0 / (1200.0 * (1.0 + 0.2 * rng.random(s2)))
    Hz = 5.0 + 3.0 * rng.random((N, s2))
    Huon = 200.0 * rng.standard_normal((N + 1, s2))
    Hvom = 200.0 * rng.standard_normal((N + 1, s2))
    W = 20.0 * rng.standard_normal((N + 1, s2))
    t0 = 1e-4 * (1.0 + rng.random((N + 1, s2)))
    ti = 1e-4 * (1.0 + rng.random((N + 1, s2)))
    g0 = 1e-7 * (1.0 + rng.random((N + 1, s2)))
    gi = 1e-7 * (1.0 + rng.random((N + 1, s2)))
    return dict(I=I, J=J, N=N, pm=pm, pn=pn, Hz=Hz, Huon=Huon, Hvom=Hvom, W=W, t0=t0, ti=ti,
                g0=g0, gi=gi)


def test_predictor_oracle_preserves_constants():
    """With a constant tke and no horizontal flux divergence the half step keeps the constant
    (the scheme is constancy preserving, gls_predictor_step.py:9-13)."""
    c = predictor_case()
    I, J, N = c["I"], c["J"], c["N"]
    s2 = I * J
    ones = np.full((N + 1, s2), 3e-4)
    Huon = np.tile(np.linspace(1.0, 2.0, N + 1)[:, None], (1, s2))   # uniform along i and j
    Hvom = np.zeros((N + 1, s2))
    W = np.zeros((N + 1, s2))
    t3, g3, tn, gn, hh = go.gls_prestep(60.0, False, I, J, N, c["pm"], c["pn"], Huon, Hvom, W,
                                        c["Hz"], ones, ones, ones, ones)
    a = t3.reshape(N + 1, J, I)[1:N, 1:J - 1, 1:I - 1]
    np.testing.assert_allclose(a, 3e-4, rtol=1e-12)


def gpu_predictor(c, precision, first):
    import ctypes
    import torch
    from sailfish_b200 import host as H
    from sailfish_b200._lib import lib, check
    from sailfish_b200.model import Context, Grid
    I, J, N = c["I"], c["J"], c["N"]
    L, M = I - 1, J - 1
    z = np.zeros(I * J)
    sc_r, sc_w, Cs_r, Cs_w = H.set_coords(N, 4, 5.0, 0.4)
    grid = Grid(L, M, N, z + 50.0, c["pm"], c["pn"], z + 1.0, z + 1.0, z, sc_r, sc_w, Cs_r,
                Cs_w, 10.0, 2)
    ctx = Context(grid, H.Boundary(L, M), precision)
    dt_ = torch.float64 if precision == "fp64" else torch.float32
    T = {k: torch.tensor(np.ascontiguousarray(c[k]), dtype=dt_, device="cuda")
         for k in ("Huon", "Hvom", "W", "Hz", "t0", "ti", "g0", "gi")}
    out = {k: torch.zeros((N + 1, I * J), dtype=dt_, device="cuda")
           for k in ("t3", "tn", "g3", "gn", "hh")}
    ptr = lambda t: ctypes.c_void_p(t.data_ptr())
    check(lib.sf_gls_predictor(ctx.ptr, 60.0, int(first), ptr(T["Huon"]), ptr(T["Hvom"]),
                               ptr(T["W"]), ptr(T["Hz"]), ptr(T["t0"]), ptr(T["ti"]),
                               ptr(out["t3"]), ptr(out["tn"]), ptr(T["g0"]), ptr(T["gi"]),
                               ptr(out["g3"]), ptr(out["gn"]), ptr(out["hh"]),
                               ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)),
          "sf_gls_predictor")
    torch.cuda.synchronize()
    return {k: v.double().cpu().numpy() for k, v in out.items()}


@pytest.mark.gpu
@pytest.mark.parametrize("first", [False, True])
@pytest.mark.parametrize("precision,rtol", [("fp64", 1e-12), ("fp32", 2e-4)])
def test_gls_predictor_matches_oracle(precision, rtol, first):
    c = predictor_case()
    ref = go.gls_prestep(60.0, first, c["I"], c["J"], c["N"], c["pm"], c["pn"], c["Huon"],
                         c["Hvom"], c["W"], c["Hz"], c["t0"], c["ti"], c["g0"], c["gi"])
    got = gpu_predictor(c, precision, first)
    N, s2 = c["N"], c["I"] * c["J"]
    for name, r in zip(("t3", "g3", "tn", "gn", "hh"), ref):
        g = got[name][1:N]
        np.testing.assert_allclose(g, r[1:N], rtol=rtol, atol=rtol * np.abs(r[1:N]).max(),
                                   err_msg=name)


@pytest.mark.gpu
def test_gls_on_a_column_list_matches_the_mask():
    """sf_gls_corrector_list over a compacted list gives the masked result exactly."""
    import ctypes
    import torch
    from sailfish_b200 import closure, configs
    from sailfish_b200.model import Model
    cfg = configs.small(24, 16, 12)
    out = []
    for use_list in (False, True):
        m = Model(cfg["grid"], cfg["boundary"], cfg["dt"], cfg["ndtfast"], precision="fp32")
        m.start()
        cols = closure.Columns(m)
        closure.wind_driven_state(m, cols, 0.1, 0.3, 500.0, np.random.default_rng(1))
        s2 = m.grid.s2
        sel = torch.zeros(s2, dtype=torch.uint8, device="cuda")
        sel[5::7] = 1
        if use_list:
            idx = torch.nonzero(sel).flatten().flip(0).to(torch.int32).contiguous()
            lst = torch.zeros(s2, dtype=torch.int32, device="cuda")
            lst[:idx.numel()] = idx
            cnt = torch.tensor([idx.numel()], dtype=torch.int32, device="cuda")
            cols.gls_step_list(lst, cnt)
        else:
            cols.gls_step(sel)
        torch.cuda.synchronize()
        out.append((m.AKv.clone(), cols.tke.clone(), cols.Akt.clone()))
    for a, b in zip(*out):
        torch.testing.assert_close(a, b, rtol=0, atol=0)
