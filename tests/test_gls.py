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


def run_oracle(c, dt=240.0):
    return go.gls_corrector(go.DEFAULT, dt, c["I"], c["J"], c["N"], c["u"], c["v"], c["z_r"], c["Hz"],
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


def gpu_run(c, precision, dt=240.0):
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
    P = GlsParams(**{k: go.DEFAULT[k] for k, _ in GlsParams._fields_})
    ptr = lambda t: ctypes.c_void_p(t.data_ptr())
    check(lib.sf_gls_corrector(ctx.ptr, ctypes.byref(P), dt, *[ptr(T[k]) for k in
                               ("u", "v", "z_r", "Hz", "bvf", "sustr", "svstr") + FIELDS],
                               ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)),
          "sf_gls_corrector")
    torch.cuda.synchronize()
    return {k: T[k].double().cpu().numpy() for k in FIELDS}


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
