"""obc_volcons (nonlinear/obc_volcons.py:6-69): boundary area/flux integrals in FP64 with
compensated sums, ubar_xs and the mass-conserving correction, against the oracle."""
import ctypes

import numpy as np
import pytest

import volcons_oracle as vo


def case(Lm=40, Mm=23, seed=0):
    rng = np.random.default_rng(seed)
    I, J = Lm + 2, Mm + 2
    s2 = I * J
    return dict(I=I, J=J, Lm=Lm, Mm=Mm, zeta=0.3 * rng.standard_normal(s2),
                h=50.0 + 4000.0 * rng.random(s2), ubar=0.2 * rng.standard_normal(s2),
                vbar=0.2 * rng.standard_normal(s2), on_u=1000.0 * (1.0 + rng.random(s2)),
                om_v=1500.0 * (1.0 + rng.random(s2)))


@pytest.mark.parametrize("edges", [1, 2, 4, 8, 5, 15])
def test_oracle_correction_closes_the_budget(edges):
    c = case()
    a, f, xs = vo.obc_volcons(c["I"], c["J"], c["zeta"], c["h"], c["ubar"], c["vbar"], c["on_u"],
                              c["om_v"], edges)
    u2, v2 = vo.conserve_mass(c["I"], c["J"], c["ubar"], c["vbar"], xs, edges)
    a2, f2, _ = vo.obc_volcons(c["I"], c["J"], c["zeta"], c["h"], u2, v2, c["on_u"], c["om_v"],
                               edges)
    assert a2 == a
    assert abs(f2) <= 1e-12 * (abs(f) + a * 0.2)


def gpu_volcons(c, precision, edges, correct):
    import torch
    from sailfish_b200 import host
    from sailfish_b200._lib import check, lib
    from sailfish_b200.model import Context, Grid
    I, J = c["I"], c["J"]
    L, M, N = I - 1, J - 1, 6
    sc_r, sc_w, Cs_r, Cs_w = host.set_coords(N, 4, 5.0, 0.4)
    z = np.zeros(I * J)
    grid = Grid(L, M, N, c["h"], z + 1e-3, z + 1e-3, c["on_u"], c["om_v"], z, sc_r, sc_w, Cs_r,
                Cs_w, 10.0, 2)
    ctx = Context(grid, host.Boundary(L, M), precision)
    dt = torch.float64 if precision == "fp64" else torch.float32
    T = {k: torch.tensor(c[k], dtype=dt, device="cuda") for k in ("zeta", "ubar", "vbar")}
    out = torch.zeros(3, dtype=torch.float64, device="cuda")
    p = lambda t: ctypes.c_void_p(t.data_ptr())
    check(lib.sf_obc_volcons(ctx.ptr, p(T["zeta"]), p(T["ubar"]), p(T["vbar"]), edges,
                             int(correct), p(out),
                             ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)),
          "sf_obc_volcons")
    torch.cuda.synchronize()
    return out.cpu().numpy(), T["ubar"].double().cpu().numpy(), T["vbar"].double().cpu().numpy()


@pytest.mark.gpu
@pytest.mark.parametrize("edges", [1, 2, 4, 8, 6, 15])
def test_volcons_fp64_matches_exact_sums(edges):
    c = case()
    a, f, xs = vo.obc_volcons(c["I"], c["J"], c["zeta"], c["h"], c["ubar"], c["vbar"], c["on_u"],
                              c["om_v"], edges)
    out, u2, v2 = gpu_volcons(c, "fp64", edges, True)
    # compensated FP64 sums: within a few ulps of the exact sums
    assert abs(out[0] - a) <= 4e-16 * abs(a)
    assert abs(out[1] - f) <= 1e-15 * (abs(f) + a * 0.2)
    assert abs(out[2] - xs) <= 1e-15 * (abs(xs) + 0.2)
    ru, rv = vo.conserve_mass(c["I"], c["J"], c["ubar"], c["vbar"], out[2], edges)
    np.testing.assert_array_equal(u2, ru)
    np.testing.assert_array_equal(v2, rv)
    _, f2, _ = vo.obc_volcons(c["I"], c["J"], c["zeta"], c["h"], u2, v2, c["on_u"], c["om_v"],
                              edges)
    assert abs(f2) <= 1e-12 * a


@pytest.mark.gpu
def test_volcons_fp32_fields_fp64_sums():
    c = case(seed=1)
    f32 = {k: (np.asarray(v, np.float32).astype(np.float64) if isinstance(v, np.ndarray) else v)
           for k, v in c.items()}
    f32["h"] = c["h"]               # the context keeps h in FP64
    a, f, xs = vo.obc_volcons(c["I"], c["J"], f32["zeta"], f32["h"], f32["ubar"], f32["vbar"],
                              f32["on_u"].astype(np.float32).astype(np.float64),
                              f32["om_v"].astype(np.float32).astype(np.float64), 15)
    out, _, _ = gpu_volcons(c, "fp32", 15, False)
    assert abs(out[0] - a) <= 1e-13 * a
    assert abs(out[2] - xs) <= 1e-12 * (abs(xs) + 0.2)


@pytest.mark.gpu
def test_closed_basin_has_no_open_edges():
    c = case(seed=2)
    out, u2, v2 = gpu_volcons(c, "fp64", 0, True)
    assert out[0] == 0.0 and out[1] == 0.0 and out[2] == 0.0
    np.testing.assert_array_equal(u2, c["ubar"])
