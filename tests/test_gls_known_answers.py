"""GLS closure against closed-form answers of its own equations (an external pin for a closure
the reference has only as pseudo-code, nonlinear/gls_corrector_step.py).

With the turbulent diffusion switched off (sigma_k = sigma_psi = 1e8) every level of a column
is a homogeneous turbulence problem, for which the generic length-scale equations (Umlauf and
Burchard 2003, J. Mar. Res. 61; psi = cmu0^p k^m l^n) have exact solutions:

* homogeneous shear (constant S, no stratification): k and psi grow exponentially in a
  structural equilibrium with P/eps = (c2 - m - n/2) / (c1 - m - n/2); for k-epsilon that is
  the classical (C_eps2 - 1)/(C_eps1 - 1) = 2.091 (Pope, Turbulent Flows, 2000, sec. 10.4.3);
  with the stability function of the corrector (Galperin et al. 1988, neutral Sm) the shear
  parameter S k / eps follows from P = nu_t S^2, nu_t = sqrt(2) Sm cmu0^3 k^2 / eps;
* homogeneous decay (no shear, no stratification): k ~ t^(-a) with
  a = -n / (c2 - m - n/2) (k-epsilon: 1/(C_eps2 - 1) = 1.087).

The implicit time stepping of the corrector converges to these as dt/(k/eps) -> 0; the
tolerances below hold at the stated time steps.  The oracle (CPU) and the CUDA kernel (GPU,
FP64) are both checked against the closed forms.
"""
import numpy as np
import pytest

import gls_oracle as go

MODELS = ("k-epsilon", "k-omega", "gen")
SM0 = go.MY_SM3          # Galperin's neutral Sm (Gh = 0)


def shear_ratio(P):
    g = P["m"] + 0.5 * P["n"]
    return (P["c2"] - g) / (P["c1"] - g)


def decay_exponent(P):
    return -P["n"] / (P["c2"] - P["m"] - 0.5 * P["n"])


def column(model, shear, N=4, H=100.0, I=3):
    """Identical columns on an I x I rho grid (I = 3: one interior column, (i, j) = (1, 1))."""
    P = dict(go.PRESETS[model], sigk=1e8, sigp=1e8, rdrag2=0.0)
    J = I
    s2 = I * J
    zw = np.linspace(-H, 0.0, N + 1)
    zr = 0.5 * (zw[1:] + zw[:-1])
    u = np.zeros((N + 1, s2))
    u[:N] = (shear * (zr + H))[:, None]
    c = dict(I=I, J=J, N=N, u=u, v=np.zeros((N + 1, s2)), z_r=np.repeat(zr[:, None], s2, 1),
             Hz=np.repeat(np.diff(zw)[:, None], s2, 1), bvf=np.zeros((N + 1, s2)),
             sustr=np.zeros(s2), svstr=np.zeros(s2))
    k0, L0 = 1.0e-4, 1.0
    c["tke"] = np.full((N + 1, s2), k0)
    c["Lscale"] = np.full((N + 1, s2), L0)
    c["gls"] = P["cmu0"] ** P["p"] * c["tke"] ** P["m"] * c["Lscale"] ** P["n"]
    for k in ("Akv", "Akt", "Akk", "Akp"):
        c[k] = np.full((N + 1, s2), 1e-5)
    return P, c


FIELDS = ("tke", "gls", "Akv", "Akt", "Akk", "Akp", "Lscale")


def eps_of(P, k, L):
    return P["cmu0"] ** 3 * k ** 1.5 / L


def oracle_steps(P, c, dt, n, every=None):
    st = [c[f] for f in FIELDS]
    hist = []
    for it in range(n):
        st = list(go.gls_corrector(P, dt, c["I"], c["J"], c["N"], c["u"], c["v"], c["z_r"], c["Hz"],
                                   c["bvf"], c["sustr"], c["svstr"], *st))
        if every and (it + 1) % every == 0:
            hist.append((it + 1, st[0].copy(), st[6].copy(), st[2].copy()))
    return dict(zip(FIELDS, st)), hist


@pytest.mark.parametrize("model", MODELS)
def test_oracle_homogeneous_shear_equilibrium(model):
    S = 0.01
    P, c = column(model, S)
    out, _ = oracle_steps(P, c, 1.0, 3000)
    m = 4                         # the interior column, mid-depth W level 2
    k, L, Akv = out["tke"][2, m], out["Lscale"][2, m], out["Akv"][2, m]
    eps = eps_of(P, k, L)
    ratio = (Akv - P["Akv_bak"]) * S * S / eps
    assert abs(ratio / shear_ratio(P) - 1.0) < 5e-3, (ratio, shear_ratio(P))
    skeps = np.sqrt(shear_ratio(P) / (np.sqrt(2.0) * SM0 * P["cmu0"] ** 3))
    assert abs(S * k / eps / skeps - 1.0) < 5e-3, (S * k / eps, skeps)


@pytest.mark.parametrize("model", MODELS)
def test_oracle_homogeneous_decay_exponent(model):
    P, c = column(model, 0.0)
    P["Kmin"] = 1e-30             # let k decay far below the floor of the ocean presets
    P["Pmin"] = 1e-300
    _, hist = oracle_steps(P, c, 2.0, 6000, every=1000)
    t = np.array([h[0] for h in hist], float) * 2.0
    k = np.array([h[1][2, 4] for h in hist])
    # late-time slope of log k against log(t + t0), t0 fitted from the first two samples'
    # decay rate: with k ~ (1 + t/t0)^-a, d ln k / dt = -a / (t0 + t)
    a = decay_exponent(P)
    rate = -np.diff(np.log(k)) / np.diff(t)        # ~ a / (t0 + t_mid)
    tm = 0.5 * (t[1:] + t[:-1])
    t0 = a / rate[-1] - tm[-1]
    slope = -np.diff(np.log(k[-3:])) / np.diff(np.log(t[-3:] + t0))
    assert np.all(np.abs(slope / a - 1.0) < 2e-2), (slope, a)


@pytest.mark.gpu
@pytest.mark.parametrize("model", MODELS)
def test_cuda_gls_homogeneous_shear_equilibrium(model):
    """The CUDA corrector in FP64, iterated on the device, against the same closed form."""
    import ctypes
    import torch
    from sailfish_b200 import host as Hm
    from sailfish_b200._lib import lib, check, GlsParams
    from sailfish_b200.model import Context, Grid
    S = 0.01
    P, c = column(model, S, N=6, I=6)      # the library's contexts need L, M >= 4 and N >= 5
    I, J, N = c["I"], c["J"], c["N"]
    sc_r, sc_w, Cs_r, Cs_w = Hm.set_coords(N, 4, 5.0, 0.4)
    z = np.zeros(I * J)
    grid = Grid(I - 1, J - 1, N, z + 100.0, z + 1e-3, z + 1e-3, z + 1.0, z + 1.0, z, sc_r, sc_w,
                Cs_r, Cs_w, 10.0, 2)
    ctx = Context(grid, Hm.Boundary(I - 1, J - 1), "fp64")
    T = {k: torch.tensor(np.ascontiguousarray(c[k]), dtype=torch.float64, device="cuda")
         for k in ("u", "v", "z_r", "Hz", "bvf", "sustr", "svstr") + FIELDS}
    prm = GlsParams(**{k: P[k] for k, _ in GlsParams._fields_})
    ptr = lambda t: ctypes.c_void_p(t.data_ptr())
    st = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    args = [ptr(T[k]) for k in ("u", "v", "z_r", "Hz", "bvf", "sustr", "svstr") + FIELDS]
    for _ in range(3000):
        check(lib.sf_gls_corrector(ctx.ptr, ctypes.byref(prm), 1.0, *args, st), "sf_gls_corrector")
    torch.cuda.synchronize()
    k, L, Akv = (float(T[f][3, 2 * I + 2]) for f in ("tke", "Lscale", "Akv"))
    eps = eps_of(P, k, L)
    ratio = (Akv - P["Akv_bak"]) * S * S / eps
    assert abs(ratio / shear_ratio(P) - 1.0) < 5e-3, (ratio, shear_ratio(P))
