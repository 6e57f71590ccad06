"""GLS vertical-mixing corrector, restated in NumPy FP64 (TEST INFRASTRUCTURE: the oracle).

The reference has the GLS closure only as untranslated ROMS Fortran inside .py files that do
not parse (nonlinear/gls_corrector_step.py, nonlinear/gls_predictor_step.py), so there is no
runnable reference to pin against: this is a restatement of that pseudo-code, vectorised over
water columns, written independently of the CUDA kernel it checks (parity unpinned).

Scope (per water column, rho-interior points i=1..L-1, j=1..M-1):
  * the predictor's initialisation of the new time level, tke(nnew) = Hz_w * tke(nstp)
    (gls_predictor_step.py:153-154), without the advective terms;
  * shear^2 at W points (gls_corrector_step.py:86-96), buoyancy frequency as input (:101);
  * production / dissipation with the buoyancy switch (:397-516);
  * surface and bottom Dirichlet conditions (:526-564) with stresses from the wind and a
    quadratic bottom drag on the bottom-level velocity (nonlinear/set_vbc.py:19-41);
  * the implicit tke and gls solves and the boundary fluxes (:568-656);
  * length-scale limitation, Galperin stability functions, Akv/Akt/Akk/Akp and Lscale
    (:662-825).
The advective terms are restated separately: the predictor's auxiliary half step
(gls_prestep, gls_predictor_step.py:18-216) and the corrector's third-order upstream horizontal
and fourth-order vertical advection of the new level (gls_advect, :172-388); gls_corrector takes
the advected new level as its start (tke_nnew/gls_nnew).

Layout: W-level arrays have N+1 levels (0..N), rho-level arrays N levels; index arrays are
flat (levels, (M+1)*(L+1)) with the reference's flat neighbour offsets (p+1 east, p+I north).
"""
import numpy as np

VONKAR = 0.41               # modules/mod_constants.py:28
EPS = 1.0e-10               # gls_corrector_step.py:673-688 (eps)
# Galperin et al. (1988) quasi-equilibrium stability functions with the Mellor-Yamada
# constants A1, A2, B1, B2, C1 (published values), as the corrector uses them (:740-748).
MY_A1, MY_A2, MY_B1, MY_B2, MY_C1 = 0.92, 0.74, 16.6, 10.1, 0.08
MY_SH1 = MY_A2 * (1.0 - 6.0 * MY_A1 / MY_B1)
MY_SH2 = 3.0 * MY_A2 * (6.0 * MY_A1 + MY_B2)
MY_SM2 = 9.0 * MY_A1 * MY_A2
MY_SM3 = MY_A1 * (1.0 - 3.0 * MY_C1 - 6.0 * MY_A1 / MY_B1)
MY_SM4 = 18.0 * MY_A1 * MY_A1 + 9.0 * MY_A1 * MY_A2
GH0, GHCRI, GHMIN = 0.0233, 0.02, -0.28

# k-epsilon parameters of the reference's input file (utility/test.in:355-367) and its
# background values (test.in:326-349, :380-381).
DEFAULT = dict(p=3.0, m=1.5, n=-1.0, cmu0=0.5477, c1=1.44, c2=1.92, c3m=-0.4, c3p=1.0, sigk=1.0,
               sigp=1.30, Kmin=7.6e-6, Pmin=1.0e-12, Akv_bak=1.0e-5, Akt_bak=1.0e-6,
               Akk_bak=5.0e-6, Akp_bak=5.0e-6, Zos=0.02, Zob=0.02, rdrag2=3.0e-3, E2=1.33)

# Other members of the GLS family with the same backgrounds and floors (Warner et al. 2005,
# Ocean Modelling 8, Table 1): k-omega, and the generic psi = cmu0^p k^m l^n model of Umlauf and
# Burchard (2003), p = 2, m = 1, n = -0.67 ("gen", the k-psi closure).
PRESETS = {
    "k-epsilon": DEFAULT,
    "k-omega": dict(DEFAULT, p=-1.0, m=0.5, n=-1.0, cmu0=0.5477, c1=0.555, c2=0.833, c3m=-0.6,
                    c3p=1.0, sigk=2.0, sigp=2.0),
    "gen": dict(DEFAULT, p=2.0, m=1.0, n=-0.67, cmu0=0.5544, c1=1.0, c2=1.22, c3m=0.05, c3p=1.0,
                sigk=0.8, sigp=1.07),
}
PRESETS["k-psi"] = PRESETS["gen"]


def gls_corrector(P, dt, I, J, N, u, v, z_r, Hz, bvf, sustr, svstr, tke, gls, Akv, Akt, Akk, Akp,
                  Lscale, tke_nnew=None, gls_nnew=None):
    """One corrector step; returns new (tke, gls, Akv, Akt, Akk, Akp, Lscale) copies.
    u, v: (N+1, s2) rho-level velocities (level N unused); z_r, Hz: (N, s2); bvf and the
    turbulence fields: (N+1, s2); sustr, svstr: (s2,) kinematic surface stress at U/V points.
    tke_nnew/gls_nnew (N+1, s2): the new level after advection (gls_advect), to which the
    production terms add (:447-450); by default Hz_w * tke/gls (no advection)."""
    p_, m_, n_ = P["p"], P["m"], P["n"]
    cmu0 = P["cmu0"]
    s2 = I * J
    idx = np.arange(s2)
    ii, jj = idx % I, idx // I
    col = idx[(ii != 0) & (ii != I - 1) & (jj != 0) & (jj != J - 1)]
    out = [a.copy() for a in (tke, gls, Akv, Akt, Akk, Akp, Lscale)]
    tke_o, gls_o = tke[:, col], gls[:, col]
    Akv_o, Akt_o, Akk_o, Akp_o, Ls_o = Akv[:, col], Akt[:, col], Akk[:, col], Akp[:, col], Lscale[:, col]
    nc = col.size

    L_sft = VONKAR
    ogls_sigp = 1.0 / P["sigp"]
    sqrt2 = np.sqrt(2.0)
    cmu_fac1 = cmu0 ** (-p_ / n_)
    cmu_fac2 = cmu0 ** (3.0 + p_ / n_)
    cmu_fac3 = 1.0 / cmu0 ** 2.0
    gls_fac2 = cmu0 ** p_ * n_ * VONKAR ** n_
    gls_fac3 = cmu0 ** p_ * n_
    gls_fac4 = cmu0 ** p_
    gls_fac5 = 0.56 ** (0.5 * n_) * cmu0 ** p_
    gls_exp1 = 1.0 / n_
    tke_exp1 = m_ / n_
    tke_exp2 = 0.5 + m_ / n_
    tke_exp4 = m_ + 0.5 * n_
    Lmy25 = p_ == 0.0 and n_ == 1.0 and m_ == 1.0
    Zos_min = max(P["Zos"], 1.0e-4)
    Zob_min = max(P["Zob"], 1.0e-4)

    # shear^2 at W points 1..N-1 (:86-96)
    sh2 = np.zeros((N + 1, nc))
    for k in range(1, N):
        cff = 0.5 / (z_r[k, col] - z_r[k - 1, col])
        du = (u[k, col] - u[k - 1, col]) + (u[k, col + 1] - u[k - 1, col + 1])
        dv = (v[k, col] - v[k - 1, col]) + (v[k, col + I] - v[k - 1, col + I])
        sh2[k] = (cff * du) ** 2 + (cff * dv) ** 2
    b2 = bvf[:, col]

    # quadratic bottom stress on the bottom-level velocity at the U/V faces of the column
    def bustr(q):
        va = 0.25 * (v[0, q] + v[0, q + I] + v[0, q - 1] + v[0, q - 1 + I])
        return P["rdrag2"] * u[0, q] * np.sqrt(u[0, q] * u[0, q] + va * va)

    def bvstr(q):
        ua = 0.25 * (u[0, q] + u[0, q + 1] + u[0, q - I] + u[0, q + 1 - I])
        return P["rdrag2"] * v[0, q] * np.sqrt(ua * ua + v[0, q] * v[0, q])

    # vertical mixing of the turbulent fields (:401-415)
    FCK = np.zeros((N + 1, nc))
    FCP = np.zeros((N + 1, nc))
    for k in range(2, N):
        FCK[k] = (-0.5 * dt) * (Akk_o[k] + Akk_o[k - 1]) / Hz[k - 1, col]
        FCP[k] = (-0.5 * dt) * (Akp_o[k] + Akp_o[k - 1]) / Hz[k - 1, col]

    tk = np.zeros((N + 1, nc))
    gl = np.zeros((N + 1, nc))
    BCK = np.zeros((N + 1, nc))
    BCP = np.zeros((N + 1, nc))
    zw_bot = None
    for k in range(1, N):
        cffz = 0.5 * (Hz[k - 1, col] + Hz[k, col])
        tk[k] = cffz * tke_o[k] if tke_nnew is None else tke_nnew[k, col]
        gl[k] = cffz * gls_o[k] if gls_nnew is None else gls_nnew[k, col]
        strat2 = b2[k]
        c3 = np.where(strat2 > 0.0, P["c3m"], P["c3p"])
        dAkt = Akt_o[k] - P["Akt_bak"]
        Kprod = sh2[k] * (Akv_o[k] - P["Akv_bak"]) - strat2 * dAkt
        Pprod = P["c1"] * sh2[k] * (Akv_o[k] - P["Akv_bak"]) - c3 * strat2 * dAkt
        cff1 = np.where(Kprod < 0.0, 0.0, 1.0)
        Kprod = np.where(Kprod < 0.0, Kprod + strat2 * dAkt, Kprod)
        cff2 = np.where(Pprod < 0.0, 0.0, 1.0)
        Pprod = np.where(Pprod < 0.0, Pprod + c3 * strat2 * dAkt, Pprod)
        tk[k] = tk[k] + dt * cffz * Kprod
        gl[k] = gl[k] + dt * cffz * Pprod * gls_o[k] / np.maximum(tke_o[k], P["Kmin"])
        wall = 1.0
        if Lmy25:   # parabolic wall function + free-surface correction (:491-497)
            raise NotImplementedError("wall function needs z_w; k-epsilon does not use it")
        diss = gls_o[k] ** (-gls_exp1) * cmu_fac2 * tke_o[k] ** tke_exp2
        BCK[k] = cffz * (1.0 + dt * diss + dt * (1.0 - cff1) * strat2 * dAkt / tke_o[k]) - FCK[k] - FCK[k + 1]
        BCP[k] = (cffz * (1.0 + dt * P["c2"] * wall * diss + dt * (1.0 - cff2) * c3 * strat2 * dAkt / tke_o[k])
                  - FCP[k] - FCP[k + 1])

    # surface / bottom Dirichlet values (:526-564)
    su = sustr[col] + sustr[col + 1]
    sv = svstr[col] + svstr[col + I]
    bu = bustr(col) + bustr(col + 1)
    bv = bvstr(col) + bvstr(col + I)
    tk[N] = np.maximum(cmu_fac3 * 0.5 * np.sqrt(su * su + sv * sv), P["Kmin"])
    tk[0] = np.maximum(cmu_fac3 * 0.5 * np.sqrt(bu * bu + bv * bv), P["Kmin"])
    Zos_eff = Zos_min
    gl[N] = np.maximum(cmu0 ** p_ * tk[N] ** m_ * (L_sft * Zos_eff) ** n_, P["Pmin"])
    gl[0] = np.maximum(gls_fac4 * (VONKAR * Zob_min) ** n_ * tk[0] ** m_, P["Pmin"])

    # tke solve (:571-604)
    CF = np.zeros((N + 1, nc))
    cff = 1.0 / BCK[N - 1]
    CF[N - 1] = cff * FCK[N - 1]
    tk[N - 1] = cff * (tk[N - 1] + 0.0)
    for k in range(N - 2, 0, -1):
        cff = 1.0 / (BCK[k] - CF[k + 1] * FCK[k + 1])
        CF[k] = cff * FCK[k]
        tk[k] = cff * (tk[k] - FCK[k + 1] * tk[k + 1])
    tk[1] = tk[1] - cff * 0.0
    tk[1] = np.maximum(tk[1], P["Kmin"])
    for k in range(2, N):
        tk[k] = tk[k] - CF[k] * tk[k - 1]
        tk[k] = np.maximum(tk[k], P["Kmin"])

    # gls solve (:608-656)
    cffT = 0.5 * (tk[N] + tk[N - 1])
    fluxt = (dt * gls_fac3 * cffT ** m_ * L_sft ** n_ * (Zos_eff + 0.5 * Hz[N - 1, col]) ** (n_ - 1.0)
             * 0.5 * (Akp_o[N] + Akp_o[N - 1]))
    cffB = 0.5 * (tk[0] + tk[1])
    fluxb = (dt * gls_fac2 * cffB ** m_ * (0.5 * Hz[0, col] + Zob_min) ** (n_ - 1.0)
             * 0.5 * (Akp_o[0] + Akp_o[1]))
    cff = 1.0 / BCP[N - 1]
    CF[N - 1] = cff * FCP[N - 1]
    gl[N - 1] = cff * (gl[N - 1] - fluxt)
    for k in range(N - 2, 0, -1):
        cff = 1.0 / (BCP[k] - CF[k + 1] * FCP[k + 1])
        CF[k] = cff * FCP[k]
        gl[k] = cff * (gl[k] - FCP[k + 1] * gl[k + 1])
    gl[1] = gl[1] - cff * fluxb
    for k in range(2, N):
        gl[k] = gl[k] - CF[k] * gl[k - 1]

    # mixing coefficients (:662-825)
    Av, At, Ak, Ap, Ls = (np.array(a) for a in (Akv_o, Akt_o, Akk_o, Akp_o, Ls_o))
    for k in range(1, N):
        tk[k] = np.maximum(tk[k], P["Kmin"])
        gl[k] = np.maximum(gl[k], P["Pmin"])
        lim = gls_fac5 * tk[k] ** tke_exp4 * (np.sqrt(np.maximum(0.0, b2[k])) + EPS) ** (-n_)
        gl[k] = np.minimum(gl[k], lim) if n_ >= 0.0 else np.maximum(gl[k], lim)
        Ls_unlmt = np.maximum(EPS, gl[k] ** gls_exp1 * cmu_fac1 * tk[k] ** (-tke_exp1))
        Ls_lmt = np.where(b2[k] > 0.0,
                          np.minimum(Ls_unlmt, np.sqrt(0.56 * tk[k] / (np.maximum(0.0, b2[k]) + EPS))),
                          Ls_unlmt)
        gl[k] = np.maximum(cmu0 ** p_ * tk[k] ** m_ * Ls_lmt ** n_, P["Pmin"])
        Gh = np.minimum(GH0, -b2[k] * Ls_lmt * Ls_lmt / (2.0 * tk[k]))
        Gh = np.minimum(Gh, Gh - (Gh - GHCRI) ** 2 / (Gh + GH0 - 2.0 * GHCRI))
        Gh = np.maximum(Gh, GHMIN)
        Sh = MY_SH1 / (1.0 - MY_SH2 * Gh)
        Sm = (MY_SM3 + Sh * Gh * MY_SM4) / (1.0 - MY_SM2 * Gh)
        ql = sqrt2 * 0.5 * (Ls_lmt * np.sqrt(tk[k]) + Ls_o[k] * np.sqrt(tke_o[k]))
        Av[k] = P["Akv_bak"] + Sm * ql
        At[k] = P["Akt_bak"] + Sh * ql
        Ak[k] = P["Akk_bak"] + Sm * ql / P["sigk"]
        Ap[k] = P["Akp_bak"] + Sm * ql * ogls_sigp
        Ls[k] = Ls_lmt
    Av[N] = P["Akv_bak"] + L_sft * Zos_eff * cmu0 * np.sqrt(tk[N])
    Av[0] = P["Akv_bak"] + VONKAR * Zob_min * cmu0 * np.sqrt(tk[0])
    Ak[N] = P["Akk_bak"] + Av[N] / P["sigk"]
    Ak[0] = P["Akk_bak"] + Av[0] / P["sigk"]
    Ap[N] = P["Akp_bak"] + Av[N] * ogls_sigp
    Ap[0] = P["Akp_bak"] + Av[0] / P["sigp"]
    At[N] = P["Akt_bak"]
    At[0] = P["Akt_bak"]
    for a, b in zip(out, (tk, gl, Av, At, Ak, Ap, Ls)):
        a[:, col] = b
    return tuple(out)


# ---------------------------------------------------------------------------------------------
# GLS predictor: the auxiliary advective half step of tke and gls
# ---------------------------------------------------------------------------------------------
GAMMA = 1.0 / 6.0   # AM3 weight of the half-step interpolation (ROMS mod_scalars Gamma)


def _edge_grad(q, axis):
    """grad(i) = q(i) - q(i-1) on i = 0..n (n+1 values, with one ghost on either side): the
    first/last differences repeated at the domain edges (gls_predictor_step.py:68-80,97-108)."""
    d = np.diff(q, axis=axis)                        # grad at i = 1..n-1 (in q's index)
    first = np.take(d, [0], axis=axis)
    last = np.take(d, [-1], axis=axis)
    return np.concatenate([first, d, last], axis=axis)   # grad(0) := grad(1), grad(n) := grad(n-1)


def _vflux_ends(q, CF, N):
    """One-sided third-order vertical fluxes at rho levels 1 and N (gls_predictor_step.py:180-189,
    gls_corrector_step.py:349-372): CF * (q0/3 + 5/6 q1 - q2/6) from the boundary inwards."""
    c1, c2, c3 = 1.0 / 3.0, 5.0 / 6.0, 1.0 / 6.0
    return (CF[1] * (c1 * q[0] + c2 * q[1] - c3 * q[2]),
            CF[N] * (c1 * q[N] + c2 * q[N - 1] - c3 * q[N - 2]))


def gls_prestep(dt, first, I, J, N, pm, pn, Huon, Hvom, W, Hz, tke_nstp, tke_indx, gls_nstp,
                gls_indx, gamma=GAMMA):
    """nonlinear/gls_predictor_step.py:18-216 (fourth-order centred horizontal advection,
    AM3-interpolated half step with Hz_half, fourth-order vertical advection) on the
    rho-interior points, W levels 1..N-1, followed by a zero-gradient lateral condition on the
    auxiliary level (edges from the adjacent interior point, corners from the diagonal one).

    Arrays: Huon, Hvom (>= N rho levels, U/V points), W (N+1), Hz (N), tke/gls (N+1), all
    flat (levels, J*I); pm, pn flat (J*I).  Returns (tke_aux, gls_aux, tke_nnew, gls_nnew,
    Hz_half) as (N+1, J*I) arrays (levels 0 and N and the points not written are 0)."""
    sh = (J, I)
    pm2, pn2 = pm.reshape(sh), pn.reshape(sh)
    if first:
        c1, c2, c3 = 1.0, 0.0, 0.5 * dt
        tke_indx, gls_indx = tke_nstp, gls_nstp
    else:
        c1, c2, c3 = 0.5 + gamma, 0.5 - gamma, (1.0 - gamma) * dt
    out_t = np.zeros((N + 1, J * I))
    out_g = np.zeros((N + 1, J * I))
    new_t = np.zeros((N + 1, J * I))
    new_g = np.zeros((N + 1, J * I))
    Hh = np.zeros((N + 1, J * I))
    Wl = W.reshape(N + 1, J, I)
    T, G = tke_nstp.reshape(N + 1, J, I), gls_nstp.reshape(N + 1, J, I)
    Ti, Gi = tke_indx.reshape(N + 1, J, I), gls_indx.reshape(N + 1, J, I)
    # vertical fluxes at rho levels 1..N (Fortran numbering), CF(k) = (W(k) + W(k-1)) / 2
    CF = np.zeros((N + 2, J, I))
    FCt = np.zeros((N + 2, J, I))
    FCg = np.zeros((N + 2, J, I))
    for k in range(1, N + 1):
        CF[k] = 0.5 * (Wl[k] + Wl[k - 1])
    for q, F in ((T, FCt), (G, FCg)):
        for k in range(2, N):
            F[k] = CF[k] * (7.0 / 12.0 * (q[k - 1] + q[k]) - 1.0 / 12.0 * (q[k - 2] + q[k + 1]))
        F[1], F[N] = _vflux_ends(q, CF, N)
    ii = slice(1, I - 1)
    jj = slice(1, J - 1)
    for k in range(1, N):
        HU = Huon.reshape(-1, J, I)[k - 1]
        HU2 = Huon.reshape(-1, J, I)[k]
        HV = Hvom.reshape(-1, J, I)[k - 1]
        HV2 = Hvom.reshape(-1, J, I)[k]
        XF = 0.5 * (HU + HU2)                 # at U points i (between rho i-1 and i)
        EF = 0.5 * (HV + HV2)                 # at V points j
        res = []
        for q, qi, F in ((T[k], Ti[k], FCt), (G[k], Gi[k], FCg)):
            gx = _edge_grad(q, 1)             # (J, I+1): index i -> grad(i), i = 0..I
            gy = _edge_grad(q, 0)             # (J+1, I)
            # FX(i), i = 1..I-1: XF(i) (q(i-1)+q(i) - (grad(i+1)-grad(i-1))/6) / 2
            FX = np.zeros(sh)
            FX[:, 1:] = XF[:, 1:] * 0.5 * (q[:, :-1] + q[:, 1:] - (1.0 / 6.0) * (gx[:, 2:] - gx[:, :-2]))
            FE = np.zeros(sh)
            FE[1:, :] = EF[1:, :] * 0.5 * (q[:-1, :] + q[1:, :] - (1.0 / 6.0) * (gy[2:, :] - gy[:-2, :]))
            res.append((FX, FE, qi))
        cff = 0.5 * (Hz.reshape(N, J, I)[k - 1] + Hz.reshape(N, J, I)[k])
        cff4 = c3 * pm2 * pn2
        divX = np.zeros(sh)
        divE = np.zeros(sh)
        divX[jj, ii] = XF[jj, 2:] - XF[jj, 1:-1]
        divE[jj, ii] = EF[2:, ii] - EF[1:-1, ii]
        hh = cff - cff4 * (divX + divE) - cff4 * (CF[k + 1] - CF[k])
        Hh[k].reshape(sh)[jj, ii] = hh[jj, ii]
        for (FX, FE, qi), q, out, new, F in ((res[0], T[k], out_t, new_t, FCt),
                                              (res[1], G[k], out_g, new_g, FCg)):
            dX = np.zeros(sh)
            dE = np.zeros(sh)
            dX[jj, ii] = FX[jj, 2:] - FX[jj, 1:-1]
            dE[jj, ii] = FE[2:, ii] - FE[1:-1, ii]
            val = cff * (c1 * q + c2 * qi) - cff4 * (dX + dE)
            val = (val - cff4 * (F[k + 1] - F[k])) / hh
            out[k].reshape(sh)[jj, ii] = val[jj, ii]
            new[k].reshape(sh)[jj, ii] = (cff * q)[jj, ii]
    for out, q in ((out_t, T), (out_g, G)):  # bottom/surface of the auxiliary level: nstp values
        for k in (0, N):
            out[k].reshape(sh)[jj, ii] = q[k][jj, ii]
    for out in (out_t, out_g):               # zero-gradient edges of the auxiliary level
        a = out.reshape(N + 1, J, I)
        a[1:N, jj, 0] = a[1:N, jj, 1]
        a[1:N, jj, I - 1] = a[1:N, jj, I - 2]
        a[1:N, 0, ii] = a[1:N, 1, ii]
        a[1:N, J - 1, ii] = a[1:N, J - 2, ii]
        a[1:N, 0, 0] = a[1:N, 1, 1]
        a[1:N, 0, I - 1] = a[1:N, 1, I - 2]
        a[1:N, J - 1, 0] = a[1:N, J - 2, 1]
        a[1:N, J - 1, I - 1] = a[1:N, J - 2, I - 2]
    return out_t, out_g, new_t, new_g, Hh


# ---------------------------------------------------------------------------------------------
# GLS corrector, advective terms
# ---------------------------------------------------------------------------------------------
GADV = 1.0 / 3.0    # third-order upstream-biased weight (gls_corrector_step.py:214-215, :236)


def gls_advect(dt, I, J, N, pm, pn, Huon, Hvom, W, tke_aux, gls_aux, tke_nnew, gls_nnew, Kmin,
               Pmin, gadv=GADV):
    """nonlinear/gls_corrector_step.py:172-388 on the rho-interior points, W levels 1..N-1:
    the new level less dt*pm*pn times the horizontal divergence of the third-order
    upstream-biased fluxes of the auxiliary level (:181-298; the curvature from the upstream
    side of the W-level flux, differences repeated at the domain edges), floored at Kmin/Pmin
    (:300-317), then less the fourth-order vertical flux divergence (:329-377), floored again
    (:378-388).  Arrays flat (levels, J*I) as in gls_prestep; returns new (tke_nnew, gls_nnew)."""
    sh = (J, I)
    cff = (dt * pm.reshape(sh)) * pn.reshape(sh)
    ii = slice(1, I - 1)
    jj = slice(1, J - 1)
    Wl = W.reshape(N + 1, J, I)
    CF = np.zeros((N + 2, J, I))
    for k in range(1, N + 1):
        CF[k] = 0.5 * (Wl[k] + Wl[k - 1])
    outs = []
    for aux, new, floor in ((tke_aux, tke_nnew, Kmin), (gls_aux, gls_nnew, Pmin)):
        q3 = aux.reshape(N + 1, J, I)
        out = new.copy().reshape(N + 1, J, I)
        FC = np.zeros((N + 2, J, I))
        for k in range(2, N):
            FC[k] = CF[k] * (7.0 / 12.0 * (q3[k - 1] + q3[k]) - 1.0 / 12.0 * (q3[k - 2] + q3[k + 1]))
        FC[1], FC[N] = _vflux_ends(q3, CF, N)
        for k in range(1, N):
            q = q3[k]
            XF = 0.5 * (Huon.reshape(-1, J, I)[k - 1] + Huon.reshape(-1, J, I)[k])
            EF = 0.5 * (Hvom.reshape(-1, J, I)[k - 1] + Hvom.reshape(-1, J, I)[k])
            gx = _edge_grad(q, 1)             # (J, I+1): grad(i), i = 0..I
            gy = _edge_grad(q, 0)             # (J+1, I)
            cx = gx[:, 1:] - gx[:, :-1]       # curv(i) = grad(i+1) - grad(i), i = 0..I-1
            cy = gy[1:, :] - gy[:-1, :]
            FX = np.zeros(sh)                 # FX(i) at U point i = 1..I-1
            up = np.where(XF[:, 1:] > 0.0, cx[:, :-1], cx[:, 1:])
            FX[:, 1:] = XF[:, 1:] * 0.5 * (q[:, :-1] + q[:, 1:] - gadv * up)
            FE = np.zeros(sh)
            up = np.where(EF[1:, :] > 0.0, cy[:-1, :], cy[1:, :])
            FE[1:, :] = EF[1:, :] * 0.5 * (q[:-1, :] + q[1:, :] - gadv * up)
            div = np.zeros(sh)
            div[jj, ii] = FX[jj, 2:] - FX[jj, 1:-1] + FE[2:, ii] - FE[1:-1, ii]
            t = np.maximum(out[k] - cff * div, floor)
            t = np.maximum(t - cff * (FC[k + 1] - FC[k]), floor)
            out[k][jj, ii] = t[jj, ii]
        outs.append(out.reshape(N + 1, J * I))
    return outs[0], outs[1]
