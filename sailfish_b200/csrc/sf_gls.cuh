// GLS vertical-mixing corrector: one thread per rho-interior water column.
//
// Restates the column physics of the reference's GLS pseudo-code (ROMS Fortran kept inside
// nonlinear/gls_corrector_step.py, which does not parse): production and dissipation with the
// buoyancy switch (:397-516), surface and bottom Dirichlet conditions (:526-564) from the wind
// stress and a quadratic bottom drag on the bottom-level velocity (nonlinear/set_vbc.py:19-41),
// the implicit tke and gls solves with their boundary fluxes (:568-656), the length-scale
// limitation, Galperin stability functions and the mixing coefficients (:662-825).  The new
// time level starts from Hz_w*tke(nstp) as the predictor leaves it without advection
// (nonlinear/gls_predictor_step.py:153-154).
#pragma once
#include "sf_internal.h"

namespace sf {

// Galperin et al. (1988) stability-function constants from the Mellor-Yamada A1, A2, B1,
// B2, C1 (published values), in the form the corrector evaluates (:740-748).
constexpr double kMyA1 = 0.92, kMyA2 = 0.74, kMyB1 = 16.6, kMyB2 = 10.1, kMyC1 = 0.08;
constexpr double kSh1 = kMyA2 * (1.0 - 6.0 * kMyA1 / kMyB1);
constexpr double kSh2 = 3.0 * kMyA2 * (6.0 * kMyA1 + kMyB2);
constexpr double kSm2 = 9.0 * kMyA1 * kMyA2;
constexpr double kSm3 = kMyA1 * (1.0 - 3.0 * kMyC1 - 6.0 * kMyA1 / kMyB1);
constexpr double kSm4 = 18.0 * kMyA1 * kMyA1 + 9.0 * kMyA1 * kMyA2;
constexpr double kGh0 = 0.0233, kGhcri = 0.02, kGhmin = -0.28;
constexpr double kVonKar = 0.41, kGlsEps = 1.0e-10;

template <typename R>
__device__ __forceinline__ R qpow(R a, R b) { return pow(a, b); }
template <>
__device__ __forceinline__ float qpow<float>(float a, float b) { return powf(a, b); }

template <typename R>
__global__ void __launch_bounds__(128) k_gls_corrector(
    Geo<R> g, sf_gls_params P, R dt, const R *__restrict__ u, const R *__restrict__ v,
    const R *__restrict__ z_r, const R *__restrict__ Hz, const R *__restrict__ bvf,
    const R *__restrict__ sustr, const R *__restrict__ svstr, R *tke, R *gls, R *Akv, R *Akt,
    R *Akk, R *Akp, R *Lscale, const uint8_t *__restrict__ sel) {
    const int pi = (int)tid_flat();
    if (pi >= g.s2) return;
    const int i = pi % g.I, j = pi / g.I;
    if (!rint_(i, j, g.I, g.J)) return;
    if (sel && !sel[pi]) return;   // column not selected: left as it is
    const long p = pi, I = g.I, s2 = g.s2;
    const int N = g.N;
    R FCK[kNMax + 1], FCP[kNMax + 1], BCK[kNMax + 1], BCP[kNMax + 1], tk[kNMax + 1], gl[kNMax + 1],
        CF[kNMax + 1];
#define AT(X, k, q) ((X)[(long)(k) * s2 + (q)])
    const R pp = (R)P.p, mm = (R)P.m, nn = (R)P.n, cmu0 = (R)P.cmu0;
    const R L_sft = (R)kVonKar, ogls_sigp = R(1) / (R)P.sigp;
    const R cmu_fac1 = qpow(cmu0, -pp / nn), cmu_fac2 = qpow(cmu0, R(3) + pp / nn);
    const R cmu_fac3 = R(1) / qpow(cmu0, R(2));
    const R gls_fac2 = qpow(cmu0, pp) * nn * qpow((R)kVonKar, nn), gls_fac3 = qpow(cmu0, pp) * nn;
    const R gls_fac4 = qpow(cmu0, pp), gls_fac5 = qpow(R(0.56), R(0.5) * nn) * qpow(cmu0, pp);
    const R gls_exp1 = R(1) / nn, tke_exp1 = mm / nn, tke_exp2 = R(0.5) + mm / nn;
    const R tke_exp4 = mm + R(0.5) * nn;
    const R Kmin = (R)P.Kmin, Pmin = (R)P.Pmin, eps = (R)kGlsEps;
    const R Zos_eff = (R)fmax(P.Zos, 1.0e-4), Zob_min = (R)fmax(P.Zob, 1.0e-4);
    const R Akv_bak = (R)P.Akv_bak, Akt_bak = (R)P.Akt_bak, Akk_bak = (R)P.Akk_bak,
            Akp_bak = (R)P.Akp_bak;

    // vertical mixing of the turbulent fields (:401-415)
    FCK[1] = FCK[N] = FCP[1] = FCP[N] = R(0);
    for (int k = 2; k < N; ++k) {
        const R hz = AT(Hz, k - 1, p);
        FCK[k] = (R(-0.5) * dt) * (AT(Akk, k, p) + AT(Akk, k - 1, p)) / hz;
        FCP[k] = (R(-0.5) * dt) * (AT(Akp, k, p) + AT(Akp, k - 1, p)) / hz;
    }
    // production and dissipation (:397-516)
    for (int k = 1; k < N; ++k) {
        const R cff = R(0.5) / (AT(z_r, k, p) - AT(z_r, k - 1, p));
        const R du = (AT(u, k, p) - AT(u, k - 1, p)) + (AT(u, k, p + 1) - AT(u, k - 1, p + 1));
        const R dv = (AT(v, k, p) - AT(v, k - 1, p)) + (AT(v, k, p + I) - AT(v, k - 1, p + I));
        const R sh2 = (cff * du) * (cff * du) + (cff * dv) * (cff * dv);
        const R cffz = R(0.5) * (AT(Hz, k - 1, p) + AT(Hz, k, p));
        const R tko = AT(tke, k, p), glo = AT(gls, k, p);
        const R strat2 = AT(bvf, k, p);
        const R c3 = strat2 > R(0) ? (R)P.c3m : (R)P.c3p;
        const R dAkt = AT(Akt, k, p) - Akt_bak, dAkv = AT(Akv, k, p) - Akv_bak;
        R Kprod = sh2 * dAkv - strat2 * dAkt;
        R Pprod = (R)P.c1 * sh2 * dAkv - c3 * strat2 * dAkt;
        R cff1 = R(1), cff2 = R(1);
        if (Kprod < R(0)) {
            Kprod = Kprod + strat2 * dAkt;
            cff1 = R(0);
        }
        if (Pprod < R(0)) {
            Pprod = Pprod + c3 * strat2 * dAkt;
            cff2 = R(0);
        }
        tk[k] = cffz * tko + dt * cffz * Kprod;
        gl[k] = cffz * glo + dt * cffz * Pprod * glo / fmax(tko, Kmin);
        const R diss = qpow(glo, -gls_exp1) * cmu_fac2 * qpow(tko, tke_exp2);
        BCK[k] = cffz * (R(1) + dt * diss + dt * (R(1) - cff1) * strat2 * dAkt / tko) - FCK[k] -
                 (k + 1 <= N ? FCK[k + 1] : R(0));
        BCP[k] = cffz * (R(1) + dt * (R)P.c2 * diss + dt * (R(1) - cff2) * c3 * strat2 * dAkt / tko) -
                 FCP[k] - (k + 1 <= N ? FCP[k + 1] : R(0));
    }
    // surface and bottom conditions (:526-564); bottom stress on the bottom-level velocity
    auto bustr = [&](long q) {
        const R va = R(0.25) * (AT(v, 0, q) + AT(v, 0, q + I) + AT(v, 0, q - 1) + AT(v, 0, q - 1 + I));
        return (R)P.rdrag2 * AT(u, 0, q) * sqrt(AT(u, 0, q) * AT(u, 0, q) + va * va);
    };
    auto bvstr = [&](long q) {
        const R ua = R(0.25) * (AT(u, 0, q) + AT(u, 0, q + 1) + AT(u, 0, q - I) + AT(u, 0, q + 1 - I));
        return (R)P.rdrag2 * AT(v, 0, q) * sqrt(ua * ua + AT(v, 0, q) * AT(v, 0, q));
    };
    const R su = sustr[p] + sustr[p + 1], sv = svstr[p] + svstr[p + I];
    const R bu = bustr(p) + bustr(p + 1), bv = bvstr(p) + bvstr(p + I);
    tk[N] = fmax(cmu_fac3 * R(0.5) * sqrt(su * su + sv * sv), Kmin);
    tk[0] = fmax(cmu_fac3 * R(0.5) * sqrt(bu * bu + bv * bv), Kmin);
    gl[N] = fmax(qpow(cmu0, pp) * qpow(tk[N], mm) * qpow(L_sft * Zos_eff, nn), Pmin);
    gl[0] = fmax(gls_fac4 * qpow((R)kVonKar * Zob_min, nn) * qpow(tk[0], mm), Pmin);
    // tke (:571-604)
    R cff = R(1) / BCK[N - 1];
    CF[N - 1] = cff * FCK[N - 1];
    tk[N - 1] = cff * tk[N - 1];
    for (int k = N - 2; k >= 1; --k) {
        cff = R(1) / (BCK[k] - CF[k + 1] * FCK[k + 1]);
        CF[k] = cff * FCK[k];
        tk[k] = cff * (tk[k] - FCK[k + 1] * tk[k + 1]);
    }
    tk[1] = fmax(tk[1], Kmin);
    for (int k = 2; k < N; ++k) tk[k] = fmax(tk[k] - CF[k] * tk[k - 1], Kmin);
    // gls (:608-656)
    const R cffT = R(0.5) * (tk[N] + tk[N - 1]);
    const R fluxt = dt * gls_fac3 * qpow(cffT, mm) * qpow(L_sft, nn) *
                    qpow(Zos_eff + R(0.5) * AT(Hz, N - 1, p), nn - R(1)) * R(0.5) *
                    (AT(Akp, N, p) + AT(Akp, N - 1, p));
    const R cffB = R(0.5) * (tk[0] + tk[1]);
    const R fluxb = dt * gls_fac2 * qpow(cffB, mm) * qpow(R(0.5) * AT(Hz, 0, p) + Zob_min, nn - R(1)) *
                    R(0.5) * (AT(Akp, 0, p) + AT(Akp, 1, p));
    cff = R(1) / BCP[N - 1];
    CF[N - 1] = cff * FCP[N - 1];
    gl[N - 1] = cff * (gl[N - 1] - fluxt);
    for (int k = N - 2; k >= 1; --k) {
        cff = R(1) / (BCP[k] - CF[k + 1] * FCP[k + 1]);
        CF[k] = cff * FCP[k];
        gl[k] = cff * (gl[k] - FCP[k + 1] * gl[k + 1]);
    }
    gl[1] = gl[1] - cff * fluxb;
    for (int k = 2; k < N; ++k) gl[k] = gl[k] - CF[k] * gl[k - 1];
    // mixing coefficients (:662-825); the old values of level k are read before it is written
    const R sqrt2 = sqrt(R(2));
    for (int k = 1; k < N; ++k) {
        const R b2 = AT(bvf, k, p);
        const R tkn = fmax(tk[k], Kmin);
        R gln = fmax(gl[k], Pmin);
        const R lim = gls_fac5 * qpow(tkn, tke_exp4) * qpow(sqrt(fmax(R(0), b2)) + eps, -nn);
        gln = nn >= R(0) ? fmin(gln, lim) : fmax(gln, lim);
        const R Ls_unlmt = fmax(eps, qpow(gln, gls_exp1) * cmu_fac1 * qpow(tkn, -tke_exp1));
        const R Ls_lmt = b2 > R(0) ? fmin(Ls_unlmt, sqrt(R(0.56) * tkn / (fmax(R(0), b2) + eps)))
                                   : Ls_unlmt;
        gln = fmax(qpow(cmu0, pp) * qpow(tkn, mm) * qpow(Ls_lmt, nn), Pmin);
        R Gh = fmin((R)kGh0, -b2 * Ls_lmt * Ls_lmt / (R(2) * tkn));
        Gh = fmin(Gh, Gh - (Gh - (R)kGhcri) * (Gh - (R)kGhcri) / (Gh + (R)kGh0 - R(2) * (R)kGhcri));
        Gh = fmax(Gh, (R)kGhmin);
        const R Sh = (R)kSh1 / (R(1) - (R)kSh2 * Gh);
        const R Sm = ((R)kSm3 + Sh * Gh * (R)kSm4) / (R(1) - (R)kSm2 * Gh);
        const R ql = sqrt2 * R(0.5) * (Ls_lmt * sqrt(tkn) + AT(Lscale, k, p) * sqrt(AT(tke, k, p)));
        AT(Akv, k, p) = Akv_bak + Sm * ql;
        AT(Akt, k, p) = Akt_bak + Sh * ql;
        AT(Akk, k, p) = Akk_bak + Sm * ql / (R)P.sigk;
        AT(Akp, k, p) = Akp_bak + Sm * ql * ogls_sigp;
        AT(Lscale, k, p) = Ls_lmt;
        AT(tke, k, p) = tkn;
        AT(gls, k, p) = gln;
    }
    const R AvN = Akv_bak + L_sft * Zos_eff * cmu0 * sqrt(tk[N]);
    const R Av0 = Akv_bak + (R)kVonKar * Zob_min * cmu0 * sqrt(tk[0]);
    AT(Akv, N, p) = AvN;
    AT(Akv, 0, p) = Av0;
    AT(Akk, N, p) = Akk_bak + AvN / (R)P.sigk;
    AT(Akk, 0, p) = Akk_bak + Av0 / (R)P.sigk;
    AT(Akp, N, p) = Akp_bak + AvN * ogls_sigp;
    AT(Akp, 0, p) = Akp_bak + Av0 / (R)P.sigp;
    AT(Akt, N, p) = Akt_bak;
    AT(Akt, 0, p) = Akt_bak;
    AT(tke, N, p) = tk[N];
    AT(tke, 0, p) = tk[0];
    AT(gls, N, p) = gl[N];
    AT(gls, 0, p) = gl[0];
#undef AT
}

}  // namespace sf
