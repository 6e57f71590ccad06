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
    R *Akk, R *Akp, R *Lscale, const R *__restrict__ tkn0, const R *__restrict__ gln0,
    const uint8_t *__restrict__ sel, const int *__restrict__ list, const int *__restrict__ count) {
    int pi = (int)tid_flat();
    if (list) {                    // a compacted list of columns: thread t takes list[t]
        if (pi >= *count) return;
        pi = list[pi];
    }
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
        // the new level starts from tke/gls(nnew) after advection when given, else from
        // Hz_w * tke/gls(nstp) (the predictor's start without the advective terms)
        const R tst = tkn0 ? AT(tkn0, k, p) : cffz * tko;
        const R gst = gln0 ? AT(gln0, k, p) : cffz * glo;
        tk[k] = tst + dt * cffz * Kprod;
        gl[k] = gst + dt * cffz * Pprod * glo / fmax(tko, Kmin);
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


// ---------------------------------------------------------------------------------------------
// GLS predictor (nonlinear/gls_predictor_step.py:18-216, ROMS pseudo-code in the reference): the
// auxiliary advective half step of tke and gls at W levels 1..N-1 on the rho-interior points.
// Fourth-order centred horizontal fluxes FX/FE with the edge differences repeated at the domain
// edges (:62-127); the LF step interpolated back half a step with the AM3 weights cff1..cff3
// and the half-step box height Hz_half (:133-157); fourth-order vertical fluxes with the
// one-sided third-order forms at the bottom and surface (:162-208).  Also tke/gls(nnew) =
// Hz_w * tke/gls(nstp), the start of the corrector's update (:153-154).
// ---------------------------------------------------------------------------------------------
template <typename R>
__device__ __forceinline__ R vflux_(const R *q, const R *W, long p, long s2, int m, int N) {
    // FC at rho level m (1..N, Fortran numbering) of the W-level field q
#define Q(k) (q[(long)(k) * s2 + p])
    const R cf = R(0.5) * (W[(long)m * s2 + p] + W[(long)(m - 1) * s2 + p]);
    if (m == 1) return cf * (R(1.0 / 3.0) * Q(0) + R(5.0 / 6.0) * Q(1) - R(1.0 / 6.0) * Q(2));
    if (m == N)
        return cf * (R(1.0 / 3.0) * Q(N) + R(5.0 / 6.0) * Q(N - 1) - R(1.0 / 6.0) * Q(N - 2));
    return cf * (R(7.0 / 12.0) * (Q(m - 1) + Q(m)) - R(1.0 / 12.0) * (Q(m - 2) + Q(m + 1)));
#undef Q
}

// One tracer's horizontal flux divergence FX(i+1)-FX(i) + FE(j+1)-FE(j) at (i, j), level k.
template <typename R>
__device__ __forceinline__ R hdiv_(const R *q, const R *XF0, const R *XF1, const R *EF0,
                                   const R *EF1, long p, int i, int j, int I, int J, long s2,
                                   int k) {
    const R *qk = q + (long)k * s2;
    auto gx = [&](int m) -> R {   // grad(m) = q(m) - q(m-1), edges repeated
        m = m < 1 ? 1 : (m > I - 1 ? I - 1 : m);
        return qk[(long)j * I + m] - qk[(long)j * I + m - 1];
    };
    auto gy = [&](int m) -> R {
        m = m < 1 ? 1 : (m > J - 1 ? J - 1 : m);
        return qk[(long)m * I + i] - qk[(long)(m - 1) * I + i];
    };
    auto FX = [&](int a) -> R {   // at U point a of row j
        const long u = (long)j * I + a;
        const R xf = R(0.5) * (XF0[u] + XF1[u]);
        return xf * R(0.5) * (qk[u - 1] + qk[u] - R(1.0 / 6.0) * (gx(a + 1) - gx(a - 1)));
    };
    auto FE = [&](int b) -> R {   // at V point b of column i
        const long v = (long)b * I + i;
        const R ef = R(0.5) * (EF0[v] + EF1[v]);
        return ef * R(0.5) * (qk[v - I] + qk[v] - R(1.0 / 6.0) * (gy(b + 1) - gy(b - 1)));
    };
    (void)p;
    return (FX(i + 1) - FX(i)) + (FE(j + 1) - FE(j));
}

template <typename R>
__global__ void __launch_bounds__(128) k_gls_prestep(Geo<R> g, GlsPre c, const R *__restrict__ Huon,
        const R *__restrict__ Hvom, const R *__restrict__ W, const R *__restrict__ Hz,
        const R *__restrict__ tke0, const R *__restrict__ tkei, R *__restrict__ tke3,
        R *__restrict__ tken, const R *__restrict__ gls0, const R *__restrict__ glsi,
        R *__restrict__ gls3, R *__restrict__ glsn, R *__restrict__ Hz_half) {
    const int pi = (int)tid_flat();
    if (pi >= g.s2) return;
    const int I = g.I, J = g.J, N = g.N;
    const int i = pi % I, j = pi / I;
    if (i < 1 || i > I - 2 || j < 1 || j > J - 2) return;
    const long p = pi, s2 = g.s2;
    const R cff4 = (R)c.c3 * (g.pm[p] * g.pn[p]);
    R FCt = vflux_(tke0, W, p, s2, 1, N), FCg = vflux_(gls0, W, p, s2, 1, N);
    R CFk = R(0.5) * (W[s2 + p] + W[p]);
    for (int k = 1; k < N; ++k) {
        const R *XF0 = Huon + (long)(k - 1) * s2, *XF1 = Huon + (long)k * s2;
        const R *EF0 = Hvom + (long)(k - 1) * s2, *EF1 = Hvom + (long)k * s2;
        const long o = (long)k * s2 + p;
        const R cff = R(0.5) * (Hz[o - s2] + Hz[o]);
        const long u = (long)j * I + i, v = u;
        const R divUV = (R(0.5) * (XF0[u + 1] + XF1[u + 1]) - R(0.5) * (XF0[u] + XF1[u])) +
                        (R(0.5) * (EF0[v + I] + EF1[v + I]) - R(0.5) * (EF0[v] + EF1[v]));
        const R CFk1 = R(0.5) * (W[o + s2] + W[o]);
        R hh = cff - cff4 * divUV;
        hh = hh - cff4 * (CFk1 - CFk);
        const R FCt1 = vflux_(tke0, W, p, s2, k + 1, N), FCg1 = vflux_(gls0, W, p, s2, k + 1, N);
        const R ht = hdiv_(tke0, XF0, XF1, EF0, EF1, p, i, j, I, J, s2, k);
        const R hg = hdiv_(gls0, XF0, XF1, EF0, EF1, p, i, j, I, J, s2, k);
        const R t = (cff * ((R)c.c1 * tke0[o] + (R)c.c2 * tkei[o]) - cff4 * ht) - cff4 * (FCt1 - FCt);
        const R q = (cff * ((R)c.c1 * gls0[o] + (R)c.c2 * glsi[o]) - cff4 * hg) - cff4 * (FCg1 - FCg);
        tke3[o] = t / hh;
        gls3[o] = q / hh;
        tken[o] = cff * tke0[o];
        glsn[o] = cff * gls0[o];
        Hz_half[o] = hh;
        FCt = FCt1;
        FCg = FCg1;
        CFk = CFk1;
    }
    // the auxiliary level's bottom and surface values are the nstp ones (no advective update
    // there); the corrector's vertical fluxes at rho levels 1 and N read them
    tke3[p] = tke0[p];
    gls3[p] = gls0[p];
    tke3[(long)N * s2 + p] = tke0[(long)N * s2 + p];
    gls3[(long)N * s2 + p] = gls0[(long)N * s2 + p];
}

// Zero-gradient lateral condition on the auxiliary level (edges from the adjacent interior
// point, corners from the diagonal one), W levels 1..N-1.
template <typename R>
__global__ void k_gls_aux_bc(Geo<R> g, R *__restrict__ tke3, R *__restrict__ gls3) {
    const int I = g.I, J = g.J;
    const int nb = 2 * I + 2 * (J - 2);
    const long e = tid_flat();
    if (e >= (long)nb * (g.N - 1)) return;
    const int k = 1 + (int)(e / nb), b = (int)(e % nb);
    int i, j;
    if (b < I) { i = b; j = 0; }
    else if (b < 2 * I) { i = b - I; j = J - 1; }
    else if (b < 2 * I + J - 2) { i = 0; j = 1 + (b - 2 * I); }
    else { i = I - 1; j = 1 + (b - 2 * I - (J - 2)); }
    const int si = i == 0 ? 1 : (i == I - 1 ? I - 2 : i);
    const int sj = j == 0 ? 1 : (j == J - 1 ? J - 2 : j);
    const long o = (long)k * g.s2;
    tke3[o + (long)j * I + i] = tke3[o + (long)sj * I + si];
    gls3[o + (long)j * I + i] = gls3[o + (long)sj * I + si];
}

// ---------------------------------------------------------------------------------------------
// GLS corrector, advective terms (nonlinear/gls_corrector_step.py:172-388): tke/gls(nnew), the
// Hz_w-weighted new level the predictor starts, less the horizontal flux divergence of the
// auxiliary level (time level 3) — third-order upstream-biased fluxes whose curvature term
// comes from the upstream side of the W-level U/V flux, weighted by Gadv (:181-298; the
// one-sided differences repeated at the domain edges, :196-212, :253-268) — then floored at
// Kmin/Pmin (:300-317); then less the vertical flux divergence of the auxiliary level
// (fourth-order, with the one-sided third-order forms at the bottom and surface, :329-377) and
// floored again (:378-388).  W levels 1..N-1 on the rho-interior points.
// ---------------------------------------------------------------------------------------------
template <typename R>
__device__ __forceinline__ R hdiv_up3_(const R *qk, const R *XF0, const R *XF1, const R *EF0,
                                       const R *EF1, int i, int j, int I, int J, R gadv) {
    auto gx = [&](int m) -> R {   // grad(m) = q(m) - q(m-1), edges repeated
        m = m < 1 ? 1 : (m > I - 1 ? I - 1 : m);
        return qk[(long)j * I + m] - qk[(long)j * I + m - 1];
    };
    auto gy = [&](int m) -> R {
        m = m < 1 ? 1 : (m > J - 1 ? J - 1 : m);
        return qk[(long)m * I + i] - qk[(long)(m - 1) * I + i];
    };
    auto FX = [&](int a) -> R {   // at U point a of row j: curv(a-1) if the flux is eastward
        const long u = (long)j * I + a;
        const R xf = R(0.5) * (XF0[u] + XF1[u]);
        const R curv = xf > R(0) ? gx(a) - gx(a - 1) : gx(a + 1) - gx(a);
        return xf * R(0.5) * (qk[u - 1] + qk[u] - gadv * curv);
    };
    auto FE = [&](int b) -> R {   // at V point b of column i
        const long v = (long)b * I + i;
        const R ef = R(0.5) * (EF0[v] + EF1[v]);
        const R curv = ef > R(0) ? gy(b) - gy(b - 1) : gy(b + 1) - gy(b);
        return ef * R(0.5) * (qk[v - I] + qk[v] - gadv * curv);
    };
    return FX(i + 1) - FX(i) + FE(j + 1) - FE(j);
}

template <typename R>
__global__ void __launch_bounds__(128) k_gls_advect(Geo<R> g, R dt, R gadv, R Kmin, R Pmin,
        const R *__restrict__ Huon, const R *__restrict__ Hvom, const R *__restrict__ W,
        const R *__restrict__ tke3, const R *__restrict__ gls3, R *__restrict__ tken,
        R *__restrict__ glsn) {
    const int pi = (int)tid_flat();
    if (pi >= g.s2) return;
    const int I = g.I, J = g.J, N = g.N;
    const int i = pi % I, j = pi / I;
    if (i < 1 || i > I - 2 || j < 1 || j > J - 2) return;
    const long p = pi, s2 = g.s2;
    const R cff = dt * g.pm[p] * g.pn[p];
    R FCt = vflux_(tke3, W, p, s2, 1, N), FCg = vflux_(gls3, W, p, s2, 1, N);
    for (int k = 1; k < N; ++k) {
        const R *XF0 = Huon + (long)(k - 1) * s2, *XF1 = Huon + (long)k * s2;
        const R *EF0 = Hvom + (long)(k - 1) * s2, *EF1 = Hvom + (long)k * s2;
        const long o = (long)k * s2 + p;
        const R ht = hdiv_up3_(tke3 + (long)k * s2, XF0, XF1, EF0, EF1, i, j, I, J, gadv);
        const R hg = hdiv_up3_(gls3 + (long)k * s2, XF0, XF1, EF0, EF1, i, j, I, J, gadv);
        const R FCt1 = vflux_(tke3, W, p, s2, k + 1, N), FCg1 = vflux_(gls3, W, p, s2, k + 1, N);
        R t = fmax(tken[o] - cff * ht, Kmin);
        R q = fmax(glsn[o] - cff * hg, Pmin);
        t = fmax(t - cff * (FCt1 - FCt), Kmin);
        q = fmax(q - cff * (FCg1 - FCg), Pmin);
        tken[o] = t;
        glsn[o] = q;
        FCt = FCt1;
        FCg = FCg1;
    }
}

template <typename R>
cudaError_t Ops<R>::gls_advect(const sf_ctx *ctx, double dt, double gadv, double Kmin,
                               double Pmin, const R *Huon, const R *Hvom, const R *W,
                               const R *tke3, const R *gls3, R *tken, R *glsn, cudaStream_t s) {
    const Geo<R> g = geo(ctx);
    k_gls_advect<R><<<(unsigned)((g.s2 + 127) / 128), 128, 0, s>>>(
        g, (R)dt, (R)gadv, (R)Kmin, (R)Pmin, Huon, Hvom, W, tke3, gls3, tken, glsn);
    return cudaGetLastError();
}

template <typename R>
cudaError_t Ops<R>::gls_prestep(const sf_ctx *ctx, GlsPre c, const R *Huon, const R *Hvom,
                                const R *W, const R *Hz, const R *tke0, const R *tkei, R *tke3,
                                R *tken, const R *gls0, const R *glsi, R *gls3, R *glsn,
                                R *Hz_half, cudaStream_t s) {
    const Geo<R> g = geo(ctx);
    k_gls_prestep<R><<<(unsigned)((g.s2 + 127) / 128), 128, 0, s>>>(
        g, c, Huon, Hvom, W, Hz, tke0, tkei, tke3, tken, gls0, glsi, gls3, glsn, Hz_half);
    const long nb = (long)(2 * g.I + 2 * (g.J - 2)) * (g.N - 1);
    k_gls_aux_bc<R><<<(unsigned)((nb + 255) / 256), 256, 0, s>>>(g, tke3, gls3);
    return cudaGetLastError();
}

}  // namespace sf
