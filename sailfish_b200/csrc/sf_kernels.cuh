// Device kernels of the time step, templated on the stencil precision R (double or float).
//
// Layout: the reference's flat C-order fields.  Thread p of a column kernel owns the flat 2D
// index p (i = p % I along xi, j = p / I along eta) and marches over the levels, so that
// at every level consecutive threads touch consecutive addresses (coalesced), and stencil
// neighbours (p +- 1, p +- I, p +- 2I) are re-read from L1/L2 by the threads next to them.
//
// Semantics: each kernel computes what the reference kernel(s) it replaces compute, node for
// node, including the reference's flat-index neighbour arithmetic (at i = 0 the "west"
// neighbour is the last point of the previous row) and its boundary quirks, which are
// cited where they occur.  Reads that the reference makes before the start of an array
// (only at level 0 of the boundary rows; they hit whatever precedes the allocation) read 0
// here; the oracle harness zero-guards its arrays, so the two agree.
//
// With R = double and FMA contraction disabled (-fmad=false, sf_kernels_f64.cu) every value
// is bit-identical to the oracle's.  With R = float the stencils run in FP32 and the
// fast-time accumulators (Zt_avg1, DU_avg1, DV_avg1), the column sums of the 3D/2D
// coupling and the depth recomputation (set_depth) stay in FP64.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include "sf_internal.h"

namespace sf {

constexpr int kBlock = 256;
constexpr int kNMax = 64;    // largest N of the column kernels' register/local arrays

__device__ __forceinline__ long tid_flat() { return (long)blockIdx.x * blockDim.x + threadIdx.x; }

// Node predicates, modules/mod_cppkernels.h:101-152 (p < s2 already checked).
__device__ __forceinline__ bool rint_(int i, int j, int I, int J) {
    return !(i == 0 || i == I - 1 || j == 0 || j == J - 1);   // mod_cppkernels.cpp:20
}
__device__ __forceinline__ bool rnode_(int i, int j) { return i > 0 && j > 0; }
__device__ __forceinline__ bool unode_(int i, int j) { return i > 1 && j > 0; }
__device__ __forceinline__ bool vnode_(int i, int j, int J) { return i > 0 && j > 1 && j < J - 1; }
__device__ __forceinline__ bool inner_(int i, int j, int I, int J) {
    return i > 1 && i < I - 2 && j > 1 && j < J - 2;
}

template <typename R>
__device__ __forceinline__ R ldz(const R *a, long idx) {   // read, 0 before the array start
    return idx >= 0 ? a[idx] : R(0);
}

// ------------------------------------------------------------------------------------------
// 2D barotropic kernels
// ------------------------------------------------------------------------------------------

// computeZetaRHS (mod_cppkernels.cpp:81-128), optionally fused with the leapfrog of
// computeZetaPred (:134-150, mode 2) or with the corrector's fast-time averages (mode 1).
template <typename R>
__global__ void __launch_bounds__(kBlock) k_zeta_rhs(
    Geo<R> g, const R *__restrict__ zeta, const R *__restrict__ ubar, const R *__restrict__ vbar,
    R *__restrict__ rzeta, int mode, double cff1, double *__restrict__ Zt,
    double *__restrict__ DU, double *__restrict__ DV, const R *__restrict__ zeta_t0,
    R *__restrict__ zeta_t2, R Dt) {
    const long p = tid_flat();
    if (p >= g.s2) return;
    const long I = g.I;
    const int i = (int)(p % I), j = (int)(p / I);
    const bool in = rint_(i, j, g.I, g.J);
    R rz = R(0);
    if (in) {
        const R *h = g.h;
        const R Dp = zeta[p] + h[p], Dw = zeta[p - 1] + h[p - 1], De = zeta[p + 1] + h[p + 1];
        const R Ds = zeta[p - I] + h[p - I], Dn = zeta[p + I] + h[p + I];
        const R DUp = ubar[p] * ((Dp + Dw) * R(0.5));
        const R DUe = ubar[p + 1] * ((De + Dp) * R(0.5));
        const R DVp = vbar[p] * ((Dp + Ds) * R(0.5));
        const R DVn = vbar[p + I] * ((Dn + Dp) * R(0.5));
        rz = (((DUe * g.on_u[p + 1] - DUp * g.on_u[p]) + (DVn * g.om_v[p + I] - DVp * g.om_v[p])) *
              g.pm[p]) * g.pn[p];
        rzeta[p] = rz;
        if (mode == 1) {
            Zt[p] = Zt[p] + cff1 * (double)zeta[p];
            DU[p] = DU[p] + (cff1 * (double)DUp) * (double)g.on_u[p];
            DV[p] = DV[p] + (cff1 * (double)DVp) * (double)g.om_v[p];
        }
    }
    if (mode == 2 && i != 0 && j != 0) {
        if (!in) rz = rzeta[p];
        zeta_t2[p] = zeta_t0[p] + Dt * rz;
    }
}

// computeZetaPred alone (mod_cppkernels.cpp:134-150).
template <typename R>
__global__ void __launch_bounds__(kBlock) k_zeta_pred(Geo<R> g, R Dt, const R *__restrict__ z0,
                                                      R *__restrict__ z2,
                                                      const R *__restrict__ rz1) {
    const long p = tid_flat();
    if (p >= g.s2) return;
    if ((p % g.I) == 0 || (p / g.I) == 0) return;
    z2[p] = z0[p] + Dt * rz1[p];
}

// Forward-Euler branch of step2dPredictor (nonlinear/step2d.py:50), every point.
template <typename R>
__global__ void __launch_bounds__(kBlock) k_zeta_euler(Geo<R> g, R Dt, const R *__restrict__ z1,
                                                       R *__restrict__ z2,
                                                       const R *__restrict__ rz1) {
    const long p = tid_flat();
    if (p >= g.s2) return;
    z2[p] = z1[p] + Dt * rz1[p];
}

// computeMomentumRHSPred/Corr (mod_cppkernels.cpp:13-77) fused with computeMomentumPred
// (:156-186), whose guard tests the flat index against szJ, the row count (:162).
template <typename R>
__global__ void __launch_bounds__(kBlock) k_momentum(
    Geo<R> g, R *__restrict__ rhs_u, R *__restrict__ rhs_v, const R *__restrict__ za,
    const R *__restrict__ zb, R grav, R w1, R w, int do_rhs, int do_pred, R Dt,
    const R *__restrict__ u_t1, R *__restrict__ u_t2, const R *__restrict__ v_t1,
    R *__restrict__ v_t2, const R *__restrict__ z1, const R *__restrict__ z2) {
    const long p = tid_flat();
    if (p >= g.s2) return;
    const long I = g.I, J = g.J;
    const int i = (int)(p % I), j = (int)(p / I);
    const R *h = g.h;
    const bool in = do_rhs && rint_(i, j, g.I, g.J);
    R ru = R(0), rv = R(0);
    if (in) {
        const R gp = w1 * za[p] + w * zb[p];
        const R gw = w1 * za[p - 1] + w * zb[p - 1];
        const R gs = w1 * za[p - I] + w * zb[p - I];
        ru = (grav * g.on_u[p]) * (((h[p] + h[p - 1]) * R(0.5)) * (gp - gw) + R(0.5) * (gp * gp - gw * gw));
        rv = (grav * g.om_v[p]) * (((h[p] + h[p - I]) * R(0.5)) * (gp - gs) + R(0.5) * (gp * gp - gs * gs));
        rhs_u[p] = ru;
        rhs_v[p] = rv;
    }
    if (do_pred && (p % J) != 0 && p >= J) {
        if (!in) {
            ru = rhs_u[p];
            rv = rhs_v[p];
        }
        const R D1p = z1[p] + h[p], D2p = z2[p] + h[p];
        const R D1U = (D1p + (z1[p - 1] + h[p - 1])) * R(0.5);
        const R D2U = (D2p + (z2[p - 1] + h[p - 1])) * R(0.5);
        // p - I < 0 only on row 0 of grids with more columns than rows; the reference reads
        // before the array there, and the result is overwritten by the closed boundary and by
        // vbar_t2[:] = 0 (nonlinear/main3d.py:189) before anything reads it.
        const R D1V = (D1p + (ldz(z1, p - I) + ldz(h, p - I))) * R(0.5);
        const R D2V = (D2p + (ldz(z2, p - I) + ldz(h, p - I))) * R(0.5);
        u_t2[p] = (u_t1[p] * D1U + ((Dt * ru) * g.pm[p]) * g.pn[p]) / D2U;
        v_t2[p] = (v_t1[p] * D1V + ((Dt * rv) * g.pm[p]) * g.pn[p]) / D2V;
    }
}

// AdamsMoultonCorr3rd (mod_cppkernels.cpp:191-209).
template <typename R>
__global__ void __launch_bounds__(kBlock) k_am3(Geo<R> g, R Dt, R *__restrict__ v,
                                                const R *__restrict__ r0, const R *__restrict__ r1,
                                                const R *__restrict__ r2) {
    const long p = tid_flat();
    if (p >= g.s2) return;
    const R A2 = R(5.0 / 12.0), A1 = R(8.0 / 12.0), A0 = R(-1.0 / 12.0);
    v[p] = v[p] + Dt * ((A2 * r2[p] + A1 * r1[p]) + A0 * r0[p]);
}

// The pointwise part of step2dCorrector (nonlinear/step2d.py:109 and :120-123) plus
// vbar_t2[:] = 0 (nonlinear/main3d.py:189):
//   zeta_t2 += Dt*(5/12 rzeta_t2 + 8/12 rzeta_t1 - 1/12 rzeta_t0)
//   ubar_t1 += Dt*(5/12 rubar_t1 + 8/12 rubar_t0 - 1/12 vbar_t1)   (the mis-bound
//              AdamsMoultonCorr3rd2 of modules/mod_operators.py:146 reads these five args)
template <typename R>
__global__ void __launch_bounds__(kBlock) k_corr_point(
    Geo<R> g, R Dt, R *__restrict__ zeta_t2, const R *__restrict__ rz0, const R *__restrict__ rz1,
    const R *__restrict__ rz2, R *__restrict__ ubar_t1, const R *__restrict__ vbar_t1,
    const R *__restrict__ rub0, const R *__restrict__ rub1, R *__restrict__ vbar_t2) {
    const long p = tid_flat();
    if (p >= g.s2) return;
    const R A2 = R(5.0 / 12.0), A1 = R(8.0 / 12.0), A0 = R(-1.0 / 12.0);
    zeta_t2[p] = zeta_t2[p] + Dt * ((A2 * rz2[p] + A1 * rz1[p]) + A0 * rz0[p]);
    ubar_t1[p] = ubar_t1[p] + Dt * ((A2 * rub1[p] + A1 * rub0[p]) + A0 * vbar_t1[p]);
    if (vbar_t2) vbar_t2[p] = R(0);
}

// Boundary programs (see BcProgram): one block, gather everything, barrier, scatter.
template <typename R>
__global__ void __launch_bounds__(1024) k_bc_apply(int n1, const int *__restrict__ d1,
                                                   const int *__restrict__ s1, R *f1, int n2,
                                                   const int *__restrict__ d2,
                                                   const int *__restrict__ s2, R *f2, R val) {
    extern __shared__ unsigned char smem_raw[];
    R *buf = reinterpret_cast<R *>(smem_raw);
    for (int k = threadIdx.x; k < n1; k += blockDim.x) {
        const int s = s1[k];
        buf[k] = s >= 0 ? f1[s] : (s == -1 ? R(0) : val);
    }
    for (int k = threadIdx.x; k < n2; k += blockDim.x) {
        const int s = s2[k];
        buf[n1 + k] = s >= 0 ? f2[s] : (s == -1 ? R(0) : val);
    }
    __syncthreads();
    for (int k = threadIdx.x; k < n1; k += blockDim.x) f1[d1[k]] = buf[k];
    for (int k = threadIdx.x; k < n2; k += blockDim.x) f2[d2[k]] = buf[n1 + k];
}

// ------------------------------------------------------------------------------------------
// 3D right-hand side (nonlinear/rhs.py:16-93): ru = rv = 0, addCoriolis (rhs_kernels.cpp:7-35),
// horizontalAdvection (:71-132), verticalAdvection (:136-196), one thread per column.
// ------------------------------------------------------------------------------------------
template <typename R>
struct Hadv {
    // Evaluates horizontalAdvection's ru and rv increments at flat node p of level base K.
    const R *U, *V, *HU, *HV;   // level-K pointers (may be indexed below 0 at K = 0)
    long I;
    bool lo;                    // level 0: guard reads before the array start
    long base;                  // K*s2, for the guard
    __device__ __forceinline__ R u_(long q) const { return lo ? ldz(U - base, base + q) : U[q]; }
    __device__ __forceinline__ R v_(long q) const { return lo ? ldz(V - base, base + q) : V[q]; }
    __device__ __forceinline__ R hu(long q) const { return lo ? ldz(HU - base, base + q) : HU[q]; }
    __device__ __forceinline__ R hv(long q) const { return lo ? ldz(HV - base, base + q) : HV[q]; }
    __device__ __forceinline__ R uR(long q) const { return (u_(q) + u_(q + 1)) * R(0.5); }
    __device__ __forceinline__ R uP(long q) const { return (u_(q) + u_(q - 1)) * R(0.5); }
    __device__ __forceinline__ R vR(long q) const { return (v_(q) + v_(q + I)) * R(0.5); }
    __device__ __forceinline__ R vP(long q) const { return (v_(q) + v_(q - I)) * R(0.5); }
    __device__ __forceinline__ R huR(long q) const { return (hu(q) + hu(q + 1)) * R(0.5); }
    __device__ __forceinline__ R huP(long q) const { return (hu(q) + hu(q - 1)) * R(0.5); }
    __device__ __forceinline__ R hvP(long q) const { return (hv(q) + hv(q - I)) * R(0.5); }
    __device__ __forceinline__ R hvR(long q) const { return (hv(q) + hv(q + I)) * R(0.5); }
    __device__ __forceinline__ R dxxU(long q) const { return (u_(q - 1) - R(2.0) * u_(q)) + u_(q + 1); }
    __device__ __forceinline__ R deeU(long q) const { return (u_(q - I) - R(2.0) * u_(q)) + u_(q + I); }
    __device__ __forceinline__ R dxxHU(long q) const { return (hu(q - 1) - R(2.0) * hu(q)) + hu(q + 1); }
    __device__ __forceinline__ R deeHU(long q) const { return (hu(q - I) - R(2.0) * hu(q)) + hu(q + I); }
    __device__ __forceinline__ R dxxHV(long q) const { return (hv(q - 1) - R(2.0) * hv(q)) + hv(q + 1); }
    __device__ __forceinline__ R deeHV(long q) const { return (hv(q - I) - R(2.0) * hv(q)) + hv(q + I); }
    // upwindUtoR(DxxUtoU(u), uR) and upwindUtoP(DeeUtoU(u), HvomP), mod_cppkernels.h:624,673
    __device__ __forceinline__ R uxxR(long q) const { return (uR(q) + uR(q + 1) >= R(0)) ? dxxU(q) : dxxU(q + 1); }
    __device__ __forceinline__ R ueeP(long q) const { return (hvP(q) + hvP(q - I) >= R(0)) ? deeU(q) : deeU(q - I); }
    __device__ __forceinline__ R huxxR(long q) const { return (dxxHU(q) + dxxHU(q + 1)) * R(0.5); }
    __device__ __forceinline__ R hueeP(long q) const { return (deeHU(q) + deeHU(q - 1)) * R(0.5); }
    __device__ __forceinline__ R hvxxP(long q) const { return (dxxHV(q) + dxxHV(q - I)) * R(0.5); }
    __device__ __forceinline__ R hveeR(long q) const { return (deeHV(q) + deeHV(q + I)) * R(0.5); }
    // Fluxes as written at rhs_kernels.cpp:121-125 (Gadv = -0.5).
    __device__ __forceinline__ R ufxR(long q) const { return uR(q) + (R(-0.5) * uxxR(q)) * (huR(q) + R(-0.5) * huxxR(q)); }
    __device__ __forceinline__ R ufeP(long q) const { return uP(q) + (R(-0.5) * ueeP(q)) * (hvP(q) + R(-0.5) * hvxxP(q)); }
    __device__ __forceinline__ R vfxP(long q) const { return vP(q) + (R(-0.5) * ueeP(q)) * (huP(q) + R(-0.5) * hueeP(q)); }
    __device__ __forceinline__ R vfeR(long q) const { return vR(q) + (R(-0.5) * uxxR(q)) * (hvR(q) + R(-0.5) * hveeR(q)); }
    __device__ __forceinline__ R du(long p) const { return (ufxR(p) - ufxR(p - 1)) + (ufeP(p) - ufeP(p - I)); }
    __device__ __forceinline__ R dv(long p) const { return (vfxP(p) - vfxP(p - 1)) + (vfeR(p) - vfeR(p - I)); }
};

template <typename R>
__global__ void __launch_bounds__(128) k_rhs3d(Geo<R> g, const R *__restrict__ u,
                                               const R *__restrict__ v, const R *__restrict__ Huon,
                                               const R *__restrict__ Hvom, const R *__restrict__ W,
                                               const R *__restrict__ Hz, R *__restrict__ ru,
                                               R *__restrict__ rv) {
    const long p = tid_flat();
    if (p >= g.s2) return;
    const long I = g.I, s2 = g.s2;
    const int N = g.N;
    const int i = (int)(p % I), j = (int)(p / I);
    const bool rn = rnode_(i, j);
    const bool va = g.bcfield[p] < 0 && inner_(i, j, g.I, g.J);   // rhs_kernels.cpp:144-149
    const R c9 = R(9.0 / 16.0), c1 = R(1.0 / 16.0);

    // Vertical-advection helpers: 4th-order interpolations (mod_cppkernels.h:723,745,767).
#define AT(X, k) ((X)[(long)(k) * s2 + p])
#define U4(X, k) (c9 * (AT(X, k) + AT(X, (k) + 1)) - c1 * (AT(X, (k) - 1) + AT(X, (k) + 2)))
#define WU4(k) (c9 * (W[(long)(k) * s2 + p] + W[(long)(k) * s2 + p + 1]) - \
                c1 * (W[(long)(k) * s2 + p - 1] + W[(long)(k) * s2 + p + 2]))
#define WV4(k) (c9 * (W[(long)(k) * s2 + p] + W[(long)(k) * s2 + p + I]) - \
                c1 * (W[(long)(k) * s2 + p - I] + W[(long)(k) * s2 + p + 2 * I]))
    R ruN3 = R(0), rvN3 = R(0), ru1 = R(0), rv1 = R(0);
    R fu_k = R(0), fv_k = R(0);   // Fsigma at level K (vertical advection, K >= 2)
    R uuu = R(0), uuu2 = R(0);
    if (va) {
        uuu = (c9 * (AT(u, 0) + AT(u, 1)) - c1 * (0 + AT(u, 2))) * WU4(1);
        uuu2 = (c9 * (0 + AT(u, 0)) - c1 * (0 + AT(u, 1))) * WU4(0);
    }
    for (int K = 0; K < N; ++K) {
        const long o = (long)K * s2;
        R aru = R(0), arv = R(0);
        if (rn) {   // addCoriolis
            const R cffp = Hz[o + p] * g.fomn[p], cffw = Hz[o + p - 1] * g.fomn[p - 1];
            const R cffs = Hz[o + p - I] * g.fomn[p - I];
            const R UFp = cffp * ((v[o + p] + v[o + p + I]) * R(0.5));
            const R UFw = cffw * ((v[o + p - 1] + v[o + p - 1 + I]) * R(0.5));
            const R VFp = cffp * ((u[o + p] + u[o + p + 1]) * R(0.5));
            const R VFs = cffs * ((u[o + p - I] + u[o + p - I + 1]) * R(0.5));
            aru = aru + (UFp + UFw) * R(0.5);
            arv = arv - (VFp + VFs) * R(0.5);
        }
        {   // horizontalAdvection
            Hadv<R> a{u + o, v + o, Huon + o, Hvom + o, I, K == 0, o};
            aru = aru - a.du(p);
            arv = arv - a.dv(p);
        }
        // The reference's out-of-range threads (p >= s2) store 0 at flat p, i.e. into levels
        // >= 1, after the in-range threads (rhs_kernels.cpp:86-91).
        if (K >= 1 && o + p < g.ref_threads) {
            aru = R(0);
            arv = R(0);
        }
        if (va) {   // verticalAdvection
            if (K == 0) {
                aru = aru - (uuu - uuu2);
            } else if (K == 1) {
                const R f1 = U4(v, 1) * WV4(1), f2 = U4(v, 2) * WV4(2), f3 = U4(v, 3) * WV4(3);
                arv -= c9 * (f1 + f2) - c1 * (f1 + f3);
                fu_k = U4(u, 2) * WU4(2);
                fv_k = f2;
                aru = aru - (fu_k - uuu);
            } else if (K <= N - 3) {
                const R fu1 = U4(u, K + 1) * WU4(K + 1), fv1 = U4(v, K + 1) * WV4(K + 1);
                aru = aru - (fu1 - fu_k);
                arv = arv - (fv1 - fv_k);
                fu_k = fu1;
                fv_k = fv1;
            } else {
                aru = ruN3;    // ru[N-2] = ru[N-3], ru[N-1] = ru[N-2] (:189-192)
                arv = rvN3;
            }
            if (K == N - 3) {
                ruN3 = aru;
                rvN3 = arv;
            }
            if (K == 1) {
                ru1 = aru;
                rv1 = arv;
            }
        }
        ru[o + p] = aru;
        rv[o + p] = (va && K == 0) ? R(0) : arv;   // rv[0] is set from rv[1] below
    }
    const long oN = (long)N * s2;
    ru[oN + p] = va ? ruN3 : R(0);   // ru_t2[:] = 0 (rhs.py:38); ru[N] = ru[N-2] (:193)
    rv[oN + p] = va ? rvN3 : R(0);
    if (va) rv[p] = rv1;             // rv[0] = rv[1] (:183)
    (void)ru1;
#undef WV4
#undef WU4
#undef U4
#undef AT
}

// ------------------------------------------------------------------------------------------
// set_maxflux (step3D_uv.kernels.cpp:372-405) + omega (:62-165) + set_zeta (:294-310)
// ------------------------------------------------------------------------------------------
template <typename R>
struct Flux {
    // Huon/Hvom at flat index f (any level): recomputed when this kernel also writes it (the
    // value is the one its owner thread stores), read from memory otherwise.
    const Geo<R> *g;
    const R *u, *v, *Hz, *Huon, *Hvom;
    bool recompute;
    __device__ __forceinline__ R hu(long f) const {
        if (recompute) {
            const long K = f / g->s2, q = f - K * g->s2;
            const int i = (int)(q % g->I), j = (int)(q / g->I);
            if (K < g->N && unode_(i, j))
                return (((Hz[f] + Hz[f - 1]) * R(0.5)) * u[f]) * g->on_u[q];
        }
        return Huon[f];
    }
    __device__ __forceinline__ R hv(long f) const {
        if (recompute) {
            const long K = f / g->s2, q = f - K * g->s2;
            const int i = (int)(q % g->I), j = (int)(q / g->I);
            if (K < g->N && vnode_(i, j, g->J))
                return (((Hz[f] + Hz[f - g->I]) * R(0.5)) * v[f]) * g->om_v[q];
        }
        return Hvom[f];
    }
};

template <typename R>
__global__ void __launch_bounds__(kBlock) k_maxflux_omega(
    Geo<R> g, const R *__restrict__ u, const R *__restrict__ v, R *Huon, R *Hvom,
    const R *__restrict__ Hz, R *__restrict__ W, const R *__restrict__ z_w, int do_flux,
    int do_omega, R *__restrict__ zeta1, R *__restrict__ zeta2, const double *__restrict__ Zt) {
    const long p = tid_flat();
    if (p >= g.s2) return;
    const long I = g.I, s2 = g.s2;
    const int N = g.N;
    const int i = (int)(p % I), j = (int)(p / I);
    if (do_flux) {
        if (unode_(i, j))
            for (int K = 0; K < N; ++K) {
                const long o = (long)K * s2 + p;
                Huon[o] = (((Hz[o] + Hz[o - 1]) * R(0.5)) * u[o]) * g.on_u[p];
            }
        if (vnode_(i, j, g.J))
            for (int K = 0; K < N; ++K) {
                const long o = (long)K * s2 + p;
                Hvom[o] = (((Hz[o] + Hz[o - I]) * R(0.5)) * v[o]) * g.om_v[p];
            }
    }
    if (do_omega && g.bcfield[p] < 0) {
        Flux<R> fx{&g, u, v, Hz, Huon, Hvom, do_flux != 0};
        R Wk = R(0);
        W[p] = R(0);
        for (int K = 1; K < N; ++K) {
            const long o = (long)K * s2 + p;
            Wk = Wk - ((fx.hu(o + 1) - fx.hu(o)) + (fx.hv(o + I) - fx.hv(o)));
            W[o] = Wk;
        }
        const R zbed = z_w[p];
        const R h = z_w[(long)(N - 1) * s2 + p] - zbed;
        const R Ws = Wk;
        for (int K = N - 1; K > 0; --K) {
            const long o = (long)K * s2 + p;
            W[o] = W[o] - (Ws * (z_w[o] - zbed)) / h;
        }
        W[(long)N * s2 + p] = R(0);
    }
    if (zeta1 && rnode_(i, j)) {
        zeta2[p] = (R)Zt[p];
        zeta1[p] = (R)Zt[p];
    }
}

// set_zeta alone (step3D_uv.kernels.cpp:294-310).
template <typename R>
__global__ void __launch_bounds__(kBlock) k_set_zeta(Geo<R> g, R *__restrict__ z1,
                                                     R *__restrict__ z2,
                                                     const double *__restrict__ Zt) {
    const long p = tid_flat();
    if (p >= g.s2) return;
    if (!rnode_((int)(p % g.I), (int)(p / g.I))) return;
    z2[p] = (R)Zt[p];
    z1[p] = (R)Zt[p];
}

// set_depth (step3D_uv.kernels.cpp:225-291), FP64 arithmetic.
template <typename R>
__global__ void __launch_bounds__(kBlock) k_set_depth(Geo<R> g, const double *__restrict__ Zt,
                                                      R *__restrict__ z_w, R *__restrict__ z_r,
                                                      R *__restrict__ Hz) {
    const long p = tid_flat();
    if (p >= g.s2) return;
    const long s2 = g.s2;
    const int N = g.N;
    const double hc = g.hc, h = g.hd[p], zt = Zt[p];
    double zprev = 0.0;
    for (int K = 0; K <= N; ++K) {
        double zw;
        if (K == N) {
            zw = zt;
        } else if (g.Vtransform == 1) {
            const double z_r0 = hc * (g.sc_r[K] - g.Cs_r[K]) + g.Cs_r[K] * h;
            const double z_w0 = hc * (g.sc_w[K] - g.Cs_w[K]) + g.Cs_w[K] * h;
            zw = z_w0 + zt * (1.0 + z_w0 / h);
            z_r[(long)K * s2 + p] = (R)(z_r0 + zt * (1.0 + z_r0 / h));
        } else {
            const double cff2_r = (hc * g.sc_r[K] + g.Cs_r[K] * h) / (hc + h);
            const double cff2_w = (hc * g.sc_w[K] + g.Cs_w[K] * h) / (hc + h);
            zw = zt + (zt + h) * cff2_w;
            z_r[(long)K * s2 + p] = (R)(zt + (zt + h) * cff2_r);
        }
        z_w[(long)K * s2 + p] = (R)zw;
        if (K > 0) Hz[(long)(K - 1) * s2 + p] = (R)(zw - zprev);
        zprev = zw;
    }
}

// ------------------------------------------------------------------------------------------
// step3d_UV (step3D_uv.kernels.cpp:646-707): implicit vertical viscosity per U and V column
// (Thomas algorithm in per-thread arrays), baroclinic-mean correction, 2D/3D coupling, and
// optionally setLateralUVBCs (:314-368) for the same column.
// ------------------------------------------------------------------------------------------
template <typename R>
struct Column {
    R FC[kNMax], BD[kNMax], RHS[kNMax];
};

// createVertViscousOpMatrix (:568-639) for the column at p; d = 1 (U) or I (V).
template <typename R>
__device__ __forceinline__ void build_matrix(const Geo<R> &g, long p, long d, R cff, R Dt,
                                             R lambda, Column<R> &c, const R *Hz, const R *Akv,
                                             const R *z_r, const R *uold, const R *ru) {
    const long s2 = g.s2;
    const int N = g.N;
    const R pmU = (g.pm[p] + g.pm[p - d]) * R(0.5), pnU = (g.pn[p] + g.pn[p - d]) * R(0.5);
    const R cdt = cff * Dt;
    const R cm = -lambda * Dt;
#define HZU(k) ((Hz[(long)(k) * s2 + p] + Hz[(long)(k) * s2 + p - d]) * R(0.5))
#define AKU(k) ((Akv[(long)(k) * s2 + p] + Akv[(long)(k) * s2 + p - d]) * R(0.5))
#define DZ(k) (((z_r[(long)(k) * s2 + p] - z_r[(long)((k) - 1) * s2 + p]) + \
                (z_r[(long)(k) * s2 + p - d] - z_r[(long)((k) - 1) * s2 + p - d])) * R(0.5))
    c.FC[N - 1] = R(0);
    for (int K = 0; K < N - 1; ++K) c.FC[K] = (cm * AKU(K)) / DZ(K + 1);
    c.RHS[0] = R(0);
    for (int K = 1; K < N; ++K) {
        const R hzu = HZU(K);
        c.RHS[K] = hzu * (uold[(long)K * s2] + (cdt * (pmU * pnU)) * ru[(long)K * s2 + p]);
        c.BD[K] = (hzu - c.FC[K]) - c.FC[K - 1];
    }
    c.BD[N - 1] = HZU(N - 1) - c.FC[N - 2];
    c.BD[0] = HZU(0) - R(2.0) * c.FC[0];
#undef DZ
#undef AKU
#undef HZU
}

// solveTri (:520-565); the solution goes to loc[0..N).
template <typename R>
__device__ __forceinline__ void solve_tri(int N, Column<R> &c, R *loc) {
    for (int k = 1; k < N; ++k) {
        const R w = c.FC[k - 1] / c.BD[k - 1];
        c.BD[k] = c.BD[k] - w * c.FC[k - 1];
        c.RHS[k] = c.RHS[k] - w * c.RHS[k - 1];
    }
    R x = c.RHS[N - 1] / c.BD[N - 1];
    loc[N - 1] = x;
    for (int k = N - 2; k >= 0; --k) {
        x = (c.RHS[k] - c.FC[k] * x) / c.BD[k];
        loc[k] = x;
    }
}

template <typename R>
__global__ void __launch_bounds__(128) k_step3d_uv(
    Geo<R> g, R *__restrict__ u, R *__restrict__ v, const R *__restrict__ ru,
    const R *__restrict__ rv, R *__restrict__ ubar_t1, R *__restrict__ vbar_t1,
    R *__restrict__ ubar_t2, R *__restrict__ vbar_t2, const R *__restrict__ Hz,
    const R *__restrict__ Akv, const R *__restrict__ z_r, const double *__restrict__ DU,
    const double *__restrict__ DV, const R *tmpU, const R *tmpV, R cff, R lambda, R Dt,
    int do_bc, R bcval) {
    const long p = tid_flat();
    if (p >= g.s2) return;
    const long I = g.I, s2 = g.s2;
    const int N = g.N;
    const int i = (int)(p % I), j = (int)(p / I);
    const bool un = unode_(i, j), vn = vnode_(i, j, g.J);
    if (un || vn) {
        Column<R> c;
        R unew[kNMax], vnew[kNMax];
        const R *uo = (tmpU ? tmpU : u) + p;
        const R *vo = (tmpV ? tmpV : v) + p;
        if (un) {
            build_matrix(g, p, 1, cff, Dt, lambda, c, Hz, Akv, z_r, uo, ru);
            solve_tri(N, c, unew);
            // correctBaroclinicMeanVel<ntU> (:475-517), against the pre-step velocity.
            double H = 0.0, Hu = 0.0;
            for (int K = 0; K < N; ++K) {
                const long o = (long)K * s2 + p;
                const R hzu = (Hz[o] + Hz[o - 1]) * R(0.5);
                H += (double)hzu;
                Hu += (double)(uo[(long)K * s2] * hzu);
            }
            const R udiff = (R)((Hu - DU[p] / (double)g.on_u[p]) / H);
            for (int K = 0; K < N; ++K) unew[K] = unew[K] - udiff;
        }
        if (vn) build_matrix(g, p, I, cff, Dt, lambda, c, Hz, Akv, z_r, vo, rv);
        bool vsolved = false;
        if (un) {   // solveTri is gated by isUNode for both directions (:525)
            solve_tri(N, c, vnew);
            vsolved = true;
        }
        if (vn) {
            if (!vsolved)   // no solve at this node: the correction applies to v as it is
                for (int K = 0; K < N; ++K) vnew[K] = v[(long)K * s2 + p];
            double H = 0.0, Hv = 0.0;
            for (int K = 0; K < N; ++K) {
                const long o = (long)K * s2 + p;
                const R hzv = (Hz[o] + Hz[o - I]) * R(0.5);
                H += (double)hzv;
                Hv += (double)(vo[(long)K * s2] * hzv);
            }
            const R vdiff = (R)((Hv - DV[p] / (double)g.om_v[p]) / H);
            for (int K = 0; K < N; ++K) vnew[K] = vnew[K] - vdiff;
        }
        if (un)
            for (int K = 0; K < N; ++K) u[(long)K * s2 + p] = unew[K];
        if (un || vn)
            if (vsolved || vn)
                for (int K = 0; K < N; ++K) v[(long)K * s2 + p] = vnew[K];
        if (un) {   // adjustBarotropicVelocity (:408-469)
            double HU = 0.0, HV = 0.0, HuU = 0.0, HvV = 0.0;
            for (int K = 0; K < N; ++K) {
                const long o = (long)K * s2 + p;
                const R hzu = (Hz[o] + Hz[o - 1]) * R(0.5), hzv = (Hz[o] + Hz[o - I]) * R(0.5);
                HU += (double)hzu;
                HV += (double)hzv;
                HuU += (double)(hzu * unew[K]);
                HvV += (double)(hzv * vnew[K]);
            }
            const double duo = DU[p] / (double)g.on_u[p], dvo = DV[p] / (double)g.om_v[p];
            const double uUpdate = (HuU - duo) / HU;
            const double vUpdate = (HvV - dvo) / HV;
            const R ub = (R)(duo / HU + uUpdate), vb = (R)(dvo / HV + vUpdate);
            ubar_t2[p] = ub;
            vbar_t2[p] = vb;
            ubar_t1[p] = ub;
            vbar_t1[p] = vb;
        }
    }
    if (do_bc) {   // setLateralUVBCs (:314-368); gradient types are rejected at context creation
        const int ut = g.utype[p], vt = g.vtype[p];
        if (ut > 0 && (ut & (1 << 4)) == 0 && (ut & (1 << 3)) != 0)
            for (int K = 0; K < N; ++K) u[(long)K * s2 + p] = bcval;
        if (vt > 0 && ((vt & (1 << 4)) != 0 || (vt & (1 << 3)) != 0))
            for (int K = 0; K < N; ++K) v[(long)K * s2 + p] = R(0);
    }
}

// setLateralUVBCs alone (step3D_uv.kernels.cpp:314-368).
template <typename R>
__global__ void __launch_bounds__(kBlock) k_lateral_uv_bc(Geo<R> g, R *__restrict__ u,
                                                          R *__restrict__ v, R bcval) {
    const long p = tid_flat();
    if (p >= g.s2) return;
    const long s2 = g.s2;
    const int ut = g.utype[p], vt = g.vtype[p];
    if (ut <= 0 && vt <= 0) return;
    if (ut > 0 && (ut & (1 << 4)) == 0 && (ut & (1 << 3)) != 0)
        for (int K = 0; K < g.N; ++K) u[(long)K * s2 + p] = bcval;
    if (vt > 0 && ((vt & (1 << 4)) != 0 || (vt & (1 << 3)) != 0))
        for (int K = 0; K < g.N; ++K) v[(long)K * s2 + p] = R(0);
}

// ------------------------------------------------------------------------------------------
// Launchers
// ------------------------------------------------------------------------------------------
inline unsigned blocks_for(long n, int b) { return (unsigned)((n + b - 1) / b); }

template <typename R>
Geo<R> Ops<R>::geo(const sf_ctx *c) {
    Geo<R> g;
    g.I = c->I;
    g.J = c->J;
    g.N = c->N;
    g.s2 = c->s2;
    g.h = (const R *)c->metrics[0];
    g.pm = (const R *)c->metrics[1];
    g.pn = (const R *)c->metrics[2];
    g.on_u = (const R *)c->metrics[3];
    g.om_v = (const R *)c->metrics[4];
    g.fomn = (const R *)c->metrics[5];
    g.hd = c->hd;
    g.sc_r = c->vert;
    g.sc_w = c->vert + c->N;
    g.Cs_r = c->vert + 2 * c->N + 1;
    g.Cs_w = c->vert + 3 * c->N + 1;
    g.hc = c->hc;
    g.Vtransform = c->Vtransform;
    g.bcfield = c->bcfield;
    g.utype = c->utype;
    g.vtype = c->vtype;
    g.ref_threads = c->ref_threads;
    return g;
}

template <typename R>
cudaError_t Ops<R>::zeta_rhs(const sf_ctx *c, const R *zeta, const R *ubar, const R *vbar,
                             R *rzeta, int mode, double cff1, double *Zt, double *DU, double *DV,
                             const R *zeta_t0, R *zeta_t2, double Dt, cudaStream_t s) {
    k_zeta_rhs<R><<<blocks_for(c->s2, kBlock), kBlock, 0, s>>>(geo(c), zeta, ubar, vbar, rzeta,
                                                               mode, cff1, Zt, DU, DV, zeta_t0,
                                                               zeta_t2, (R)Dt);
    return cudaGetLastError();
}
template <typename R>
cudaError_t Ops<R>::zeta_pred(const sf_ctx *c, double Dt, const R *z0, R *z2, const R *rz1,
                              cudaStream_t s) {
    k_zeta_pred<R><<<blocks_for(c->s2, kBlock), kBlock, 0, s>>>(geo(c), (R)Dt, z0, z2, rz1);
    return cudaGetLastError();
}
template <typename R>
cudaError_t Ops<R>::zeta_euler(const sf_ctx *c, double Dt, const R *z1, R *z2, const R *rz1,
                               cudaStream_t s) {
    k_zeta_euler<R><<<blocks_for(c->s2, kBlock), kBlock, 0, s>>>(geo(c), (R)Dt, z1, z2, rz1);
    return cudaGetLastError();
}
template <typename R>
cudaError_t Ops<R>::momentum(const sf_ctx *c, R *rhs_u, R *rhs_v, const R *za, const R *zb,
                             double g, double weight, int do_rhs, int do_pred, double Dt,
                             const R *u_t1, R *u_t2, const R *v_t1, R *v_t2, const R *z1,
                             const R *z2, cudaStream_t s) {
    const double w1 = 1 - weight;
    k_momentum<R><<<blocks_for(c->s2, kBlock), kBlock, 0, s>>>(
        geo(c), rhs_u, rhs_v, za, zb, (R)g, (R)w1, (R)weight, do_rhs, do_pred, (R)Dt, u_t1, u_t2,
        v_t1, v_t2, z1, z2);
    return cudaGetLastError();
}
template <typename R>
cudaError_t Ops<R>::am3(const sf_ctx *c, double Dt, R *v, const R *r0, const R *r1, const R *r2,
                        cudaStream_t s) {
    k_am3<R><<<blocks_for(c->s2, kBlock), kBlock, 0, s>>>(geo(c), (R)Dt, v, r0, r1, r2);
    return cudaGetLastError();
}
template <typename R>
cudaError_t Ops<R>::corr_point(const sf_ctx *c, double Dt, R *zeta_t2, const R *rz0,
                               const R *rz1, const R *rz2, R *ubar_t1, const R *vbar_t1,
                               const R *rub0, const R *rub1, R *vbar_t2, cudaStream_t s) {
    k_corr_point<R><<<blocks_for(c->s2, kBlock), kBlock, 0, s>>>(
        geo(c), (R)Dt, zeta_t2, rz0, rz1, rz2, ubar_t1, vbar_t1, rub0, rub1, vbar_t2);
    return cudaGetLastError();
}
template <typename R>
cudaError_t Ops<R>::bc_apply(const sf_ctx *c, const BcProgram &p1, R *f1, const BcProgram &p2,
                             R *f2, double val, cudaStream_t s) {
    const int n = p1.n + p2.n;
    if (n == 0) return cudaSuccess;
    const size_t smem = (size_t)n * sizeof(R);
    if (smem > 48 * 1024) {
        cudaError_t e = cudaFuncSetAttribute(k_bc_apply<R>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                             (int)smem);
        if (e != cudaSuccess) return e;
    }
    k_bc_apply<R><<<1, 1024, smem, s>>>(p1.n, p1.dst, p1.src, f1, p2.n, p2.dst, p2.src, f2, (R)val);
    return cudaGetLastError();
}
template <typename R>
cudaError_t Ops<R>::rhs3d(const sf_ctx *c, const R *u, const R *v, const R *Huon, const R *Hvom,
                          const R *W, const R *Hz, R *ru, R *rv, cudaStream_t s) {
    k_rhs3d<R><<<blocks_for(c->s2, 128), 128, 0, s>>>(geo(c), u, v, Huon, Hvom, W, Hz, ru, rv);
    return cudaGetLastError();
}
template <typename R>
cudaError_t Ops<R>::maxflux_omega(const sf_ctx *c, const R *u, const R *v, R *Huon, R *Hvom,
                                  const R *Hz, R *W, const R *z_w, int do_flux, int do_omega,
                                  R *zeta1, R *zeta2, const double *Zt, cudaStream_t s) {
    k_maxflux_omega<R><<<blocks_for(c->s2, kBlock), kBlock, 0, s>>>(
        geo(c), u, v, Huon, Hvom, Hz, W, z_w, do_flux, do_omega, zeta1, zeta2, Zt);
    return cudaGetLastError();
}
template <typename R>
cudaError_t Ops<R>::set_zeta(const sf_ctx *c, R *z1, R *z2, const double *Zt, cudaStream_t s) {
    k_set_zeta<R><<<blocks_for(c->s2, kBlock), kBlock, 0, s>>>(geo(c), z1, z2, Zt);
    return cudaGetLastError();
}
template <typename R>
cudaError_t Ops<R>::set_depth(const sf_ctx *c, const double *Zt, R *z_w, R *z_r, R *Hz,
                              cudaStream_t s) {
    k_set_depth<R><<<blocks_for(c->s2, kBlock), kBlock, 0, s>>>(geo(c), Zt, z_w, z_r, Hz);
    return cudaGetLastError();
}
template <typename R>
cudaError_t Ops<R>::step3d_uv(const sf_ctx *c, R *u, R *v, const R *ru, const R *rv, R *ubar_t1,
                              R *vbar_t1, R *ubar_t2, R *vbar_t2, const R *Hz, const R *Akv,
                              const R *z_r, const double *DU, const double *DV, const R *tmpU,
                              const R *tmpV, double cff, double lambda, double Dt, int do_bc,
                              double bcval, cudaStream_t s) {
    k_step3d_uv<R><<<blocks_for(c->s2, 128), 128, 0, s>>>(
        geo(c), u, v, ru, rv, ubar_t1, vbar_t1, ubar_t2, vbar_t2, Hz, Akv, z_r, DU, DV, tmpU, tmpV,
        (R)cff, (R)lambda, (R)Dt, do_bc, (R)bcval);
    return cudaGetLastError();
}
template <typename R>
cudaError_t Ops<R>::lateral_uv_bc(const sf_ctx *c, R *u, R *v, double val, cudaStream_t s) {
    k_lateral_uv_bc<R><<<blocks_for(c->s2, kBlock), kBlock, 0, s>>>(geo(c), u, v, (R)val);
    return cudaGetLastError();
}

}  // namespace sf
