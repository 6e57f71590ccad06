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
#include <type_traits>
#include <cuda_runtime.h>
#include <stdint.h>

#include "sf_internal.h"

namespace sf {

constexpr int kBlock = kPointBlock;
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

// Division by a depth or a layer thickness (the momentum predictors, the vertical velocity
// integral): IEEE division in FP64 (the reference's arithmetic); in FP32 the hardware
// reciprocal form __fdividef (2 ulp for divisors in [2^-126, 2^126]; depths and thicknesses
// here are centimetres to kilometres), a few instructions instead of the IEEE sequence, well
// inside the FP32 form's stated per-field tolerances.
template <typename R>
__device__ __forceinline__ R ddiv(R a, R b) { return a / b; }
template <>
__device__ __forceinline__ float ddiv<float>(float a, float b) { return __fdividef(a, b); }

// ------------------------------------------------------------------------------------------
// 2D barotropic kernels
// ------------------------------------------------------------------------------------------

// computeZetaRHS (mod_cppkernels.cpp:81-128), optionally fused with the leapfrog of
// computeZetaPred (:134-150, mode 2) or with the corrector's fast-time averages (mode 1).
template <typename R>
__device__ __forceinline__ void zeta_rhs_body(
    const Geo<R> &g, const R *__restrict__ zeta, const R *__restrict__ ubar, const R *__restrict__ vbar,
    R *__restrict__ rzeta, int mode, double cff1, double *__restrict__ Zt,
    double *__restrict__ DU, double *__restrict__ DV, const R *__restrict__ zeta_t0,
    R *__restrict__ zeta_t2, R Dt, const long p) {
    if (p >= g.s2) return;
    const long I = g.I;
    const int j = fdiv((int)p, g.dI), i = (int)p - j * g.I;
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
__device__ __forceinline__ void momentum_body(
    const Geo<R> &g, R *__restrict__ rhs_u, R *__restrict__ rhs_v, const R *__restrict__ za,
    const R *__restrict__ zb, R grav, R w1, R w, int do_rhs, int do_pred, R Dt,
    const R *__restrict__ u_t1, R *__restrict__ u_t2, const R *__restrict__ v_t1,
    R *__restrict__ v_t2, const R *__restrict__ z1, const R *__restrict__ z2, const long p) {
    if (p >= g.s2) return;
    const long I = g.I, J = g.J;
    const int j = fdiv((int)p, g.dI), i = (int)p - j * g.I;
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
    if (do_pred && (int)p - fdiv((int)p, g.dJ) * g.J != 0 && p >= J) {   // p % J != 0
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
        u_t2[p] = ddiv(u_t1[p] * D1U + ((Dt * ru) * g.pm[p]) * g.pn[p], D2U);
        v_t2[p] = ddiv(v_t1[p] * D1V + ((Dt * rv) * g.pm[p]) * g.pn[p], D2V);
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
__device__ __forceinline__ void corr_point_body(
    const Geo<R> &g, R Dt, R *__restrict__ zeta_t2, const R *__restrict__ rz0, const R *__restrict__ rz1,
    const R *__restrict__ rz2, R *__restrict__ ubar_t1, const R *__restrict__ vbar_t1,
    const R *__restrict__ rub0, const R *__restrict__ rub1, R *__restrict__ vbar_t2, const long p) {
    if (p >= g.s2) return;
    const R A2 = R(5.0 / 12.0), A1 = R(8.0 / 12.0), A0 = R(-1.0 / 12.0);
    const R vb = vbar_t1 ? vbar_t1[p] : R(0);   // null: vbar_t1 is all zeros (see corr_point4)
    zeta_t2[p] = zeta_t2[p] + Dt * ((A2 * rz2[p] + A1 * rz1[p]) + A0 * rz0[p]);
    ubar_t1[p] = ubar_t1[p] + Dt * ((A2 * rub1[p] + A1 * rub0[p]) + A0 * vb);
    if (vbar_t2) vbar_t2[p] = R(0);
}

// ------------------------------------------------------------------------------------------
// Four-point forms of the 2D kernels (single grids): thread t owns the flat points
// p0 = 4t .. 4t+3 and loads each array's four values with 16-byte vector loads where the
// address allows it (checked at run time; the check is uniform across a warp), the
// neighbours p0-1 and p0+4 with scalar loads.  Each point's arithmetic is the scalar body's,
// operation for operation.  Threads whose stencil would reach outside the arrays (the first
// and last rows) run the scalar body on their four points.
// ------------------------------------------------------------------------------------------
template <typename R>
__device__ __forceinline__ void ld4(const R *__restrict__ a, long p, R (&o)[4]) {
    const R *q = a + p;
    const uintptr_t ad = reinterpret_cast<uintptr_t>(q);
    if constexpr (sizeof(R) == 4) {
        if ((ad & 15) == 0) {
            const float4 t = *reinterpret_cast<const float4 *>(q);
            o[0] = t.x; o[1] = t.y; o[2] = t.z; o[3] = t.w;
            return;
        }
        if ((ad & 7) == 0) {
            const float2 t0 = reinterpret_cast<const float2 *>(q)[0];
            const float2 t1 = reinterpret_cast<const float2 *>(q)[1];
            o[0] = t0.x; o[1] = t0.y; o[2] = t1.x; o[3] = t1.y;
            return;
        }
    } else {
        if ((ad & 15) == 0) {
            const double2 t0 = reinterpret_cast<const double2 *>(q)[0];
            const double2 t1 = reinterpret_cast<const double2 *>(q)[1];
            o[0] = t0.x; o[1] = t0.y; o[2] = t1.x; o[3] = t1.y;
            return;
        }
    }
#pragma unroll
    for (int u = 0; u < 4; ++u) o[u] = q[u];
}

// Stores the lanes u with (mask >> u) & 1; one vector store when all four are set and aligned.
template <typename R>
__device__ __forceinline__ void st4(R *__restrict__ a, long p, const R (&v)[4], unsigned mask) {
    R *q = a + p;
    const uintptr_t ad = reinterpret_cast<uintptr_t>(q);
    if (mask == 15u) {
        if constexpr (sizeof(R) == 4) {
            if ((ad & 15) == 0) {
                *reinterpret_cast<float4 *>(q) = make_float4(v[0], v[1], v[2], v[3]);
                return;
            }
        } else {
            if ((ad & 15) == 0) {
                reinterpret_cast<double2 *>(q)[0] = make_double2(v[0], v[1]);
                reinterpret_cast<double2 *>(q)[1] = make_double2(v[2], v[3]);
                return;
            }
        }
    }
#pragma unroll
    for (int u = 0; u < 4; ++u)
        if ((mask >> u) & 1u) q[u] = v[u];
}

// (i, j) of the four points from those of the first: one wrap to the next row at most (I >= 5).
__device__ __forceinline__ void ij4(int i0, int j0, int I, int (&i)[4], int (&j)[4]) {
#pragma unroll
    for (int u = 0; u < 4; ++u) {
        const int a = i0 + u;
        const bool w = a >= I;
        i[u] = w ? a - I : a;
        j[u] = w ? j0 + 1 : j0;
    }
}

template <typename R>
__device__ __forceinline__ void zeta_rhs4(
    const Geo<R> &g, const R *__restrict__ zeta, const R *__restrict__ ubar,
    const R *__restrict__ vbar, R *__restrict__ rzeta, int mode, double cff1,
    double *__restrict__ Zt, double *__restrict__ DU, double *__restrict__ DV,
    const R *__restrict__ zeta_t0, R *__restrict__ zeta_t2, R Dt, const long p0) {
    const long I = g.I, s2 = g.s2;
    if (p0 >= s2) return;
    if (p0 < I || p0 + 3 + I >= s2) {
        for (int u = 0; u < 4; ++u)
            zeta_rhs_body(g, zeta, ubar, vbar, rzeta, mode, cff1, Zt, DU, DV, zeta_t0, zeta_t2,
                          Dt, p0 + u);
        return;
    }
    const int j0 = fdiv((int)p0, g.dI), i0 = (int)p0 - j0 * g.I;
    int ii[4], jj[4];
    ij4(i0, j0, g.I, ii, jj);
    unsigned inm = 0;
#pragma unroll
    for (int u = 0; u < 4; ++u) inm |= (rint_(ii[u], jj[u], g.I, g.J) ? 1u : 0u) << u;
    R rz[4] = {R(0), R(0), R(0), R(0)};
    double DUp_[4], DVp_[4];
    if (inm) {
        const R *h = g.h;
        R z[4], zs[4], zn[4], hh[4], hs[4], hn[4], ub[4], vb[4], vn[4], ou[4], ov[4], ovn[4],
            pm[4], pn[4];
        ld4(zeta, p0, z);
        ld4(zeta, p0 - I, zs);
        ld4(zeta, p0 + I, zn);
        ld4(h, p0, hh);
        ld4(h, p0 - I, hs);
        ld4(h, p0 + I, hn);
        ld4(ubar, p0, ub);
        ld4(vbar, p0, vb);
        ld4(vbar, p0 + I, vn);
        ld4(g.on_u, p0, ou);
        ld4(g.om_v, p0, ov);
        ld4(g.om_v, p0 + I, ovn);
        ld4(g.pm, p0, pm);
        ld4(g.pn, p0, pn);
        const R zw = zeta[p0 - 1], ze = zeta[p0 + 4], hw = h[p0 - 1], he = h[p0 + 4];
        const R ue = ubar[p0 + 4], oue = g.on_u[p0 + 4];
#pragma unroll
        for (int u = 0; u < 4; ++u) {
            const R Dp = z[u] + hh[u];
            const R Dw = u == 0 ? zw + hw : z[u - 1] + hh[u - 1];
            const R De = u == 3 ? ze + he : z[u + 1] + hh[u + 1];
            const R Ds = zs[u] + hs[u], Dn = zn[u] + hn[u];
            const R DUp = ub[u] * ((Dp + Dw) * R(0.5));
            const R DUe = (u == 3 ? ue : ub[u + 1]) * ((De + Dp) * R(0.5));
            const R DVp = vb[u] * ((Dp + Ds) * R(0.5));
            const R DVn = vn[u] * ((Dn + Dp) * R(0.5));
            const R oe = u == 3 ? oue : ou[u + 1];
            rz[u] = (((DUe * oe - DUp * ou[u]) + (DVn * ovn[u] - DVp * ov[u])) * pm[u]) * pn[u];
            DUp_[u] = (cff1 * (double)DUp) * (double)ou[u];
            DVp_[u] = (cff1 * (double)DVp) * (double)ov[u];
        }
        st4(rzeta, p0, rz, inm);
        if (mode == 1) {
            double zt[4], du[4], dv[4];
            ld4(Zt, p0, zt);
            ld4(DU, p0, du);
            ld4(DV, p0, dv);
#pragma unroll
            for (int u = 0; u < 4; ++u) {
                zt[u] = zt[u] + cff1 * (double)z[u];
                du[u] = du[u] + DUp_[u];
                dv[u] = dv[u] + DVp_[u];
            }
            st4(Zt, p0, zt, inm);
            st4(DU, p0, du, inm);
            st4(DV, p0, dv, inm);
        }
    }
    if (mode == 2) {
        unsigned wm = 0;
#pragma unroll
        for (int u = 0; u < 4; ++u) wm |= (ii[u] != 0 && jj[u] != 0 ? 1u : 0u) << u;
        R z0[4], out[4];
        ld4(zeta_t0, p0, z0);
#pragma unroll
        for (int u = 0; u < 4; ++u) {
            const R r = ((inm >> u) & 1u) ? rz[u] : (((wm >> u) & 1u) ? rzeta[p0 + u] : R(0));
            out[u] = z0[u] + Dt * r;
        }
        st4(zeta_t2, p0, out, wm);
    }
}

template <typename R>
__device__ __forceinline__ void momentum4(
    const Geo<R> &g, R *__restrict__ rhs_u, R *__restrict__ rhs_v, const R *__restrict__ za,
    const R *__restrict__ zb, R grav, R w1, R w, int do_rhs, int do_pred, R Dt,
    const R *__restrict__ u_t1, R *__restrict__ u_t2, const R *__restrict__ v_t1,
    R *__restrict__ v_t2, const R *__restrict__ z1, const R *__restrict__ z2, const long p0) {
    const long I = g.I, J = g.J, s2 = g.s2;
    if (p0 >= s2) return;
    if (p0 < I + 1 || p0 + 3 >= s2) {
        for (int u = 0; u < 4; ++u)
            momentum_body(g, rhs_u, rhs_v, za, zb, grav, w1, w, do_rhs, do_pred, Dt, u_t1, u_t2,
                          v_t1, v_t2, z1, z2, p0 + u);
        return;
    }
    const R *h = g.h;
    const int j0 = fdiv((int)p0, g.dI), i0 = (int)p0 - j0 * g.I;
    int ii[4], jj[4];
    ij4(i0, j0, g.I, ii, jj);
    unsigned inm = 0, pdm = 0;
#pragma unroll
    for (int u = 0; u < 4; ++u) {
        const int q = (int)p0 + u;
        inm |= (do_rhs && rint_(ii[u], jj[u], g.I, g.J) ? 1u : 0u) << u;
        pdm |= (do_pred && q - fdiv(q, g.dJ) * g.J != 0 && q >= J ? 1u : 0u) << u;
    }
    R hh[4], hs[4];
    ld4(h, p0, hh);
    ld4(h, p0 - I, hs);
    const R hw = h[p0 - 1];
    R ru[4] = {R(0), R(0), R(0), R(0)}, rv[4] = {R(0), R(0), R(0), R(0)};
    if (inm) {
        R a[4], as[4], b[4], bs[4], ou[4], ov[4];
        ld4(za, p0, a);
        ld4(za, p0 - I, as);
        ld4(zb, p0, b);
        ld4(zb, p0 - I, bs);
        ld4(g.on_u, p0, ou);
        ld4(g.om_v, p0, ov);
        const R aw = za[p0 - 1], bw = zb[p0 - 1];
#pragma unroll
        for (int u = 0; u < 4; ++u) {
            const R gp = w1 * a[u] + w * b[u];
            const R gw = u == 0 ? w1 * aw + w * bw : w1 * a[u - 1] + w * b[u - 1];
            const R gs = w1 * as[u] + w * bs[u];
            const R hwu = u == 0 ? hw : hh[u - 1];
            ru[u] = (grav * ou[u]) * (((hh[u] + hwu) * R(0.5)) * (gp - gw) + R(0.5) * (gp * gp - gw * gw));
            rv[u] = (grav * ov[u]) * (((hh[u] + hs[u]) * R(0.5)) * (gp - gs) + R(0.5) * (gp * gp - gs * gs));
        }
        st4(rhs_u, p0, ru, inm);
        st4(rhs_v, p0, rv, inm);
    }
    if (pdm) {
        R c1[4], c1s[4], c2[4], c2s[4], ut[4], vt[4], pm[4], pn[4], uo[4], vo[4];
        ld4(z1, p0, c1);
        ld4(z1, p0 - I, c1s);
        ld4(z2, p0, c2);
        ld4(z2, p0 - I, c2s);
        ld4(u_t1, p0, ut);
        ld4(v_t1, p0, vt);
        ld4(g.pm, p0, pm);
        ld4(g.pn, p0, pn);
        const R c1w = z1[p0 - 1], c2w = z2[p0 - 1];
#pragma unroll
        for (int u = 0; u < 4; ++u) {
            R fu = ru[u], fv = rv[u];
            if (((pdm >> u) & 1u) && !((inm >> u) & 1u)) {
                fu = rhs_u[p0 + u];
                fv = rhs_v[p0 + u];
            }
            const R hwu = u == 0 ? hw : hh[u - 1];
            const R D1p = c1[u] + hh[u], D2p = c2[u] + hh[u];
            const R D1U = (D1p + ((u == 0 ? c1w : c1[u - 1]) + hwu)) * R(0.5);
            const R D2U = (D2p + ((u == 0 ? c2w : c2[u - 1]) + hwu)) * R(0.5);
            const R D1V = (D1p + (c1s[u] + hs[u])) * R(0.5);
            const R D2V = (D2p + (c2s[u] + hs[u])) * R(0.5);
            uo[u] = ddiv(ut[u] * D1U + ((Dt * fu) * pm[u]) * pn[u], D2U);
            vo[u] = ddiv(vt[u] * D1V + ((Dt * fv) * pm[u]) * pn[u], D2V);
        }
        st4(u_t2, p0, uo, pdm);
        st4(v_t2, p0, vo, pdm);
    }
}

template <typename R>
__device__ __forceinline__ void corr_point4(
    const Geo<R> &g, R Dt, R *__restrict__ zeta_t2, const R *__restrict__ rz0,
    const R *__restrict__ rz1, const R *__restrict__ rz2, R *__restrict__ ubar_t1,
    const R *__restrict__ vbar_t1, const R *__restrict__ rub0, const R *__restrict__ rub1,
    R *__restrict__ vbar_t2, const long p0) {
    if (p0 >= g.s2) return;
    if (p0 + 3 >= g.s2) {
        for (int u = 0; u < 4; ++u)
            corr_point_body(g, Dt, zeta_t2, rz0, rz1, rz2, ubar_t1, vbar_t1, rub0, rub1, vbar_t2,
                            p0 + u);
        return;
    }
    const R A2 = R(5.0 / 12.0), A1 = R(8.0 / 12.0), A0 = R(-1.0 / 12.0);
    R z[4], r0[4], r1[4], r2[4], ub[4], vb[4], b0[4], b1[4];
    ld4(zeta_t2, p0, z);
    ld4(rz0, p0, r0);
    ld4(rz1, p0, r1);
    ld4(rz2, p0, r2);
    ld4(ubar_t1, p0, ub);
    // vbar_t1 null: it is all +0 (the loop's substeps after the first, whose previous corrector
    // zeroed it, main3d.py:189), the same operand without the load
    if (vbar_t1) {
        ld4(vbar_t1, p0, vb);
    } else {
#pragma unroll
        for (int u = 0; u < 4; ++u) vb[u] = R(0);
    }
    ld4(rub0, p0, b0);
    ld4(rub1, p0, b1);
#pragma unroll
    for (int u = 0; u < 4; ++u) {
        z[u] = z[u] + Dt * ((A2 * r2[u] + A1 * r1[u]) + A0 * r0[u]);
        ub[u] = ub[u] + Dt * ((A2 * b1[u] + A1 * b0[u]) + A0 * vb[u]);
    }
    st4(zeta_t2, p0, z, 15u);
    st4(ubar_t1, p0, ub, 15u);
    if (vbar_t2) {
        const R zero[4] = {R(0), R(0), R(0), R(0)};
        st4(vbar_t2, p0, zero, 15u);
    }
}

// Boundary programs (see BcProgram): independent entries one per thread over as many blocks
// as needed; each group of chained entries by one warp, all reads before all writes.
template <typename R>
__device__ __forceinline__ R bc_value(const R *f, int s, R val) {
    return s >= 0 ? f[s] : (s == -1 ? R(0) : val);
}

template <typename R>
__global__ void __launch_bounds__(256) k_bc_apply(BcProgram p1, R *f1, BcProgram p2, R *f2, R val0,
                                                  const double *valp) {
    asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
    // The programs' index lists are the context's, uploaded synchronously at set-up: they are
    // read before waiting for the preceding kernel, whose outputs (the field values, and the
    // clamped value that a kernel writes before a graph replay) are read only after the wait.
    const long t = tid_flat();
    int dst = -1, src = 0;
    R *fi = f1;
    if (t < p1.n) {
        dst = p1.dst[t];
        src = p1.src[t];
    } else if (t < (long)p1.n + p2.n) {
        const long k = t - p1.n;
        dst = p2.dst[k];
        src = p2.src[k];
        fi = f2;
    }
    // chained entries: group g (one per member, at most 32 entries) by warp g of the grid, one
    // entry per lane; every lane reads, the warp synchronises, then every lane writes, so all
    // reads come before all writes.  (Independent entries neither read nor write a node of a
    // chained group, so the two parts need no ordering.)
    const long w = t >> 5;
    const bool grp = w < (long)p1.ngr + p2.ngr;   // uniform across the warp
    const bool first = w < p1.ngr;
    R *fc = first ? f1 : f2;
    int dc = -1, sc = 0;
    if (grp) {
        const BcProgram &pp = first ? p1 : p2;
        const int g = (int)(first ? w : w - p1.ngr), lane = (int)(t & 31);
        const int a = pp.gofs[g], b = pp.gofs[g + 1];
        if (lane < b - a) {
            dc = pp.dst_ch[a + lane];
            sc = pp.src_ch[a + lane];
        }
    }
    asm volatile("griddepcontrol.wait;" ::: "memory");
    const R val = valp ? (R)valp[0] : val0;   // time-dependent value from the device (graphs)
    if (dst >= 0) fi[dst] = bc_value(fi, src, val);
    if (grp) {
        const R x = dc >= 0 ? bc_value(fc, sc, val) : R(0);
        __syncwarp();
        if (dc >= 0) fc[dc] = x;
    }
}

// ------------------------------------------------------------------------------------------
// 3D right-hand side (nonlinear/rhs.py:16-93): ru = rv = 0, addCoriolis (rhs_kernels.cpp:7-35),
// horizontalAdvection (:71-132), verticalAdvection (:136-196), one thread per column.
// ------------------------------------------------------------------------------------------

// Tiled form: a block owns a TX x TY tile of rho points and marches over the levels; at each
// level the tile of u, v, Huon, Hvom, Hz (level K) and W (level K+1) is staged in shared memory
// with a halo of rows j-3..j+2 and columns i-2..i+2.  The halo is addressed by flat index
// (j0+r)*I + (i0+c), so columns beyond the row ends wrap into the neighbouring rows exactly as
// the reference's flat-index stencils do; reads before the array start or past its end stage 0.
// Tile shapes (TX x TY): 32 x 8 (the default), 32 x 4, 64 x 4 and 32 x 16, chosen per context
// (sf_ctx_set_tile, e.g. by the autotuner); the staged tile adds the halo.
constexpr int kTX = kTileX, kTY = kTileY;
constexpr int kHY0 = 3, kHY1 = 2, kHX0 = 2, kHX1 = 2;          // halo extents
template <int TX, int TY>
struct RhsTile {
    static constexpr int SX = TX + kHX0 + kHX1, SY = TY + kHY0 + kHY1, SN = SX * SY;
    static constexpr int FX = TX + 1, FN = (TX + 1) * (TY + 1);   // face-flux tile
};
// Dynamic shared memory of the tiled right-hand side: rhs_bufs<R>() staging buffers of 6
// fields and the four face-flux arrays.  FP32 keeps three buffers: level K+2 is issued after
// the first barrier of level K, when every thread has finished level K-1 (its reads of the
// buffer being refilled and of the face fluxes), so a level needs two barriers.  FP64, whose
// buffers are twice the size, keeps two (three blocks per SM) and a third barrier per level.
template <typename R>
__host__ __device__ constexpr int rhs_bufs() { return sizeof(R) == 4 ? 3 : 2; }
template <typename R, int TX, int TY>
constexpr size_t rhs_smem_bytes() {
    return sizeof(R) * ((size_t)rhs_bufs<R>() * 6 * RhsTile<TX, TY>::SN +
                        4 * (size_t)RhsTile<TX, TY>::FN);
}

template <typename R, int SX>
struct Tile {
    const R *t;
    int base;   // index of the thread's own node in the staged tile
    __device__ __forceinline__ R operator()(int dr, int dc) const { return t[base + dr * SX + dc]; }
};

// Asynchronous staging (cp.async, completes in the background while the previous level is
// computed); out-of-range elements are zero-filled by a zero source size.
__device__ __forceinline__ void cp_async(float *dst, const float *src, bool ok) {
    const unsigned d = (unsigned)__cvta_generic_to_shared(dst);
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4, %2;\n" ::"r"(d), "l"(src), "r"(ok ? 4 : 0));
}
__device__ __forceinline__ void cp_async(double *dst, const double *src, bool ok) {
    const unsigned d = (unsigned)__cvta_generic_to_shared(dst);
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;\n" ::"r"(d), "l"(src), "r"(ok ? 8 : 0));
}
// 4-byte copy of n (4 or 0) source bytes to shared-window byte address saddr + OFF: 0
// zero-fills the destination without reading.
template <int OFF>
__device__ __forceinline__ void cp_async_at(uint32_t saddr, const float *src, int n) {
    asm volatile("cp.async.ca.shared.global [%0+%3], [%1], 4, %2;\n" ::"r"(saddr), "l"(src), "r"(n),
                 "n"(OFF));
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::); }
// 16 bytes global -> shared, L2 only (both addresses 16-byte aligned)
__device__ __forceinline__ void cp_async16(uint32_t saddr, const void *src) {
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(saddr), "l"(src));
}
template <int n>
__device__ __forceinline__ void cp_async_wait() { asm volatile("cp.async.wait_group %0;\n" ::"n"(n)); }

// The staged elements of a thread: e = tid + q*TX*TY, q < kPer; their flat offsets within a
// level are computed once per block (the division by the staged row length is not repeated
// for every level and field).
template <int TX, int TY>
struct StageMap {
    static constexpr int kPer = (RhsTile<TX, TY>::SN + TX * TY - 1) / (TX * TY);
    long rel[kPer];
    __device__ __forceinline__ StageMap(long I, long j0, long i0, int tid) {
        using T = RhsTile<TX, TY>;
#pragma unroll
        for (int q = 0; q < kPer; ++q) {
            const int e = tid + q * TX * TY;
            const int r = e / T::SX - kHY0, c = e % T::SX - kHX0;
            rel[q] = (j0 + r) * I + (i0 + c);
        }
    }
};

template <typename R, int TX, int TY>
__device__ __forceinline__ void stage(R *dst, const R *src, long lvl_off, long len,
                                      const StageMap<TX, TY> &sm, int tid) {
    using T = RhsTile<TX, TY>;
#pragma unroll
    for (int q = 0; q < StageMap<TX, TY>::kPer; ++q) {
        const int e = tid + q * TX * TY;
        if (e < T::SN) {
            const long f = lvl_off + sm.rel[q];
            const bool ok = f >= 0 && f < len;
            cp_async(dst + e, ok ? src + f : src, ok);
        }
    }
}

// Pair staging: when the row length I is even and every field starts on a 2-element boundary,
// the staged tile (SX even, first column i0 - 2 even) is a set of aligned element pairs, copied
// 8 (FP32) or 16 (FP64) bytes at a time: half the copies of element staging.  A level whose
// whole tile lies inside every field (all but the first and the last few rows of the array) is
// staged without per-copy bounds checks.  Offsets fit 32 bits (the host requires s2 < 2^30).
__device__ __forceinline__ void cp_async2(float *dst, const float *src) {
    const unsigned d = (unsigned)__cvta_generic_to_shared(dst);
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(d), "l"(src));
}
__device__ __forceinline__ void cp_async2(double *dst, const double *src) {
    const unsigned d = (unsigned)__cvta_generic_to_shared(dst);
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(d), "l"(src));
}
__device__ __forceinline__ void cp_async2(float *dst, const float *src, bool ok) {
    const unsigned d = (unsigned)__cvta_generic_to_shared(dst);
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;\n" ::"r"(d), "l"(src), "r"(ok ? 8 : 0));
}
__device__ __forceinline__ void cp_async2(double *dst, const double *src, bool ok) {
    const unsigned d = (unsigned)__cvta_generic_to_shared(dst);
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(d), "l"(src), "r"(ok ? 16 : 0));
}
template <int TX, int TY>
struct PairMap {
    using T = RhsTile<TX, TY>;
    static_assert(T::SX % 2 == 0 && kHX0 % 2 == 0, "pair staging needs even tile rows");
    static constexpr int kPairs = T::SN / 2;
    static constexpr int kPer = (kPairs + TX * TY - 1) / (TX * TY);
    int rel[kPer];   // flat offset (within a level) of each pair's first element
    int rmin, rmax;  // first and last flat offset of the staged tile
    __device__ __forceinline__ PairMap(int I, int j0, int i0, int tid) {
#pragma unroll
        for (int q = 0; q < kPer; ++q) {
            const int e = 2 * (tid + q * TX * TY);
            const int r = e / T::SX - kHY0, c = e % T::SX - kHX0;
            rel[q] = (j0 + r) * I + (i0 + c);
        }
        rmin = (j0 - kHY0) * I + (i0 - kHX0);
        rmax = (j0 + TY - 1 + kHY1) * I + (i0 + TX - 1 + kHX1);
    }
};
template <typename R, int TX, int TY>
__device__ __forceinline__ void stage2(R *dst, const R *src, long lvl_off, long len, bool safe,
                                       const PairMap<TX, TY> &pm, int tid) {
    using M = PairMap<TX, TY>;
#pragma unroll
    for (int q = 0; q < M::kPer; ++q) {
        const int e = tid + q * TX * TY;
        if (M::kPairs % (TX * TY) == 0 || e < M::kPairs) {
            if (safe) {
                cp_async2(dst + 2 * e, src + lvl_off + pm.rel[q]);
            } else {
                const long f = lvl_off + pm.rel[q];
                const bool ok = f >= 0 && f < len;   // len and f even: the pair is wholly in or out
                cp_async2(dst + 2 * e, ok ? src + f : src, ok);
            }
        }
    }
}

template <typename R, int TX, int TY, bool P2>
__device__ __forceinline__ void rhs3d_body(const Geo<R> &g, const R *__restrict__ u,
                                           const R *__restrict__ v, const R *__restrict__ Huon,
                                           const R *__restrict__ Hvom, const R *__restrict__ W,
                                           const R *__restrict__ Hz, R *__restrict__ ru,
                                           R *__restrict__ rv, const int bx, const int by) {
    using T = RhsTile<TX, TY>;
    constexpr int kSX = T::SX, kSN = T::SN, kFX = T::FX, kFN = T::FN;
    extern __shared__ __align__(16) unsigned char rhs_smem[];
    R(*sbuf)[6][kSN] = reinterpret_cast<R(*)[6][kSN]>(rhs_smem);
    constexpr int kBufs = rhs_bufs<R>();
    R *sF = reinterpret_cast<R *>(rhs_smem) + kBufs * 6 * kSN;   // [4][kFN] face fluxes
    const int tx = threadIdx.x, ty = threadIdx.y, tid = ty * TX + tx;
    const long I = g.I, s2 = g.s2;
    const int N = g.N;
    const long i0 = (long)bx * TX, j0 = (long)by * TY;
    const int i = (int)(i0 + tx), j = (int)(j0 + ty);
    const bool live = i < g.I && j < g.J;
    const long p = (long)j * I + i;
    const long len3 = (long)(N + 1) * s2, lenHz = (long)N * s2;
    const bool rn = live && rnode_(i, j);
    const bool va = live && g.bcfield[p] < 0 && inner_(i, j, g.I, g.J);   // rhs_kernels.cpp:144-149
    const R c9 = R(9.0 / 16.0), c1 = R(1.0 / 16.0), G = R(-0.5);
    const int b = (ty + kHY0) * kSX + (tx + kHX0);

    // Own-column values for the vertical advection (rhs_kernels.cpp:158-194).
#define COL(X, k) ((X)[(long)(k) * s2 + p])
#define U4C(a, b_, c, d) (c9 * ((b_) + (c)) - c1 * ((a) + (d)))
#define WU4G(k) (c9 * (W[(long)(k) * s2 + p] + W[(long)(k) * s2 + p + 1]) - \
                 c1 * (W[(long)(k) * s2 + p - 1] + W[(long)(k) * s2 + p + 2]))
#define WV4G(k) (c9 * (W[(long)(k) * s2 + p] + W[(long)(k) * s2 + p + I]) - \
                 c1 * (W[(long)(k) * s2 + p - I] + W[(long)(k) * s2 + p + 2 * I]))
    R uuu = R(0), uuu2 = R(0), fv1 = R(0), fv2 = R(0), fv3 = R(0), fu2 = R(0);
    R uw0 = R(0), uw1 = R(0), uw2 = R(0), uw3 = R(0), vw0 = R(0), vw1 = R(0), vw2 = R(0), vw3 = R(0);
    if (va) {
        uuu = (c9 * (COL(u, 0) + COL(u, 1)) - c1 * (0 + COL(u, 2))) * WU4G(1);
        uuu2 = (c9 * (0 + COL(u, 0)) - c1 * (0 + COL(u, 1))) * WU4G(0);
        fv1 = U4C(COL(v, 0), COL(v, 1), COL(v, 2), COL(v, 3)) * WV4G(1);
        fv2 = U4C(COL(v, 1), COL(v, 2), COL(v, 3), COL(v, 4)) * WV4G(2);
        fv3 = U4C(COL(v, 2), COL(v, 3), COL(v, 4), COL(v, 5)) * WV4G(3);
        fu2 = U4C(COL(u, 1), COL(u, 2), COL(u, 3), COL(u, 4)) * WU4G(2);
        uw0 = COL(u, 2); uw1 = COL(u, 3); uw2 = COL(u, 4); uw3 = COL(u, 5);   // u(K..K+3), K = 2
        vw0 = COL(v, 2); vw1 = COL(v, 3); vw2 = COL(v, 4); vw3 = COL(v, 5);
    }
    R fu_k = fu2, fv_k = fv2;
    R ruN3 = R(0), rvN3 = R(0), rv1 = R(0);
    const R fp = live ? g.fomn[p] : R(0);
    const R fw = (live && p >= 1) ? g.fomn[p - 1] : R(0);
    const R fs = (live && p >= I) ? g.fomn[p - I] : R(0);

    // the staging offsets of this thread, once per block
    const std::conditional_t<P2, PairMap<TX, TY>, StageMap<TX, TY>> pm(g.I, (int)j0, (int)i0, tid);
    auto issue = [&](int K, int buf) {   // level K into staging buffer buf (= K % kBufs)
        const long o = (long)K * s2;
        R(*bf)[kSN] = sbuf[buf];
        if constexpr (P2) {
            // W is staged from level K+1 and Hz has N levels: o + rmax < N s2 covers all six
            const bool safe = o + pm.rmin >= 0 && o + pm.rmax < lenHz;
            stage2<R, TX, TY>(bf[0], u, o, len3, safe, pm, tid);
            stage2<R, TX, TY>(bf[1], v, o, len3, safe, pm, tid);
            stage2<R, TX, TY>(bf[2], Huon, o, len3, safe, pm, tid);
            stage2<R, TX, TY>(bf[3], Hvom, o, len3, safe, pm, tid);
            stage2<R, TX, TY>(bf[4], Hz, o, lenHz, safe, pm, tid);
            stage2<R, TX, TY>(bf[5], W, o + s2, len3, safe, pm, tid);
        } else {
            stage<R, TX, TY>(bf[0], u, o, len3, pm, tid);
            stage<R, TX, TY>(bf[1], v, o, len3, pm, tid);
            stage<R, TX, TY>(bf[2], Huon, o, len3, pm, tid);
            stage<R, TX, TY>(bf[3], Hvom, o, len3, pm, tid);
            stage<R, TX, TY>(bf[4], Hz, o, lenHz, pm, tid);
            stage<R, TX, TY>(bf[5], W, o + s2, len3, pm, tid);
        }
        cp_async_commit();
    };
    issue(0, 0);
    if constexpr (kBufs == 3) {
        if (N > 1) issue(1, 1);
        else cp_async_commit();
    }
    // the level loop is unrolled over the staging buffers, so that each level's buffer (and
    // every shared-memory offset into it) is a constant
    for (int K0 = 0; K0 < N; K0 += kBufs) {
#pragma unroll
    for (int kb = 0; kb < kBufs; ++kb) {
        const int K = K0 + kb;
        if (K >= N) break;   // uniform over the block
        const long o = (long)K * s2;
        if constexpr (kBufs == 3) {
            cp_async_wait<1>();   // level K's group (level K+1's may still be in flight)
            __syncthreads();      // ... and every thread is done with level K-1
            if (K + 2 < N) issue(K + 2, (kb + 2) % kBufs);
            else cp_async_commit();
        } else {
            if (K + 1 < N) {
                issue(K + 1, (kb + 1) % kBufs);
                cp_async_wait<1>();
            } else {
                cp_async_wait<0>();
            }
            __syncthreads();
        }
        R(*bf)[kSN] = sbuf[kb];
        const Tile<R, kSX> U{bf[0], b}, V{bf[1], b}, HU{bf[2], b}, HV{bf[3], b}, HZ{bf[4], b}, WW{bf[5], b};
        // Every thread reaches both barriers of each level: the compute is predicated on
        // `live` rather than skipped with `continue` (an aligned barrier must not diverge).
        R aru = R(0), arv = R(0);
        if (live) {
        if (rn) {   // addCoriolis (rhs_kernels.cpp:7-35)
            const R cffp = HZ(0, 0) * fp, cffw = HZ(0, -1) * fw, cffs = HZ(-1, 0) * fs;
            const R UFp = cffp * ((V(0, 0) + V(1, 0)) * R(0.5));
            const R UFw = cffw * ((V(0, -1) + V(1, -1)) * R(0.5));
            const R VFp = cffp * ((U(0, 0) + U(0, 1)) * R(0.5));
            const R VFs = cffs * ((U(-1, 0) + U(-1, 1)) * R(0.5));
            aru = aru + (UFp + UFw) * R(0.5);
            arv = arv - (VFp + VFs) * R(0.5);
        }
        }   // (the live region closes before the flux barrier; it reopens below)
        // horizontalAdvection (rhs_kernels.cpp:93-130) in two phases.  Each cell's divergence
        // is "own face flux minus the west (south) neighbour's", and the neighbour's face flux
        // is the same expression evaluated at the neighbour: phase 1 evaluates every face flux
        // once (the tile's cells plus the west column and south row of halo cells) into shared
        // memory, phase 2 differences them, with the reference's operations in its order.
#define UR(r, c) ((U(r, c) + U(r, (c) + 1)) * R(0.5))
#define UP(r, c) ((U(r, c) + U(r, (c) - 1)) * R(0.5))
#define VR(r, c) ((V(r, c) + V((r) + 1, c)) * R(0.5))
#define VP(r, c) ((V(r, c) + V((r) - 1, c)) * R(0.5))
#define HUR(r, c) ((HU(r, c) + HU(r, (c) + 1)) * R(0.5))
#define HUP(r, c) ((HU(r, c) + HU(r, (c) - 1)) * R(0.5))
#define HVP(r, c) ((HV(r, c) + HV((r) - 1, c)) * R(0.5))
#define HVR(r, c) ((HV(r, c) + HV((r) + 1, c)) * R(0.5))
#define DXX(T, r, c) (((T)(r, (c) - 1) - R(2.0) * (T)(r, c)) + (T)(r, (c) + 1))
#define DEE(T, r, c) (((T)((r) - 1, c) - R(2.0) * (T)(r, c)) + (T)((r) + 1, c))
#define UXXR(r, c) ((UR(r, c) + UR(r, (c) + 1) >= R(0)) ? DXX(U, r, c) : DXX(U, r, (c) + 1))
#define UEEP(r, c) ((HVP(r, c) + HVP((r) - 1, c) >= R(0)) ? DEE(U, r, c) : DEE(U, (r) - 1, c))
#define HUXXR(r, c) ((DXX(HU, r, c) + DXX(HU, r, (c) + 1)) * R(0.5))
#define HUEEP(r, c) ((DEE(HU, r, c) + DEE(HU, r, (c) - 1)) * R(0.5))
#define HVXXP(r, c) ((DXX(HV, r, c) + DXX(HV, (r) - 1, c)) * R(0.5))
#define HVEER(r, c) ((DEE(HV, r, c) + DEE(HV, (r) + 1, c)) * R(0.5))
        // phase 1: face fluxes of cell (r, c), -1 <= r < TY, -1 <= c < TX.  Each thread takes
        // its own cell; warp row 0 also the south halo row and warp row 1 the west halo column
        // (the corner cell is nobody's neighbour).  A warp's lanes stay in one row, so its
        // shared loads are conflict-free (a lane mapping running across the 36-float staged rows
        // put lanes 4 columns apart in adjacent rows on one bank).
        auto face_flux = [&](int r, int c) {
            const int e = (r + 1) * kFX + (c + 1);
            const int bb = (r + kHY0) * kSX + (c + kHX0);
            const Tile<R, kSX> U{bf[0], bb}, V{bf[1], bb}, HU{bf[2], bb}, HV{bf[3], bb};
            // all four first, then the stores (a store between them would force the staged
            // values to be read again: the compiler cannot tell sF from the staged tile)
            const R uxx = UXXR(0, 0), uee = UEEP(0, 0);
            const R ufx = UR(0, 0) + (G * uxx) * (HUR(0, 0) + G * HUXXR(0, 0));
            const R ufe = UP(0, 0) + (G * uee) * (HVP(0, 0) + G * HVXXP(0, 0));
            const R vfx = VP(0, 0) + (G * uee) * (HUP(0, 0) + G * HUEEP(0, 0));
            const R vfe = VR(0, 0) + (G * uxx) * (HVR(0, 0) + G * HVEER(0, 0));
            sF[0 * kFN + e] = ufx;
            sF[1 * kFN + e] = ufe;
            sF[2 * kFN + e] = vfx;
            sF[3 * kFN + e] = vfe;
        };
        // two vertically adjacent cells per thread where the tile allows it: their loads are
        // evaluated together (the second cell's stencil is the first's one row up, so the
        // shared staged values are loaded once), then the eight stores
        auto face_flux_pair = [&](int r, int c) {
            const int e = (r + 1) * kFX + (c + 1);
            const int bb = (r + kHY0) * kSX + (c + kHX0);
            const Tile<R, kSX> U{bf[0], bb}, V{bf[1], bb}, HU{bf[2], bb}, HV{bf[3], bb};
            const R uxx = UXXR(0, 0), uee = UEEP(0, 0);
            const R ufx = UR(0, 0) + (G * uxx) * (HUR(0, 0) + G * HUXXR(0, 0));
            const R ufe = UP(0, 0) + (G * uee) * (HVP(0, 0) + G * HVXXP(0, 0));
            const R vfx = VP(0, 0) + (G * uee) * (HUP(0, 0) + G * HUEEP(0, 0));
            const R vfe = VR(0, 0) + (G * uxx) * (HVR(0, 0) + G * HVEER(0, 0));
            const R uxx1 = UXXR(1, 0), uee1 = UEEP(1, 0);
            const R ufx1 = UR(1, 0) + (G * uxx1) * (HUR(1, 0) + G * HUXXR(1, 0));
            const R ufe1 = UP(1, 0) + (G * uee1) * (HVP(1, 0) + G * HVXXP(1, 0));
            const R vfx1 = VP(1, 0) + (G * uee1) * (HUP(1, 0) + G * HUEEP(1, 0));
            const R vfe1 = VR(1, 0) + (G * uxx1) * (HVR(1, 0) + G * HVEER(1, 0));
            sF[0 * kFN + e] = ufx;
            sF[1 * kFN + e] = ufe;
            sF[2 * kFN + e] = vfx;
            sF[3 * kFN + e] = vfe;
            sF[0 * kFN + e + kFX] = ufx1;
            sF[1 * kFN + e + kFX] = ufe1;
            sF[2 * kFN + e + kFX] = vfx1;
            sF[3 * kFN + e + kFX] = vfe1;
        };
        if constexpr (TY % 2 == 0 && TY >= 4) {
            // warps 0 .. TY/2-1: rows 2 ty - 1 and 2 ty; warp TY/2: row TY-1; warp TY/2+1:
            // the west halo column (rows 0 .. TY-1; the corner cell is nobody's neighbour)
            if (ty < TY / 2) face_flux_pair(2 * ty - 1, tx);
            else if (ty == TY / 2) face_flux(TY - 1, tx);
            else if (ty == TY / 2 + 1 && tx < TY) face_flux(tx, -1);
        } else {
            face_flux(ty, tx);
            if (ty == 0) face_flux(-1, tx);
            else if (ty == 1 && tx < TY) face_flux(tx, -1);
        }
        __syncthreads();
        if (live) {
        {   // phase 2: this cell's divergence
            const int e0 = (ty + 1) * kFX + (tx + 1), ew = e0 - 1, es = e0 - kFX;
            const R ufx0 = sF[e0], ufxw = sF[ew];
            const R ufe0 = sF[kFN + e0], ufes = sF[kFN + es];
            const R vfx0 = sF[2 * kFN + e0], vfxw = sF[2 * kFN + ew];
            const R vfe0 = sF[3 * kFN + e0], vfes = sF[3 * kFN + es];
            aru = aru - ((ufx0 - ufxw) + (ufe0 - ufes));
            arv = arv - ((vfx0 - vfxw) + (vfe0 - vfes));
        }
#undef HVEER
#undef HVXXP
#undef HUEEP
#undef HUXXR
#undef UEEP
#undef UXXR
#undef DEE
#undef DXX
#undef HVR
#undef HVP
#undef HUP
#undef HUR
#undef VP
#undef VR
#undef UP
#undef UR
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
                arv -= c9 * (fv1 + fv2) - c1 * (fv1 + fv3);
                aru = aru - (fu2 - uuu);
            } else if (K <= N - 3) {
                const R u4 = K + 4 <= N ? COL(u, K + 4) : R(0), v4 = K + 4 <= N ? COL(v, K + 4) : R(0);
                const R wu = c9 * (WW(0, 0) + WW(0, 1)) - c1 * (WW(0, -1) + WW(0, 2));
                const R wv = c9 * (WW(0, 0) + WW(1, 0)) - c1 * (WW(-1, 0) + WW(2, 0));
                const R fu1 = U4C(uw0, uw1, uw2, uw3) * wu, fv1_ = U4C(vw0, vw1, vw2, vw3) * wv;
                aru = aru - (fu1 - fu_k);
                arv = arv - (fv1_ - fv_k);
                fu_k = fu1;
                fv_k = fv1_;
                uw0 = uw1; uw1 = uw2; uw2 = uw3; uw3 = u4;
                vw0 = vw1; vw1 = vw2; vw2 = vw3; vw3 = v4;
            } else {
                aru = ruN3;    // ru[N-2] = ru[N-3], ru[N-1] = ru[N-2] (:189-192)
                arv = rvN3;
            }
            if (K == N - 3) {
                ruN3 = aru;
                rvN3 = arv;
            }
            if (K == 1) rv1 = arv;
        }
        ru[o + p] = aru;
        rv[o + p] = (va && K == 0) ? R(0) : arv;   // rv[0] is set from rv[1] below
        }
        if constexpr (kBufs == 2) __syncthreads();   // the buffer of level K is refilled next
    }
    }
    if (!live) return;
    const long oN = (long)N * s2;
    ru[oN + p] = va ? ruN3 : R(0);   // ru_t2[:] = 0 (rhs.py:38); ru[N] = ru[N-2] (:193)
    rv[oN + p] = va ? rvN3 : R(0);
    if (va) rv[p] = rv1;             // rv[0] = rv[1] (:183)
#undef WV4G
#undef WU4G
#undef U4C
#undef COL
}

// ------------------------------------------------------------------------------------------
// rhs3d, marching form (single grids, N >= 6): the same operations as rhs3d_body, value for
// value, with each thread walking RW rows of one column.  A warp spans 32 columns, i0 - 1 ..
// i0 + 30: lane 0 evaluates the west halo column (its x-face fluxes and its Coriolis term
// reach lane 1 by a shuffle) and lanes 1..31 own the block's 31 output columns.  Walking up a
// column, a node's south y-face fluxes and its Coriolis "s" term are the previous row's own
// (the same expressions at the same node), its west x-face fluxes and Coriolis "w" term the
// west lane's; a warp evaluates the south y-faces of its first row once per level.  The
// stencil's shared loads repeat from row to row at constant offsets and are loaded once (the
// walk holds no shared store); a level takes one block barrier (the staging ring) instead of
// two.  The levels are staged as in rhs3d_body (STG 0: elements, 1: aligned pairs, columns
// xs .. xs+37 with xs = i0 - 3, rounded down to even for pairs), or (STG 2, FP32) as 16-byte
// chunks: each staged row's 36 columns i0-3 .. i0+32 are copied as the ten aligned chunks
// that hold them, the row placed at a shift of 0..3 elements in shared memory so that the
// chunks land aligned; a row pitch SX = I (mod 4) makes the shifts cancel, so element (r, c)
// sits at r SX + A + c for a constant A of the block.
// ------------------------------------------------------------------------------------------
constexpr int kMarchX = 31;   // output columns per block
template <int NW, int RW, int SX_>
struct MarchTile {
    static constexpr int TY = NW * RW;           // output rows per block
    static constexpr int SY = TY + kHY0 + kHY1;  // staged rows j0-3 .. j0+TY+1
    static constexpr int SX = SX_;               // row pitch of the staged tile
    static constexpr int SN = (SX * SY + 8 + 3) / 4 * 4;   // a field's staged level (16-byte multiple)
    static constexpr int NT = 32 * NW;           // threads per block
};
template <typename R>
__host__ __device__ constexpr int march_bufs() { return sizeof(R) == 4 ? 3 : 2; }
template <typename R, int NW, int RW, int SX>
constexpr size_t march_smem_bytes() {
    return sizeof(R) * (size_t)march_bufs<R>() * 6 * MarchTile<NW, RW, SX>::SN;
}
__device__ __forceinline__ int mod4(int x) { return x & 3; }   // two's complement: x mod 4 in 0..3
// a thread's staged units (chunks of 16 bytes, element pairs, or elements) with their flat
// offsets within a level and their shared-memory indices, and the block's extent of them
template <int NW, int RW, int STG, int SX>
struct MarchMap {
    using T = MarchTile<NW, RW, SX>;
    static constexpr int kRowChunks = 10;   // 40 elements hold any 36-column span
    static constexpr int kUnits = STG == 2 ? T::SY * kRowChunks : STG == 1 ? T::SX * T::SY / 2 : T::SX * T::SY;
    static constexpr int kPer = (kUnits + T::NT - 1) / T::NT;
    int rel[kPer], dst[kPer];
    int rmin, rmax;   // first and last flat offset staged
    int A;            // staged index of column xs in row 0
    __device__ __forceinline__ MarchMap(int I, int j0, int xs, int tid) {
        const int F0 = (j0 - kHY0) * I + xs;   // flat offset of (row 0, column xs)
        if constexpr (STG == 2) {
            A = 3 + mod4(F0 - 3);               // A = F0 (mod 4), 3 <= A <= 6
#pragma unroll
            for (int q = 0; q < kPer; ++q) {
                const int e = tid + q * T::NT, r = e / kRowChunks, k = e % kRowChunks;
                const int Fr = F0 + r * I, m = mod4(Fr);
                rel[q] = Fr - m + 4 * k;        // a 16-byte-aligned chunk of row r
                dst[q] = r * SX + A - m + 4 * k;   // = 0 (mod 4): SX = I, A = F0 (mod 4)
            }
            const int Fl = F0 + (T::SY - 1) * I;
            rmin = F0 - mod4(F0);
            rmax = Fl - mod4(Fl) + 4 * kRowChunks - 1;
        } else {
            A = 0;
#pragma unroll
            for (int q = 0; q < kPer; ++q) {
                const int e = (STG == 1 ? 2 : 1) * (tid + q * T::NT);
                rel[q] = (j0 - kHY0 + e / T::SX) * I + xs + e % T::SX;
                dst[q] = e;
            }
            rmin = F0;
            rmax = (j0 - kHY0 + T::SY - 1) * I + xs + T::SX - 1;
        }
    }
};
__device__ __forceinline__ void cp_async16z(uint32_t saddr, const void *src, bool ok) {
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(saddr), "l"(src),
                 "r"(ok ? 16 : 0));
}
template <typename R, int NW, int RW, int STG, int SX>
__device__ __forceinline__ void march_stage(R *dst, const R *src, long off, long len, bool safe,
                                            const MarchMap<NW, RW, STG, SX> &m, int tid) {
    using M = MarchMap<NW, RW, STG, SX>;
#pragma unroll
    for (int q = 0; q < M::kPer; ++q) {
        const int e = tid + q * MarchTile<NW, RW, SX>::NT;
        if (M::kUnits % MarchTile<NW, RW, SX>::NT == 0 || e < M::kUnits) {
            const long f = off + m.rel[q];
            if constexpr (STG == 2) {
                // f and len are multiples of 4: a chunk is wholly in or out of the array
                const uint32_t d = (uint32_t)__cvta_generic_to_shared(dst + m.dst[q]);
                if (safe) {
                    cp_async16(d, src + f);
                } else {
                    const bool ok = f >= 0 && f < len;
                    cp_async16z(d, ok ? src + f : src, ok);
                }
            } else if constexpr (STG == 1) {
                if (safe) {
                    cp_async2(dst + m.dst[q], src + f);
                } else {
                    const bool ok = f >= 0 && f < len;   // f and len even: the pair is in or out
                    cp_async2(dst + m.dst[q], ok ? src + f : src, ok);
                }
            } else {
                const bool ok = f >= 0 && f < len;
                cp_async(dst + m.dst[q], ok ? src + f : src, ok);
            }
        }
    }
}

template <typename R, int NW, int RW, int STG, int SX_, bool SPLIT>
__device__ __forceinline__ void rhs3d_march_body(const Geo<R> &g, const R *__restrict__ u,
                                                 const R *__restrict__ v, const R *__restrict__ Huon,
                                                 const R *__restrict__ Hvom, const R *__restrict__ W,
                                                 const R *__restrict__ Hz, R *__restrict__ ru,
                                                 R *__restrict__ rv, const int bx, const int by) {
    using T = MarchTile<NW, RW, SX_>;
    constexpr int SX = T::SX, SN = T::SN, TY = T::TY;
    constexpr int kBufs = march_bufs<R>();
    constexpr unsigned kAll = 0xffffffffu;
    extern __shared__ __align__(16) unsigned char rhs_smem[];
    R(*sbuf)[6][SN] = reinterpret_cast<R(*)[6][SN]>(rhs_smem);
    const int lane = threadIdx.x, w = threadIdx.y, tid = w * 32 + lane;
    const int I = g.I, J = g.J, N = g.N;
    const long s2 = g.s2;
    const long len3 = (long)(N + 1) * s2, lenHz = (long)N * s2;
    const int i0 = bx * kMarchX, j0 = by * TY;
    const int col = i0 - 1 + lane;                             // lane 0: the west halo column
    const int xs = STG == 1 ? ((i0 - 3) & ~1) : (i0 - 3);      // first staged column
    const int r0 = w * RW;                                     // the warp's first row in the tile
    const MarchMap<NW, RW, STG, SX> mm(I, j0, xs, tid);
    const int b0 = (r0 + kHY0) * SX + mm.A + (col - xs);       // staged index of (r0, col)
    const R c9 = R(9.0 / 16.0), c1 = R(1.0 / 16.0), G = R(-0.5);

    // Per node: output (lanes 1..31 inside the grid), Coriolis (rnode), vertical advection
    // (rhs_kernels.cpp:144-149) as bit masks; f at the node (lane 0: at its column, the west
    // term of lane 1's node); the flat index within a level.
    unsigned outm = 0, rnm = 0, vam = 0;
    R fp[RW];
    int pf[RW];
#pragma unroll
    for (int rr = 0; rr < RW; ++rr) {
        const int j = j0 + r0 + rr, p = j * I + col;
        pf[rr] = p;
        const bool live = lane >= 1 && col < I && j < J;
        if (live) {
            outm |= 1u << rr;
            if (rnode_(col, j)) rnm |= 1u << rr;
            if (g.bcfield[p] < 0 && inner_(col, j, I, J)) vam |= 1u << rr;
        }
        fp[rr] = lane >= 1 ? (live ? g.fomn[p] : R(0)) : ((j < J && p >= 0) ? g.fomn[p] : R(0));
    }
    // f of the row below the warp's first row (the Coriolis "s" term of that row's nodes)
    const R fpw = ((outm & 1u) && pf[0] >= I) ? g.fomn[pf[0] - I] : R(0);
    // vertical advection carried from level to level: the flux through the level's lower face
    // and u, v at the next three levels of the node's column
    R fuk[RW], fvk[RW], uw1[RW], uw2[RW], uw3[RW], vw1[RW], vw2[RW], vw3[RW];
#pragma unroll
    for (int rr = 0; rr < RW; ++rr) {
        fuk[rr] = fvk[rr] = uw1[rr] = uw2[rr] = uw3[rr] = vw1[rr] = vw2[rr] = vw3[rr] = R(0);
    }

    auto issue = [&](int K, int buf) {
        const long o = (long)K * s2;
        R(*bf)[SN] = sbuf[buf];
        // W is staged from level K+1 and Hz has N levels: o + rmax < N s2 covers all six
        const bool safe = o + mm.rmin >= 0 && o + mm.rmax < lenHz;
        march_stage<R, NW, RW, STG, SX>(bf[0], u, o, len3, safe, mm, tid);
        march_stage<R, NW, RW, STG, SX>(bf[1], v, o, len3, safe, mm, tid);
        march_stage<R, NW, RW, STG, SX>(bf[2], Huon, o, len3, safe, mm, tid);
        march_stage<R, NW, RW, STG, SX>(bf[3], Hvom, o, len3, safe, mm, tid);
        march_stage<R, NW, RW, STG, SX>(bf[4], Hz, o, lenHz, safe, mm, tid);
        march_stage<R, NW, RW, STG, SX>(bf[5], W, o + s2, len3, safe, mm, tid);
        cp_async_commit();
    };

#define COL(X, k) ((X)[(long)(k) * s2 + pp])
#define U4C(a, b_, c, d) (c9 * ((b_) + (c)) - c1 * ((a) + (d)))
#define WU4G(k) (c9 * (W[(long)(k) * s2 + pp] + W[(long)(k) * s2 + pp + 1]) - \
                 c1 * (W[(long)(k) * s2 + pp - 1] + W[(long)(k) * s2 + pp + 2]))
#define WV4G(k) (c9 * (W[(long)(k) * s2 + pp] + W[(long)(k) * s2 + pp + I]) - \
                 c1 * (W[(long)(k) * s2 + pp - I] + W[(long)(k) * s2 + pp + 2 * I]))
#define UR(r, c) ((U(r, c) + U(r, (c) + 1)) * R(0.5))
#define UP(r, c) ((U(r, c) + U(r, (c) - 1)) * R(0.5))
#define VR(r, c) ((V(r, c) + V((r) + 1, c)) * R(0.5))
#define VP(r, c) ((V(r, c) + V((r) - 1, c)) * R(0.5))
#define HUR(r, c) ((HU(r, c) + HU(r, (c) + 1)) * R(0.5))
#define HUP(r, c) ((HU(r, c) + HU(r, (c) - 1)) * R(0.5))
#define HVP(r, c) ((HV(r, c) + HV((r) - 1, c)) * R(0.5))
#define HVR(r, c) ((HV(r, c) + HV((r) + 1, c)) * R(0.5))
#define DXX(T, r, c) (((T)(r, (c) - 1) - R(2.0) * (T)(r, c)) + (T)(r, (c) + 1))
#define DEE(T, r, c) (((T)((r) - 1, c) - R(2.0) * (T)(r, c)) + (T)((r) + 1, c))
#define UXXR(r, c) ((UR(r, c) + UR(r, (c) + 1) >= R(0)) ? DXX(U, r, c) : DXX(U, r, (c) + 1))
#define UEEP(r, c) ((HVP(r, c) + HVP((r) - 1, c) >= R(0)) ? DEE(U, r, c) : DEE(U, (r) - 1, c))
#define HUXXR(r, c) ((DXX(HU, r, c) + DXX(HU, r, (c) + 1)) * R(0.5))
#define HUEEP(r, c) ((DEE(HU, r, c) + DEE(HU, r, (c) - 1)) * R(0.5))
#define HVXXP(r, c) ((DXX(HV, r, c) + DXX(HV, (r) - 1, c)) * R(0.5))
#define HVEER(r, c) ((DEE(HV, r, c) + DEE(HV, (r) + 1, c)) * R(0.5))

    issue(0, 0);
    if constexpr (kBufs == 3) {
        if (N > 1) issue(1, 1);
        else cp_async_commit();
    }
    for (int K0 = 0; K0 < N; K0 += kBufs) {
#pragma unroll
    for (int kb = 0; kb < kBufs; ++kb) {
        const int K = K0 + kb;
        if (K >= N) break;   // uniform over the block
        const long o = (long)K * s2;
        if constexpr (kBufs == 3) {
            cp_async_wait<1>();   // level K's group (level K+1's may still be in flight)
            __syncthreads();      // ... and every thread is done with level K-1
            if (K + 2 < N) issue(K + 2, (kb + 2) % kBufs);
            else cp_async_commit();
        } else {
            if (K + 1 < N) {
                issue(K + 1, (kb + 1) % kBufs);
                cp_async_wait<1>();
            } else {
                cp_async_wait<0>();
            }
            __syncthreads();
        }
        R(*bf)[SN] = sbuf[kb];
        const Tile<R, SX> U{bf[0], b0}, V{bf[1], b0}, HU{bf[2], b0}, HV{bf[3], b0}, HZ{bf[4], b0},
            WW{bf[5], b0};
        // the row below the warp's first row: its y-face fluxes and its Coriolis "p" term in v
        R ufe_s, vfe_s, VF_s;
        {
            const R uxx = UXXR(-1, 0), uee = UEEP(-1, 0);
            ufe_s = UP(-1, 0) + (G * uee) * (HVP(-1, 0) + G * HVXXP(-1, 0));
            vfe_s = VR(-1, 0) + (G * uxx) * (HVR(-1, 0) + G * HVEER(-1, 0));
            VF_s = (HZ(-1, 0) * fpw) * ((U(-1, 0) + U(-1, 1)) * R(0.5));
        }
        // Coriolis and horizontal advection of row rr (every level)
        auto horiz = [&](const int rr, R &aru, R &arv) {
            // addCoriolis (rhs_kernels.cpp:7-35): UFw is the west node's UFp, VFs the south
            // node's VFp
            const R cffp = HZ(rr, 0) * fp[rr];
            const R UFp = cffp * ((V(rr, 0) + V(rr + 1, 0)) * R(0.5));
            const R VFp = cffp * ((U(rr, 0) + U(rr, 1)) * R(0.5));
            const R UFw = __shfl_up_sync(kAll, UFp, 1);
            const bool rn = rnm >> rr & 1u;
            aru = rn ? R(0) + (UFp + UFw) * R(0.5) : R(0);
            arv = rn ? R(0) - (VFp + VF_s) * R(0.5) : R(0);
            VF_s = VFp;
            // horizontalAdvection (rhs_kernels.cpp:93-130): own face fluxes, the west node's
            // x-faces and the south node's y-faces
            const R uxx = UXXR(rr, 0), uee = UEEP(rr, 0);
            const R ufx = UR(rr, 0) + (G * uxx) * (HUR(rr, 0) + G * HUXXR(rr, 0));
            const R ufe = UP(rr, 0) + (G * uee) * (HVP(rr, 0) + G * HVXXP(rr, 0));
            const R vfx = VP(rr, 0) + (G * uee) * (HUP(rr, 0) + G * HUEEP(rr, 0));
            const R vfe = VR(rr, 0) + (G * uxx) * (HVR(rr, 0) + G * HVEER(rr, 0));
            const R ufxw = __shfl_up_sync(kAll, ufx, 1), vfxw = __shfl_up_sync(kAll, vfx, 1);
            aru = aru - ((ufx - ufxw) + (ufe - ufe_s));
            arv = arv - ((vfx - vfxw) + (vfe - vfe_s));
            ufe_s = ufe;
            vfe_s = vfe;
        };
        R aru_[RW], arv_[RW];
        if (SPLIT && K >= 2 && K <= N - 4) {
            // Levels 2 .. N-4: the vertical advection's interior form on every node, kept where
            // the node takes it; u, v four levels up loaded before the walk (one exposed load
            // latency per level); no special stores.  (The reference's out-of-range threads
            // reach levels 0 and 1 only: they number less than s2 + 512.)
            R u4[RW], v4[RW];
#pragma unroll
            for (int rr = 0; rr < RW; ++rr) {
                const long pp = pf[rr];
                const bool va = vam >> rr & 1u;
                u4[rr] = va ? COL(u, K + 4) : R(0);
                v4[rr] = va ? COL(v, K + 4) : R(0);
            }
#pragma unroll
            for (int rr = 0; rr < RW; ++rr) {
                R aru, arv;
                horiz(rr, aru, arv);
                const R wu = c9 * (WW(rr, 0) + WW(rr, 1)) - c1 * (WW(rr, -1) + WW(rr, 2));
                const R wv = c9 * (WW(rr, 0) + WW(rr + 1, 0)) - c1 * (WW(rr - 1, 0) + WW(rr + 2, 0));
                const R fu1 = U4C(U(rr, 0), uw1[rr], uw2[rr], uw3[rr]) * wu;
                const R fv1_ = U4C(V(rr, 0), vw1[rr], vw2[rr], vw3[rr]) * wv;
                const bool va = vam >> rr & 1u;
                aru_[rr] = va ? aru - (fu1 - fuk[rr]) : aru;
                arv_[rr] = va ? arv - (fv1_ - fvk[rr]) : arv;
                fuk[rr] = fu1;
                fvk[rr] = fv1_;
                uw1[rr] = uw2[rr]; uw2[rr] = uw3[rr]; uw3[rr] = u4[rr];
                vw1[rr] = vw2[rr]; vw2[rr] = vw3[rr]; vw3[rr] = v4[rr];
            }
            // stores after the walk, so that no store separates the walk's repeated shared loads
#pragma unroll
            for (int rr = 0; rr < RW; ++rr) {
                if (outm >> rr & 1u) {
                    ru[o + pf[rr]] = aru_[rr];
                    rv[o + pf[rr]] = arv_[rr];
                }
            }
        } else {
            // every level (the walk's general form; with SPLIT levels 0, 1 and N-3 .. N-1).  The
            // vertical advection's loads of u, v four levels up are issued before the walk.
            R u4[RW], v4[RW];
            const bool mid = K >= 2 && K <= N - 3 && K + 4 <= N;
#pragma unroll
            for (int rr = 0; rr < RW; ++rr) {
                const long pp = pf[rr];
                const bool ld = mid && (vam >> rr & 1u);
                u4[rr] = ld ? COL(u, K + 4) : R(0);
                v4[rr] = ld ? COL(v, K + 4) : R(0);
            }
#pragma unroll
            for (int rr = 0; rr < RW; ++rr) {
                R aru, arv;
                horiz(rr, aru, arv);
                // the reference's out-of-range threads store 0 into levels >= 1 (rhs_kernels.cpp:86-91)
                if (K >= 1 && o + pf[rr] < g.ref_threads) {
                    aru = R(0);
                    arv = R(0);
                }
                if (vam >> rr & 1u) {   // verticalAdvection (rhs_kernels.cpp:158-194)
                    const long pp = pf[rr];
                    if (K == 0) {
                        const R uuu = (c9 * (COL(u, 0) + COL(u, 1)) - c1 * (0 + COL(u, 2))) * WU4G(1);
                        const R uuu2 = (c9 * (0 + COL(u, 0)) - c1 * (0 + COL(u, 1))) * WU4G(0);
                        aru = aru - (uuu - uuu2);
                        fuk[rr] = uuu;
                    } else if (K == 1) {
                        const R fv1 = U4C(COL(v, 0), COL(v, 1), COL(v, 2), COL(v, 3)) * WV4G(1);
                        const R fv2 = U4C(COL(v, 1), COL(v, 2), COL(v, 3), COL(v, 4)) * WV4G(2);
                        const R fv3 = U4C(COL(v, 2), COL(v, 3), COL(v, 4), COL(v, 5)) * WV4G(3);
                        const R fu2 = U4C(COL(u, 1), COL(u, 2), COL(u, 3), COL(u, 4)) * WU4G(2);
                        arv -= c9 * (fv1 + fv2) - c1 * (fv1 + fv3);
                        aru = aru - (fu2 - fuk[rr]);
                        fuk[rr] = fu2;
                        fvk[rr] = fv2;
                        uw1[rr] = COL(u, 3); uw2[rr] = COL(u, 4); uw3[rr] = COL(u, 5);
                        vw1[rr] = COL(v, 3); vw2[rr] = COL(v, 4); vw3[rr] = COL(v, 5);
                    } else if (K <= N - 3) {
                        const R wu = c9 * (WW(rr, 0) + WW(rr, 1)) - c1 * (WW(rr, -1) + WW(rr, 2));
                        const R wv = c9 * (WW(rr, 0) + WW(rr + 1, 0)) - c1 * (WW(rr - 1, 0) + WW(rr + 2, 0));
                        const R fu1 = U4C(U(rr, 0), uw1[rr], uw2[rr], uw3[rr]) * wu;
                        const R fv1_ = U4C(V(rr, 0), vw1[rr], vw2[rr], vw3[rr]) * wv;
                        aru = aru - (fu1 - fuk[rr]);
                        arv = arv - (fv1_ - fvk[rr]);
                        fuk[rr] = fu1;
                        fvk[rr] = fv1_;
                        uw1[rr] = uw2[rr]; uw2[rr] = uw3[rr]; uw3[rr] = u4[rr];
                        vw1[rr] = vw2[rr]; vw2[rr] = vw3[rr]; vw3[rr] = v4[rr];
                    }   // levels N-2 and N-1 repeat level N-3 (:189-192), stored with it
                }
                aru_[rr] = aru;
                arv_[rr] = arv;
            }
#pragma unroll
            for (int rr = 0; rr < RW; ++rr) {
                if (!(outm >> rr & 1u)) continue;
                const long q = o + pf[rr];
                if (!(vam >> rr & 1u)) {
                    ru[q] = aru_[rr];
                    rv[q] = arv_[rr];
                    if (K == N - 1) {   // ru_t2[:] = 0 (rhs.py:38) at level N
                        ru[(long)N * s2 + pf[rr]] = R(0);
                        rv[(long)N * s2 + pf[rr]] = R(0);
                    }
                } else if (K <= N - 3) {
                    ru[q] = aru_[rr];
                    if (K >= 1) rv[q] = arv_[rr];
                    if (K == 1) rv[pf[rr]] = arv_[rr];   // rv[0] = rv[1] (:183)
                    if (K == N - 3) {   // ru[N-2] = ru[N-1] = ru[N-3], ru[N] = ru[N-2] (:189-193)
#pragma unroll
                        for (int k = 1; k <= 3; ++k) {
                            ru[q + k * s2] = aru_[rr];
                            rv[q + k * s2] = arv_[rr];
                        }
                    }
                }
            }
        }
        if constexpr (kBufs == 2) __syncthreads();   // the buffer of level K is refilled next
    }
    }
#undef HVEER
#undef HVXXP
#undef HUEEP
#undef HUXXR
#undef UEEP
#undef UXXR
#undef DEE
#undef DXX
#undef HVR
#undef HVP
#undef HUP
#undef HUR
#undef VP
#undef VR
#undef UP
#undef UR
#undef WV4G
#undef WU4G
#undef U4C
#undef COL
}

// ------------------------------------------------------------------------------------------
// set_maxflux (step3D_uv.kernels.cpp:372-405) + omega (:62-165) + set_zeta (:294-310)
// ------------------------------------------------------------------------------------------
// C > 0: levels whose loads the fused flux/omega kernel issues together on its interior
// columns (sf_ctx_tune knob SF_TUNE_MO_CHUNK); 0: one level at a time, the loop unrolled by 4;
// -1: omega alone (no fluxes), the fluxes' loads issued 16 levels at a time
template <typename R, int C = 0>
__device__ __forceinline__ void maxflux_omega_body(
    const Geo<R> &g, const R *__restrict__ u, const R *__restrict__ v, R *Huon, R *Hvom,
    const R *__restrict__ Hz, R *__restrict__ W, const R *__restrict__ z_w, int do_flux,
    int do_omega, R *__restrict__ zeta1, R *__restrict__ zeta2, const double *__restrict__ Zt,
    const long pl) {
    if (pl >= g.s2) return;
    const int pi = (int)pl;
    const long p = pi;
    const long I = g.I, s2 = g.s2;
    const int N = g.N;
    const int i = pi % g.I, j = pi / g.I;
    const bool un = unode_(i, j), vn = vnode_(i, j, g.J);
    const bool om = do_omega && g.bcfield[p] < 0;
    const bool fu = do_flux && un, fv = do_flux && vn;   // this thread writes Huon / Hvom
    const R onu = fu ? g.on_u[p] : R(0), omv = fv ? g.om_v[p] : R(0);
    if (!om) {   // fluxes only
        if (fu) {
#pragma unroll 4
            for (int K = 0; K < N; ++K) {
                const long o = (long)K * s2 + p;
                Huon[o] = (((Hz[o] + Hz[o - 1]) * R(0.5)) * u[o]) * onu;
            }
        }
        if (fv) {
#pragma unroll 4
            for (int K = 0; K < N; ++K) {
                const long o = (long)K * s2 + p;
                Hvom[o] = (((Hz[o] + Hz[o - I]) * R(0.5)) * v[o]) * omv;
            }
        }
    } else {
        // One pass over the levels: this column's fluxes (written where this kernel computes
        // them) and the running integral of the flux divergence.  Huon at p+1 and Hvom at p+I
        // are recomputed where this kernel also writes them (the value their owner thread
        // stores), read from memory elsewhere (nobody writes them here).  p+1 past the row end
        // is the next row's column 0 and p+I past the last row is row 0 of the next level;
        // neither is a U or V node.
        const bool rc = do_flux != 0;
        const bool ue = rc && i + 1 < g.I && unode_(i + 1, j);
        const bool vnn = rc && j + 1 < g.J && vnode_(i, j + 1, g.J);
        const R onu_e = ue ? g.on_u[p + 1] : R(0), omv_n = vnn ? g.om_v[p + I] : R(0);
        // the column's bed and depth for the correction, loaded before the integral
        const R zbed = z_w[p];
        const R h = z_w[(long)(N - 1) * s2 + p] - zbed;
        // the running integral in shared memory ([level][thread]), not in per-thread local
        // memory, whose footprint over all resident threads spills out of L1 and L2
        extern __shared__ __align__(16) unsigned char mo_smem[];
        R *Wcol = reinterpret_cast<R *>(mo_smem) + threadIdx.x;
#define Wc(K) Wcol[(K) * (int)blockDim.x]
        R Wk = R(0);
        Wc(0) = R(0);
        if (C < 0 && !rc) {
            // omega alone: the four fluxes of a chunk of kO levels loaded together (basin4:
            // 0.45 ms with 16, 0.48 with 8, 0.66 one level at a time)
            constexpr int kO = 16;
            for (int K0 = 1; K0 < N; K0 += kO) {
                R hu[kO], hv[kO], hE[kO], hN[kO];
#pragma unroll
                for (int c = 0; c < kO; ++c) {
                    const long o = (long)(K0 + c < N ? K0 + c : N - 1) * s2 + p;
                    hu[c] = Huon[o];
                    hv[c] = Hvom[o];
                    hE[c] = Huon[o + 1];
                    hN[c] = Hvom[o + I];
                }
#pragma unroll
                for (int c = 0; c < kO; ++c) {
                    if (K0 + c < N) {
                        Wk = Wk - ((hE[c] - hu[c]) + (hN[c] - hv[c]));
                        Wc(K0 + c) = Wk;
                    }
                }
            }
        } else if (C > 0 && fu && fv && ue && vnn) {
            // every flux this column needs is computed here: the loads of a chunk of levels
            // (Hz, u, v only, never the flux arrays being written) are issued together
            // before any of the chunk's arithmetic, the same expressions as below
            // 32-bit element offsets (the launcher takes this form only where (N+1) s2 < 2^31)
            const int s2i = (int)s2, Ii = (int)I;
            // two chunks per iteration: the second chunk's loads may issue before the first
            // chunk's arithmetic and stores
#pragma unroll 2
            for (int K0 = 0; K0 < N; K0 += (C > 0 ? C : 1)) {
                constexpr int CC = C > 0 ? C : 1;
                R hz[CC], hzw[CC], hzs[CC], hze[CC], hzn[CC], uu[CC], uE[CC], vv[CC], vN[CC];
#pragma unroll
                for (int c = 0; c < CC; ++c) {
                    const int o = (K0 + c < N ? K0 + c : N - 1) * s2i + pi;
                    hz[c] = Hz[o];
                    hzw[c] = Hz[o - 1];
                    hzs[c] = Hz[o - Ii];
                    hze[c] = Hz[o + 1];
                    hzn[c] = Hz[o + Ii];
                    uu[c] = u[o];
                    uE[c] = u[o + 1];
                    vv[c] = v[o];
                    vN[c] = v[o + Ii];
                }
#pragma unroll
                for (int c = 0; c < CC; ++c) {
                    const int K = K0 + c;
                    if (K < N) {
                        const int o = K * s2i + pi;
                        const R hup = (((hz[c] + hzw[c]) * R(0.5)) * uu[c]) * onu;
                        const R hvp = (((hz[c] + hzs[c]) * R(0.5)) * vv[c]) * omv;
                        Huon[o] = hup;
                        Hvom[o] = hvp;
                        if (K >= 1) {
                            const R hue = (((hze[c] + hz[c]) * R(0.5)) * uE[c]) * onu_e;
                            const R hvn = (((hzn[c] + hz[c]) * R(0.5)) * vN[c]) * omv_n;
                            Wk = Wk - ((hue - hup) + (hvn - hvp));
                            Wc(K) = Wk;
                        }
                    }
                }
            }
        } else {
#pragma unroll 4
        for (int K = 0; K < N; ++K) {
            const long o = (long)K * s2 + p;
            const R hzp = rc ? Hz[o] : R(0);   // Hz is given (and used) only with the fluxes
            const R hup = fu ? (((hzp + Hz[o - 1]) * R(0.5)) * u[o]) * onu : Huon[o];
            const R hvp = fv ? (((hzp + Hz[o - I]) * R(0.5)) * v[o]) * omv : Hvom[o];
            if (fu) Huon[o] = hup;
            if (fv) Hvom[o] = hvp;
            if (K >= 1) {
                const R hue = ue ? (((Hz[o + 1] + hzp) * R(0.5)) * u[o + 1]) * onu_e : Huon[o + 1];
                const R hvn = vnn ? (((Hz[o + I] + hzp) * R(0.5)) * v[o + I]) * omv_n : Hvom[o + I];
                Wk = Wk - ((hue - hup) + (hvn - hvp));
                Wc(K) = Wk;
            }
        }
        }
        const R Ws = Wk;
        W[p] = R(0);
        // the correction, z_w loaded kZ levels at a time (one exposed load latency per chunk):
        // 32 for omega alone, 16 after the fluxes (basin4: 0.45 and 0.82 ms; 32 after the
        // fluxes takes 1.14 ms)
        {
            constexpr int kZ = C < 0 ? 32 : 16;
            for (int K0 = 1; K0 < N; K0 += kZ) {
                R zw[kZ];
#pragma unroll
                for (int c = 0; c < kZ; ++c) {
                    const int K = K0 + c < N ? K0 + c : N - 1;
                    zw[c] = C > 0 ? z_w[K * (int)s2 + pi] : z_w[(long)K * s2 + p];
                }
#pragma unroll
                for (int c = 0; c < kZ; ++c) {
                    const int K = K0 + c;
                    if (K < N) {
                        const R wv = Wc(K) - ddiv(Ws * (zw[c] - zbed), h);
                        if (C > 0) W[K * (int)s2 + pi] = wv;
                        else W[(long)K * s2 + p] = wv;
                    }
                }
            }
        }
#undef Wc
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
__device__ __forceinline__ void set_depth_body(const Geo<R> &g, const double *__restrict__ Zt,
                                               R *__restrict__ z_w, R *__restrict__ z_r,
                                               R *__restrict__ Hz, const long p) {
    if (p >= g.s2) return;
    const long s2 = g.s2;
    const int N = g.N;
    const double hc = g.hc, h = g.hd[p], zt = Zt[p];
    // The FP32 form, whose outputs are rounded to FP32, multiplies by the column's reciprocal
    // depth instead of dividing at every level; FP64 divides as the reference does.
    constexpr bool recip = sizeof(R) == 4;
    const double ih = recip ? 1.0 / h : 0.0, ihc = recip ? 1.0 / (hc + h) : 0.0;
    double zprev = 0.0;
    for (int K = 0; K <= N; ++K) {
        double zw;
        if (K == N) {
            zw = zt;
        } else if (g.Vtransform == 1) {
            const double z_r0 = hc * (g.sc_r[K] - g.Cs_r[K]) + g.Cs_r[K] * h;
            const double z_w0 = hc * (g.sc_w[K] - g.Cs_w[K]) + g.Cs_w[K] * h;
            zw = z_w0 + zt * (1.0 + (recip ? z_w0 * ih : z_w0 / h));
            z_r[(long)K * s2 + p] = (R)(z_r0 + zt * (1.0 + (recip ? z_r0 * ih : z_r0 / h)));
        } else {
            const double nr = hc * g.sc_r[K] + g.Cs_r[K] * h, nw = hc * g.sc_w[K] + g.Cs_w[K] * h;
            const double cff2_r = recip ? nr * ihc : nr / (hc + h);
            const double cff2_w = recip ? nw * ihc : nw / (hc + h);
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
// Tridiagonal storage of one column: per-thread arrays (local memory, cached in L1), element
// k of each at FC[k*B + t] (B = 1, t = 0 here).
template <typename R>
struct Tri {
    R *FC, *BD, *RHS;
    int B, t;
    __device__ __forceinline__ R &fc(int k) const { return FC[k * B + t]; }
    __device__ __forceinline__ R &bd(int k) const { return BD[k * B + t]; }
    __device__ __forceinline__ R &rhs(int k) const { return RHS[k * B + t]; }
};

// createVertViscousOpMatrix (:568-639) for the column at p (d = 1: U, d = I: V) fused with the
// forward elimination of solveTri (:547-554): row k is built and eliminated against row k-1
// with the same operations, in the same order, as building the whole matrix first.  Also
// returns H = sum HzU and Hu = sum old*HzU (correctBaroclinicMeanVel, :502-506), ascending.
template <typename R>
__device__ __forceinline__ void build_eliminate(const Geo<R> &g, long p, long d, R cff, R Dt,
                                                R lambda, const Tri<R> &m, const R *Hz,
                                                const R *Akv, const R *z_r, const R *old,
                                                const R *ru, double &H, double &Hu) {
    const long s2 = g.s2;
    const int N = g.N;
    const R pmU = (g.pm[p] + g.pm[p - d]) * R(0.5), pnU = (g.pn[p] + g.pn[p - d]) * R(0.5);
    const R cdt = cff * Dt;
    const R cm = -lambda * Dt;
    const R cmn = cdt * (pmU * pnU);
#define AT(X, k, q) ((X)[(long)(k) * s2 + (q)])
    R zr0 = AT(z_r, 0, p), zr0d = AT(z_r, 0, p - d);
    R zr1 = AT(z_r, 1, p), zr1d = AT(z_r, 1, p - d);
    R fcm = (cm * ((AT(Akv, 0, p) + AT(Akv, 0, p - d)) * R(0.5))) /
            (((zr1 - zr0) + (zr1d - zr0d)) * R(0.5));
    R hz = (AT(Hz, 0, p) + AT(Hz, 0, p - d)) * R(0.5);
    R bdm = hz - R(2.0) * fcm;
    R rhsm = R(0);
    m.fc(0) = fcm;
    m.bd(0) = bdm;
    m.rhs(0) = rhsm;
    H = (double)hz;
    Hu = (double)(old[0] * hz);
#pragma unroll 2
    for (int k = 1; k < N; ++k) {
        hz = (AT(Hz, k, p) + AT(Hz, k, p - d)) * R(0.5);
        R fck = R(0);
        if (k < N - 1) {
            const R zr2 = AT(z_r, k + 1, p), zr2d = AT(z_r, k + 1, p - d);
            fck = (cm * ((AT(Akv, k, p) + AT(Akv, k, p - d)) * R(0.5))) /
                  (((zr2 - zr1) + (zr2d - zr1d)) * R(0.5));
            zr1 = zr2;
            zr1d = zr2d;
        }
        const R ok = old[(long)k * s2];
        const R rhsk = hz * (ok + cmn * AT(ru, k, p));
        const R bdk = (k < N - 1) ? (hz - fck) - fcm : hz - fcm;
        const R w = fcm / bdm;
        bdm = bdk - w * fcm;
        rhsm = rhsk - w * rhsm;
        m.fc(k) = fck;
        m.bd(k) = bdm;
        m.rhs(k) = rhsm;
        fcm = fck;
        H += (double)hz;
        Hu += (double)(ok * hz);
    }
#undef AT
}

// A second forward elimination of an already eliminated system (solveTri applied twice, :525).
template <typename R>
__device__ __forceinline__ void eliminate_again(int N, const Tri<R> &m) {
    R bdm = m.bd(0), rhsm = m.rhs(0);
    for (int k = 1; k < N; ++k) {
        const R fcm = m.fc(k - 1);
        const R w = fcm / bdm;
        bdm = m.bd(k) - w * fcm;
        rhsm = m.rhs(k) - w * rhsm;
        m.bd(k) = bdm;
        m.rhs(k) = rhsm;
    }
}

// Back substitution of solveTri (:557-563) into out[k*s2], minus `sub` (:512-515).
template <typename R>
__device__ __forceinline__ void back_substitute(int N, long s2, const Tri<R> &m, R *out, R sub) {
    R x = m.rhs(N - 1) / m.bd(N - 1);
    out[(long)(N - 1) * s2] = x - sub;
    for (int k = N - 2; k >= 0; --k) {
        x = (m.rhs(k) - m.fc(k) * x) / m.bd(k);
        out[(long)k * s2] = x - sub;
    }
}

template <typename R>
__device__ __forceinline__ R mean_correction(int N, long s2, long p, long d, const R *Hz,
                                             const R *old, double DUp, double on) {
    double H = 0.0, Hu = 0.0;
#pragma unroll 4
    for (int K = 0; K < N; ++K) {
        const long o = (long)K * s2 + p;
        const R hzu = (Hz[o] + Hz[o - d]) * R(0.5);
        H += (double)hzu;
        Hu += (double)(old[(long)K * s2] * hzu);
    }
    return (R)((Hu - DUp / on) / H);
}

template <typename R>
__device__ __forceinline__ void step3d_uv_body(const Geo<R> &g, R *__restrict__ u, R *__restrict__ v,
                            const R *__restrict__ ru, const R *__restrict__ rv,
                            R *__restrict__ ubar_t1, R *__restrict__ vbar_t1,
                            R *__restrict__ ubar_t2, R *__restrict__ vbar_t2,
                            const R *__restrict__ Hz, const R *__restrict__ Akv,
                            const R *__restrict__ z_r, const double *__restrict__ DU,
                            const double *__restrict__ DV, const R *tmpU, const R *tmpV, R cff,
                            R lambda, R Dt, int do_bc, R bcval, const long pl) {
    const int N = g.N;
    R FCa[kNMax], BDa[kNMax], RHSa[kNMax];
    const Tri<R> m{FCa, BDa, RHSa, 1, 0};
    if (pl >= g.s2) return;      // no barriers below
    const int pi = (int)pl;
    const long p = pi;
    const long I = g.I, s2 = g.s2;
    const int i = pi % g.I, j = pi / g.I;
    const bool un = unode_(i, j), vn = vnode_(i, j, g.J);
    if (un || vn) {
        const R *uo = (tmpU ? tmpU : u) + p;
        const R *vo = (tmpV ? tmpV : v) + p;
        if (un) {
            double H, Hu;
            build_eliminate(g, p, 1, cff, Dt, lambda, m, Hz, Akv, z_r, uo, ru, H, Hu);
            const R udiff = (R)((Hu - DU[p] / (double)g.on_u[p]) / H);
            back_substitute(N, s2, m, u + p, udiff);
        }
        if (vn && un) {
            double H, Hv;
            build_eliminate(g, p, I, cff, Dt, lambda, m, Hz, Akv, z_r, vo, rv, H, Hv);
            const R vdiff = (R)((Hv - DV[p] / (double)g.om_v[p]) / H);
            back_substitute(N, s2, m, v + p, vdiff);
        } else if (un) {
            // solveTri is gated by isUNode for both directions (:525): where p is a U node but
            // not a V node it solves the U system left in the scratch a second time.
            eliminate_again(N, m);
            back_substitute(N, s2, m, v + p, R(0));
        } else {
            const R vdiff = mean_correction(N, s2, p, I, Hz, vo, DV[p], (double)g.om_v[p]);
            for (int K = 0; K < N; ++K) v[(long)K * s2 + p] = v[(long)K * s2 + p] - vdiff;
        }
        if (un) {   // adjustBarotropicVelocity (:408-469)
            double HU = 0.0, HV = 0.0, HuU = 0.0, HvV = 0.0;
#pragma unroll 4
            for (int K = 0; K < N; ++K) {
                const long o = (long)K * s2 + p;
                const R hzu = (Hz[o] + Hz[o - 1]) * R(0.5), hzv = (Hz[o] + Hz[o - I]) * R(0.5);
                HU += (double)hzu;
                HV += (double)hzv;
                HuU += (double)(hzu * u[o]);
                HvV += (double)(hzv * v[o]);
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

// ---- FP32 form of step3d_UV: a pipelined column solve --------------------------------------
// The same systems as build_eliminate/back_substitute for a tile of 64 consecutive flat points.
// Memory and arithmetic are decoupled: the block streams the levels of its tile through a
// ring of kPipeDepth shared-memory slots with cp.async (Hz, Akv, z_r at p, p-1 and p-I; the
// old velocities and ru/rv at p), several levels ahead of the elimination, so that the bytes
// in flight do not depend on how many threads an SM holds.  The U and V systems are
// eliminated in one pass in the normalised Thomas form (c'_k = c_k / m_k,
// d'_k = (r_k - a_k d'_{k-1}) / m_k, x_k = d'_k - c'_k x_{k+1}) with c' in shared memory and
// d' in the output column itself (level k of u or v, whose old value the ring has already
// staged; the back substitution reads it back in chunks and overwrites it with x_k), which
// keeps a block's shared memory small enough for five blocks per SM,
// and the barotropic sums of adjustBarotropicVelocity come from the column identity
// sum_k hz_k x_k = sum_k r_k + fc_0 x_0 (the rows of the system summed: the off-diagonal terms
// telescope, the bottom row keeps -fc_0 x_0), so the back-substitution reads nothing from
// memory.  Rounding differs from the FP64 kernel's order of operations, within the FP32
// form's tolerance.  Columns on the rows where the reference solves the U system a second
// time for V (solveTri gated by isUNode, :525) and where V gets only the mean correction take
// the general path above after the pipelined part.
constexpr int kPipeCols = kPipeTile;
constexpr int kPipeGroup = 2;               // levels consumed per barrier pair
constexpr int kPipeDepth = 3 * kPipeGroup;  // levels in flight (shared-memory ring slots)
constexpr int kPipeThreads = 2 * kPipeCols;   // one thread per system (U, V) and column
// A ring slot holds one level: rows of Hz, Akv and z_r(k+1) followed by the old u, old v, ru and
// rv of the tile's columns.  Element staging (cp.async): a row is [p0-1, p0+63] then
// [p0-I, p0-I+63] (kRow floats).  Bulk staging (cp.async.bulk): a row is two 16-byte-aligned
// spans of 68 floats, [p0-4, p0+64) and [p0-I-r, p0-I-r+68) with r = (-I) mod 4 (kRowB floats).
constexpr int kRow = 2 * kPipeCols + 1;
constexpr int kSpan = kPipeCols + 4;
constexpr int kRowB = 2 * kSpan;
constexpr int kSlotE = 3 * kRow + 4 * kPipeCols, kSlotB = 3 * kRowB + 4 * kPipeCols;
constexpr int kPipeSlot = kSlotE > kSlotB ? kSlotE : kSlotB;   // floats per level
static_assert((kRowB * 4) % 16 == 0 && (kSpan * 4) % 16 == 0 && (kPipeSlot * 4) % 16 == 0,
              "bulk-copy destinations must stay 16-byte aligned");

__host__ __device__ constexpr size_t pipe_smem_bytes(int N) {
    // [N][kPipeThreads] c' | ring of kPipeDepth slots | kPipeDepth mbarriers (bulk staging)
    return sizeof(float) * ((size_t)N * kPipeThreads + (size_t)kPipeDepth * kPipeSlot) +
           8 * (size_t)kPipeDepth;
}
// levels of d' read ahead per step of the back substitution (basin4: 1.19 ms with 8, 1.17 with
// 16 or 32)
constexpr int kBackChunk = 16;

// Bulk copies (the TMA unit's non-tensor form) into shared memory, completing on an mbarrier.
__device__ __forceinline__ void mbar_init1(uint32_t a) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(a) : "memory");
}
__device__ __forceinline__ void mbar_expect_tx(uint32_t a, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(a), "r"(bytes)
                 : "memory");
}
__device__ __forceinline__ void bulk_g2s(uint32_t dst, const void *src, uint32_t bytes, uint32_t bar) {
    asm volatile(
        "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(dst),
        "l"(src), "r"(bytes), "r"(bar)
        : "memory");
}
// Bounded wait for an mbarrier phase: false (and the context's error word set) if it gave up.
__device__ __forceinline__ bool mbar_wait_bounded(uint32_t a, uint32_t parity, int *err) {
    for (int it = 0; it < (1 << 22); ++it) {
        uint32_t done;
        asm volatile(
            "{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
            "selp.u32 %0, 1, 0, p;\n\t}\n"
            : "=r"(done)
            : "r"(a), "r"(parity)
            : "memory");
        if (done) return true;
    }
    if (err) atomicExch(err, 1);
    return false;
}

// MODE 0: every thread stages its own elements with 4-byte cp.async.  MODE 1: the tile's levels
// arrive by bulk copies issued by thread 0 (ten per level, one mbarrier per ring slot).  MODE 2:
// the threads stage the same 16-byte-aligned spans as MODE 1 with 16-byte cp.async, chunks
// spread over the block (two per thread per level), completing through cp.async groups as in
// MODE 0.  The arithmetic is the same in every mode, so they give identical results; modes 1
// and 2 are used for tiles whose spans lie inside the fields (all but the first row of tiles
// and the last tile) when the plane size and the field addresses keep the spans 16-byte
// aligned.
template <typename R, int MODE>   // R = float only: the FP32 form
__device__ __forceinline__ void step3d_uv_pipe_body(const Geo<R> &g, float *__restrict__ u,
        float *__restrict__ v, const float *__restrict__ ru, const float *__restrict__ rv,
        float *__restrict__ ubar_t1, float *__restrict__ vbar_t1, float *__restrict__ ubar_t2,
        float *__restrict__ vbar_t2, const float *__restrict__ Hz, const float *__restrict__ Akv,
        const float *__restrict__ z_r, const double *__restrict__ DU,
        const double *__restrict__ DV, const float *tmpU, const float *tmpV, float cff,
        float lambda, float Dt, int do_bc, float bcval, const long tile) {
    constexpr bool BULK = MODE == 1;       // bulk copies completing on mbarriers
    constexpr bool LAYB = MODE != 0;       // the aligned-span ring layout
    extern __shared__ __align__(16) float spipe[];
    const int N = g.N;
    const long I = g.I, s2 = g.s2;
    // two threads per column: sys 0 solves the U system of column col, sys 1 its V system
    const int col = threadIdx.x & (kPipeCols - 1), sys = threadIdx.x / kPipeCols;
    const long p0 = tile * kPipeCols;
    const long p = p0 + col;
    float *cc = spipe + threadIdx.x;   // [level][thread]
    float *ring = spipe + N * kPipeThreads;
    float *const outc = (sys == 0 ? u : v) + p;   // this system's output column (d', then x)
    const float *uo_all = tmpU ? tmpU : u, *vo_all = tmpV ? tmpV : v;
    const uint32_t ring_s = (uint32_t)__cvta_generic_to_shared(ring);
    const uint32_t bar_s = ring_s + 4u * kPipeDepth * kPipeSlot;
    const int s2i = (int)s2;
    const int rB = (int)((4 - (I & 3)) & 3);   // the second span starts r before p0 - I
    constexpr int row = LAYB ? kRowB : kRow;    // floats between the Hz, Akv and z_r rows
    // this thread's own (p) and neighbour (p-1 or p-I) entries in a row
    const int iP = LAYB ? col + 4 : col + 1;
    const int iQ = LAYB ? (sys == 0 ? col + 3 : kSpan + rB + col) : (sys == 0 ? col : kPipeCols + 1 + col);

    // level k goes to ring slot k % kPipeDepth; the main loop is unrolled over one turn of the
    // ring so that every slot index (and so every shared-memory offset) is a constant
    // element staging: level k into slot: Hz(k), Akv(k), z_r(k+1) at [p0-1, p0+63] (sys 0
    // copies these, plus old u and ru) and [p0-I, p0-I+63] (sys 1, plus old v and rv); sources
    // outside [0, s2) in the plane are zero-filled (their columns are not U/V nodes).
    const long q = sys == 0 ? p0 - 1 + col : p0 - I + col, qE = p0 + kPipeCols - 1;
    const bool okq = q >= 0 && q < s2, okP = p < s2;
    const bool okE = sys == 0 && col == 0 && qE < s2;
    const int seg = sys == 0 ? col : kPipeCols + 1 + col;
    const long qq = okq ? q : 0, qe = okE ? qE : 0, pp = okP ? p : 0;
    const float *const cHz = Hz + qq, *const cAk = Akv + qq, *const cZr = z_r + s2 + qq;
    const float *const eHz = Hz + qe, *const eAk = Akv + qe, *const eZr = z_r + s2 + qe;
    const float *const cO = (sys == 0 ? uo_all : vo_all) + pp, *const cR = (sys == 0 ? ru : rv) + pp;
    const int nq = okq ? 4 : 0, ne = okE ? 4 : 0, np = okP ? 4 : 0;
    const bool edge = sys == 0 && col == 0;
    const int oO = 3 * kRow + sys * kPipeCols + col, oR = 3 * kRow + (2 + sys) * kPipeCols + col;
    // destinations as shared-window byte addresses in slot 0 (a level adds its slot's offset;
    // the three fields of a row at immediate offsets), sources as 32-bit element offsets from
    // level 0 (the launcher keeps (N+1) s2 below 2^31 for this kernel)
    const uint32_t dq = ring_s + 4u * seg, dE = ring_s + 4u * kPipeCols;
    const uint32_t dO = ring_s + 4u * oO, dR = ring_s + 4u * oR;
    // MODE 2: this thread's two 16-byte chunks of every level, fixed per thread: 17 chunks per
    // span (Hz, Akv, z_r(k+1) at p0 - 4 and p0 - I - r), then 16 per column field (old u, old
    // v, ru, rv); destination byte offsets within a slot, sources at level 0
    bool vact[2] = {false, false}, vzr[2] = {false, false};
    uint32_t vdst[2] = {0u, 0u};
    const float *vsrc[2] = {Hz, Hz};
    if constexpr (MODE == 2) {
        constexpr int kSpanCh = kSpan / 4, kColCh = kPipeCols / 4;
#pragma unroll
        for (int h = 0; h < 2; ++h) {
            const int ch = (int)threadIdx.x + h * kPipeThreads;
            if (ch < 6 * kSpanCh) {
                const int s = ch / kSpanCh, q = ch - s * kSpanCh;
                const int fld = s >> 1, half = s & 1;
                const float *base = fld == 0 ? Hz : fld == 1 ? Akv : z_r + s2;
                vact[h] = true;
                vzr[h] = fld == 2;
                vdst[h] = 4u * (uint32_t)(fld * row + half * kSpan + 4 * q);
                vsrc[h] = base + (half ? p0 - I - rB : p0 - 4) + 4 * q;
            } else if (ch < 6 * kSpanCh + 4 * kColCh) {
                const int c4 = ch - 6 * kSpanCh, f4 = c4 / kColCh, q = c4 - f4 * kColCh;
                const float *base = f4 == 0 ? uo_all : f4 == 1 ? vo_all : f4 == 2 ? ru : rv;
                vact[h] = true;
                vdst[h] = 4u * (uint32_t)(3 * row + f4 * kPipeCols + 4 * q);
                vsrc[h] = base + p0 + 4 * q;
            }
        }
    }
    auto issue = [&](int k, int sl) {
        const uint32_t sb = (uint32_t)sl * (4u * kPipeSlot);
        const int o = k * s2i;
        const bool zr = k + 1 < N;   // z_r(k+1) exists for k < N-1 only
        if constexpr (BULK) {   // thread 0 only
            const uint32_t bar = bar_s + 8u * sl, d0 = ring_s + sb;
            constexpr uint32_t sp = 4u * kSpan, cb = 4u * kPipeCols;
            mbar_expect_tx(bar, (zr ? 6u : 4u) * sp + 4u * cb);
            const long a = o + p0 - 4, b = o + p0 - I - rB;
            bulk_g2s(d0, Hz + a, sp, bar);
            bulk_g2s(d0 + sp, Hz + b, sp, bar);
            bulk_g2s(d0 + 4u * row, Akv + a, sp, bar);
            bulk_g2s(d0 + 4u * row + sp, Akv + b, sp, bar);
            if (zr) {
                bulk_g2s(d0 + 8u * row, z_r + s2 + a, sp, bar);
                bulk_g2s(d0 + 8u * row + sp, z_r + s2 + b, sp, bar);
            }
            const uint32_t dv = d0 + 12u * row;
            bulk_g2s(dv, uo_all + o + p0, cb, bar);
            bulk_g2s(dv + cb, vo_all + o + p0, cb, bar);
            bulk_g2s(dv + 2u * cb, ru + o + p0, cb, bar);
            bulk_g2s(dv + 3u * cb, rv + o + p0, cb, bar);
        } else if constexpr (MODE == 2) {
            const uint32_t d0 = ring_s + sb;
#pragma unroll
            for (int h = 0; h < 2; ++h)
                if (vact[h] && (zr || !vzr[h])) cp_async16(d0 + vdst[h], vsrc[h] + o);
        } else {
            const int oz = zr ? o : o - s2i;
            cp_async_at<0>(dq + sb, cHz + o, nq);
            cp_async_at<4 * kRow>(dq + sb, cAk + o, nq);
            cp_async_at<8 * kRow>(dq + sb, cZr + oz, zr ? nq : 0);
            if (edge) {
                cp_async_at<0>(dE + sb, eHz + o, ne);
                cp_async_at<4 * kRow>(dE + sb, eAk + o, ne);
                cp_async_at<8 * kRow>(dE + sb, eZr + oz, zr ? ne : 0);
            }
            cp_async_at<0>(dO + sb, cO + o, np);
            cp_async_at<0>(dR + sb, cR + o, np);
        }
    };
    const int i = (int)(p % I), j = (int)(p / I);
    const bool live = p < s2;
    const bool un = live && unode_(i, j), vn = live && vnode_(i, j, g.J);
    const bool both = un && vn;
    const long d = sys == 0 ? 1 : I;   // the neighbour of this system's face

    constexpr int kAhead = kPipeDepth - kPipeGroup;   // levels issued before the first group
    if constexpr (BULK) {
        if (threadIdx.x == 0) {
            for (int k = 0; k < kPipeDepth; ++k) mbar_init1(bar_s + 8u * k);
            asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
        }
        __syncthreads();
        if (threadIdx.x == 0) {
#pragma unroll
            for (int k = 0; k < kAhead; ++k)
                if (k < N) issue(k, k);
        }
    } else {
#pragma unroll
        for (int k = 0; k < kAhead; ++k) {
            if (k < N) issue(k, k);
            cp_async_commit();
        }
    }
    const float cm = -lambda * Dt;
    float cmn = 0.f, zP = 0.f, zQ = 0.f;
    if (both) {
        cmn = cff * Dt * (((g.pm[p] + g.pm[p - d]) * 0.5f) * ((g.pn[p] + g.pn[p - d]) * 0.5f));
        zP = z_r[p];
        zQ = z_r[p - d];
    }
    float fc = 0.f, fc0 = 0.f, ccp = 0.f, ddp = 0.f;
    double H = 0.0, O = 0.0, Rs = 0.0;
    // levels in groups of kPipeGroup: one wait and one barrier per group.  After the barrier of
    // group g every thread has finished group g-1, whose slots (kPipeDepth is a multiple of the
    // group) are refilled with group g+2, so two groups are in flight while one is eliminated
    static_assert(kPipeDepth % kPipeGroup == 0, "levels are consumed in whole groups");
    auto level = [&](int k, int slot) {
        const float *sl = ring + slot * kPipeSlot;
        const float *sHz = sl, *sAk = sl + row, *sZr = sl + 2 * row;
        const float *sO = sl + 3 * row + sys * kPipeCols, *sR = sl + 3 * row + (2 + sys) * kPipeCols;
        const float hz = (sHz[iP] + sHz[iQ]) * 0.5f;
        float gk = 0.f;
        if (k < N - 1) {
            const float zP1 = sZr[iP], zQ1 = sZr[iQ];
            // divisions by layer spacings and pivots (metres): the reciprocal form, as ddiv
            gk = __fdividef(cm * ((sAk[iP] + sAk[iQ]) * 0.5f), ((zP1 - zP) + (zQ1 - zQ)) * 0.5f);
            zP = zP1;
            zQ = zQ1;
        }
        const float ok = sO[col];
        if (k == 0) {   // bottom row: right-hand side forced to 0 (:610)
            fc0 = gk;
            ccp = __fdividef(gk, hz - 2.f * gk);
            ddp = 0.f;
        } else {
            const float rr = hz * (ok + cmn * sR[col]);
            const float bd = (k < N - 1) ? (hz - gk) - fc : hz - fc;
            const float iv = __fdividef(1.f, bd - fc * ccp);
            ccp = gk * iv;
            ddp = (rr - fc * ddp) * iv;
            Rs += (double)rr;
        }
        cc[k * kPipeThreads] = ccp;
        outc[k * s2i] = ddp;
        fc = gk;
        H += (double)hz;
        O += (double)(ok * hz);
    };
    for (int k0 = 0; k0 < N; k0 += kPipeDepth) {   // one turn of the ring
        const uint32_t parity = (uint32_t)((k0 / kPipeDepth) & 1);
#pragma unroll
        for (int gs = 0; gs < kPipeDepth; gs += kPipeGroup) {   // group in slots gs, gs+1, ...
            const int kg = k0 + gs;
            if (kg < N) {   // uniform over the block
                if constexpr (BULK) {
#pragma unroll
                    for (int h = 0; h < kPipeGroup; ++h)
                        if (kg + h < N) mbar_wait_bounded(bar_s + 8u * (gs + h), parity, g.err);
                    __syncthreads();
                    if (threadIdx.x == 0) {
                        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
#pragma unroll
                        for (int h = 0; h < kPipeGroup; ++h)
                            if (kg + kAhead + h < N) issue(kg + kAhead + h, (gs + kAhead + h) % kPipeDepth);
                    }
                } else {
                    cp_async_wait<kAhead - kPipeGroup>();   // this group's levels (the next may be in flight)
                    __syncthreads();
#pragma unroll
                    for (int h = 0; h < kPipeGroup; ++h) {
                        if (kg + kAhead + h < N) issue(kg + kAhead + h, (gs + kAhead + h) % kPipeDepth);
                        cp_async_commit();
                    }
                }
                if (both) {
#pragma unroll
                    for (int h = 0; h < kPipeGroup; ++h)
                        if (kg + h < N) level(kg + h, gs + h);
                }
            }
        }
    }
    cp_async_wait<0>();
    if (both) {
        const double dbar = sys == 0 ? DU[p] / (double)g.on_u[p] : DV[p] / (double)g.om_v[p];
        const float sub = (float)((O - dbar) / H);
        float x = ddp;
        outc[(N - 1) * s2i] = x - sub;
        for (int k = N - 2; k >= 0; k -= kBackChunk) {
            float dv[kBackChunk];   // the chunk's d' first (independent loads), then the chain
#pragma unroll
            for (int h = 0; h < kBackChunk; ++h) dv[h] = k - h >= 0 ? outc[(k - h) * s2i] : 0.f;
#pragma unroll
            for (int h = 0; h < kBackChunk; ++h) {
                if (k - h >= 0) {
                    x = dv[h] - cc[(k - h) * kPipeThreads] * x;
                    outc[(k - h) * s2i] = x - sub;
                }
            }
        }
        // sum_k hz_k (x_k - sub) from the column identity
        const double Hx = Rs + (double)fc0 * (double)x - (double)sub * H;
        const float bar = (float)(dbar / H + (Hx - dbar) / H);
        if (sys == 0) {
            ubar_t2[p] = bar;
            ubar_t1[p] = bar;
        } else {
            vbar_t2[p] = bar;
            vbar_t1[p] = bar;
        }
    } else if ((un || vn) && sys == 0) {
        const float *uo = uo_all + p, *vo = vo_all + p;
        float FCa[kNMax], BDa[kNMax], RHSa[kNMax];
        const Tri<float> m{FCa, BDa, RHSa, 1, 0};
        if (un) {
            double Hh, Hu;
            build_eliminate(g, p, 1, cff, Dt, lambda, m, Hz, Akv, z_r, uo, ru, Hh, Hu);
            const float udiff = (float)((Hu - DU[p] / (double)g.on_u[p]) / Hh);
            back_substitute(N, s2, m, u + p, udiff);
            eliminate_again(N, m);
            back_substitute(N, s2, m, v + p, 0.f);
            double HU2 = 0.0, HV2 = 0.0, HuU = 0.0, HvV = 0.0;
            for (int K = 0; K < N; ++K) {
                const long o = (long)K * s2 + p;
                const float hzu = (Hz[o] + Hz[o - 1]) * 0.5f, hzv = (Hz[o] + Hz[o - I]) * 0.5f;
                HU2 += (double)hzu;
                HV2 += (double)hzv;
                HuU += (double)(hzu * u[o]);
                HvV += (double)(hzv * v[o]);
            }
            const double duo = DU[p] / (double)g.on_u[p], dvo = DV[p] / (double)g.om_v[p];
            const float ub = (float)(duo / HU2 + (HuU - duo) / HU2);
            const float vb = (float)(dvo / HV2 + (HvV - dvo) / HV2);
            ubar_t2[p] = ub;
            vbar_t2[p] = vb;
            ubar_t1[p] = ub;
            vbar_t1[p] = vb;
        } else {
            const float vdiff = mean_correction(N, s2, p, I, Hz, vo, DV[p], (double)g.om_v[p]);
            for (int K = 0; K < N; ++K) v[(long)K * s2 + p] = v[(long)K * s2 + p] - vdiff;
        }
    }
    if (do_bc && live) {   // by the thread that wrote the column's field last
        const bool uown = sys == 0, vown = both ? sys == 1 : sys == 0;
        const int ut = g.utype[p], vt = g.vtype[p];
        if (uown && ut > 0 && (ut & (1 << 4)) == 0 && (ut & (1 << 3)) != 0)
            for (int K = 0; K < N; ++K) u[(long)K * s2 + p] = bcval;
        if (vown && vt > 0 && ((vt & (1 << 4)) != 0 || (vt & (1 << 3)) != 0))
            for (int K = 0; K < N; ++K) v[(long)K * s2 + p] = 0.f;
    }
}

// ---- obc_volcons (nonlinear/obc_volcons.py:6-69, ROMS pseudo-code in the reference) -------
// Area and volume flux through the open edges (W=1, E=2, S=4, N=8 in `edges`), in FP64 with
// compensated (two-sum) accumulation in a fixed order, so the result is deterministic:
//   W: cff = (D(0,j) + D(1,j))/2 on_u(1,j),    flux += cff ubar(1,j)
//   E: cff = (D(L-1,j) + D(L,j))/2 on_u(L,j),  flux -= cff ubar(L,j)
//   S: cff = (D(i,0) + D(i,1))/2 om_v(i,1),    flux += cff vbar(i,1)
//   N: cff = (D(i,M-1) + D(i,M))/2 om_v(i,M),  flux -= cff vbar(i,M)
// with D = zeta + h, j = 1..M-1, i = 1..L-1; ubar_xs = flux / area.
struct TwoSum {
    double s = 0.0, c = 0.0;
    __device__ void add(double x) {       // Neumaier's compensated summation
        const double t = s + x;
        c += fabs(s) >= fabs(x) ? (s - t) + x : (x - t) + s;
        s = t;
    }
    __device__ double value() const { return s + c; }
};

constexpr int kVolThreads = 256;

template <typename R>
__global__ void __launch_bounds__(kVolThreads) k_obc_volcons(Geo<R> g, const R *__restrict__ zeta,
                                                             const R *__restrict__ ubar,
                                                             const R *__restrict__ vbar, int edges,
                                                             double *__restrict__ out) {
    const int I = g.I, J = g.J, L = I - 1, M = J - 1;
    const int nj = M - 1, ni = L - 1;          // interior rows / columns
    TwoSum area, flux;
    const int n = 2 * nj + 2 * ni;
    for (int e = threadIdx.x; e < n; e += kVolThreads) {
        int side, a;
        if (e < nj) { side = 0; a = 1 + e; }
        else if (e < 2 * nj) { side = 1; a = 1 + e - nj; }
        else if (e < 2 * nj + ni) { side = 2; a = 1 + e - 2 * nj; }
        else { side = 3; a = 1 + e - 2 * nj - ni; }
        if (!(edges & (1 << side))) continue;
        long q0, q1, f;
        double metric, vel, sgn;
        if (side < 2) {
            const int i1 = side == 0 ? 1 : L;
            q0 = (long)a * I + i1 - 1;
            q1 = q0 + 1;
            f = (long)a * I + i1;
            metric = (double)g.on_u[f];
            vel = (double)ubar[f];
            sgn = side == 0 ? 1.0 : -1.0;
        } else {
            const int j1 = side == 2 ? 1 : M;
            q0 = (long)(j1 - 1) * I + a;
            q1 = q0 + I;
            f = (long)j1 * I + a;
            metric = (double)g.om_v[f];
            vel = (double)vbar[f];
            sgn = side == 2 ? 1.0 : -1.0;
        }
        const double cff = 0.5 * (((double)zeta[q0] + g.hd[q0]) + ((double)zeta[q1] + g.hd[q1])) * metric;
        area.add(cff);
        flux.add(sgn * cff * vel);
    }
    __shared__ double sa[kVolThreads], sf[kVolThreads];
    sa[threadIdx.x] = area.value();
    sf[threadIdx.x] = flux.value();
    __syncthreads();
    if (threadIdx.x == 0) {
        TwoSum A, F;
        for (int t = 0; t < kVolThreads; ++t) {
            A.add(sa[t]);
            F.add(sf[t]);
        }
        const double a = A.value(), fl = F.value();
        out[0] = a;
        out[1] = fl;
        out[2] = a > 0.0 ? fl / a : 0.0;     // ubar_xs
    }
}

// conserve_mass_tile: the normal velocity on the open edges corrected by ubar_xs.
template <typename R>
__global__ void k_conserve_mass(Geo<R> g, R *__restrict__ ubar, R *__restrict__ vbar, int edges,
                                const double *__restrict__ xs_in) {
    const int I = g.I, J = g.J, L = I - 1, M = J - 1;
    const int nj = M - 1, ni = L - 1;
    const int e = (int)tid_flat();
    if (e >= 2 * nj + 2 * ni) return;
    const double xs = xs_in[2];
    if (e < nj) {
        if (edges & 1) ubar[(long)(1 + e) * I + 1] -= (R)xs;
    } else if (e < 2 * nj) {
        if (edges & 2) ubar[(long)(1 + e - nj) * I + L] += (R)xs;
    } else if (e < 2 * nj + ni) {
        if (edges & 4) vbar[(long)1 * I + 1 + e - 2 * nj] -= (R)xs;
    } else {
        if (edges & 8) vbar[(long)M * I + 1 + e - 2 * nj - ni] += (R)xs;
    }
}

template <typename R>
cudaError_t Ops<R>::obc_volcons(const sf_ctx *c, const R *zeta, R *ubar, R *vbar, int edges,
                                int correct, double *out, cudaStream_t s) {
    k_obc_volcons<R><<<1, kVolThreads, 0, s>>>(geo(c), zeta, ubar, vbar, edges, out);
    if (correct) {
        const int n = 2 * (c->J - 2) + 2 * (c->I - 2);
        k_conserve_mass<R><<<(unsigned)((n + kBlock - 1) / kBlock), kBlock, 0, s>>>(geo(c), ubar,
                                                                                  vbar, edges, out);
    }
    return cudaGetLastError();
}

// setLateralUVBCs alone (step3D_uv.kernels.cpp:314-368).
template <typename R>
__device__ __forceinline__ void lateral_uv_bc_at(const Geo<R> &g, R *__restrict__ u,
                                                 R *__restrict__ v, R bcval, const long p) {
    if (p >= g.s2) return;
    const long s2 = g.s2;
    const int ut = g.utype[p], vt = g.vtype[p];
    if (ut <= 0 && vt <= 0) return;
    if (ut > 0 && (ut & (1 << 4)) == 0 && (ut & (1 << 3)) != 0)
        for (int K = 0; K < g.N; ++K) u[(long)K * s2 + p] = bcval;
    if (vt > 0 && ((vt & (1 << 4)) != 0 || (vt & (1 << 3)) != 0))
        for (int K = 0; K < g.N; ++K) v[(long)K * s2 + p] = R(0);
}
template <typename R>
__global__ void __launch_bounds__(kBlock) k_lateral_uv_bc(Geo<R> g, R *__restrict__ u,
                                                          R *__restrict__ v, R bcval) {
    lateral_uv_bc_at(g, u, v, bcval, tid_flat());
}

}  // namespace sf

#include "sf_gls.cuh"
#include "sf_pred2d.cuh"

namespace sf {

// ------------------------------------------------------------------------------------------
// Kernels: one grid (the arrays as given) and ensembles (pools; each block finds its member
// and its block within the member from a block map, and offsets the pools by the member's
// 2D / N+1-level / N-level offsets).  Both run the same bodies.
// ------------------------------------------------------------------------------------------
#define SF_MEMBER(bm)                                 \
    const int2 mb_ = (bm)[blockIdx.x];                 \
    const Member<R> &M_ = mt[mb_.x];                   \
    const Geo<R> g = M_.g;                             \
    const long o2 = M_.off2, o3 = M_.off3, oN = M_.offN; \
    (void)o2; (void)o3; (void)oN;
#define O2(x) ((x) ? (x) + o2 : (x))
#define O3(x) ((x) ? (x) + o3 : (x))
#define ON(x) ((x) ? (x) + oN : (x))

template <typename R>
__global__ void __launch_bounds__(kBlock, 3) k_zeta_rhs(
    Geo<R> g, const R *__restrict__ zeta, const R *__restrict__ ubar, const R *__restrict__ vbar, R *__restrict__ rzeta, int mode, double cff1,
    double *__restrict__ Zt, double *__restrict__ DU, double *__restrict__ DV, const R *__restrict__ zeta_t0, R *__restrict__ zeta_t2, R Dt) {
    pdl_enter();
    zeta_rhs4(g, zeta, ubar, vbar, rzeta, mode, cff1, Zt, DU, DV, zeta_t0, zeta_t2, Dt,
              4 * (long)tid_flat());
}
template <typename R>
__global__ void __launch_bounds__(kBlock) kb_zeta_rhs(
    const Member<R> *mt, const int2 *bm, const R *__restrict__ zeta, const R *__restrict__ ubar, const R *__restrict__ vbar, R *__restrict__ rzeta,
    int mode, double cff1, double *__restrict__ Zt, double *__restrict__ DU, double *__restrict__ DV, const R *__restrict__ zeta_t0, R *__restrict__ zeta_t2,
    R Dt) {
    pdl_enter();
    SF_MEMBER(bm)
    zeta_rhs_body(g, O2(zeta), O2(ubar), O2(vbar), O2(rzeta), mode, cff1, O2(Zt), O2(DU), O2(DV),
                  O2(zeta_t0), O2(zeta_t2), Dt, (long)mb_.y * kBlock + threadIdx.x);
}

template <typename R>
__global__ void __launch_bounds__(kBlock) k_momentum(
    Geo<R> g, R *__restrict__ rhs_u, R *__restrict__ rhs_v, const R *__restrict__ za, const R *__restrict__ zb, R grav, R w1, R w, int do_rhs,
    int do_pred, R Dt, const R *__restrict__ u_t1, R *__restrict__ u_t2, const R *__restrict__ v_t1, R *__restrict__ v_t2, const R *__restrict__ z1,
    const R *__restrict__ z2) {
    pdl_enter();
    momentum4(g, rhs_u, rhs_v, za, zb, grav, w1, w, do_rhs, do_pred, Dt, u_t1, u_t2, v_t1, v_t2,
              z1, z2, 4 * (long)tid_flat());
}
template <typename R>
__global__ void __launch_bounds__(kBlock) kb_momentum(
    const Member<R> *mt, const int2 *bm, R *__restrict__ rhs_u, R *__restrict__ rhs_v, const R *__restrict__ za, const R *__restrict__ zb, R grav,
    R w1, R w, int do_rhs, int do_pred, R Dt, const R *__restrict__ u_t1, R *__restrict__ u_t2, const R *__restrict__ v_t1, R *__restrict__ v_t2,
    const R *__restrict__ z1, const R *__restrict__ z2) {
    pdl_enter();
    SF_MEMBER(bm)
    momentum_body(g, O2(rhs_u), O2(rhs_v), O2(za), O2(zb), grav, w1, w, do_rhs, do_pred, Dt,
                  O2(u_t1), O2(u_t2), O2(v_t1), O2(v_t2), O2(z1), O2(z2),
                  (long)mb_.y * kBlock + threadIdx.x);
}

template <typename R>
__global__ void __launch_bounds__(kBlock) k_corr_point(
    Geo<R> g, R Dt, R *__restrict__ zeta_t2, const R *__restrict__ rz0, const R *__restrict__ rz1, const R *__restrict__ rz2, R *__restrict__ ubar_t1,
    const R *__restrict__ vbar_t1, const R *__restrict__ rub0, const R *__restrict__ rub1, R *__restrict__ vbar_t2) {
    pdl_enter();
    corr_point4(g, Dt, zeta_t2, rz0, rz1, rz2, ubar_t1, vbar_t1, rub0, rub1, vbar_t2,
                4 * (long)tid_flat());
}
template <typename R>
__global__ void __launch_bounds__(kBlock) kb_corr_point(
    const Member<R> *mt, const int2 *bm, R Dt, R *__restrict__ zeta_t2, const R *__restrict__ rz0, const R *__restrict__ rz1,
    const R *__restrict__ rz2, R *__restrict__ ubar_t1, const R *__restrict__ vbar_t1, const R *__restrict__ rub0, const R *__restrict__ rub1, R *__restrict__ vbar_t2) {
    pdl_enter();
    SF_MEMBER(bm)
    corr_point_body(g, Dt, O2(zeta_t2), O2(rz0), O2(rz1), O2(rz2), O2(ubar_t1), O2(vbar_t1),
                    O2(rub0), O2(rub1), O2(vbar_t2), (long)mb_.y * kBlock + threadIdx.x);
}

template <typename R, int TX, int TY, bool P2>
__global__ void __launch_bounds__(TX * TY, 1024 / (TX * TY)) k_rhs3d(Geo<R> g, const R *__restrict__ u, const R *__restrict__ v,
                                                  const R *Huon, const R *Hvom, const R *__restrict__ W,
                                                  const R *__restrict__ Hz, R *__restrict__ ru, R *__restrict__ rv) {
    rhs3d_body<R, TX, TY, P2>(g, u, v, Huon, Hvom, W, Hz, ru, rv, (int)blockIdx.x, (int)blockIdx.y);
}
// blocks of the marching form that fit an SM's shared memory (233,472 bytes, 1 KB of it
// reserved per block), at most 2048 threads
template <typename R, int NW, int RW, int SX>
constexpr int march_min_blocks() {
    const int b = (int)(233472 / (march_smem_bytes<R, NW, RW, SX>() + 1024));
    const int t = 2048 / (32 * NW);
    return b < 1 ? 1 : (b < t ? b : t);
}
template <typename R, int NW, int RW, int STG, int SX, bool SPLIT, int MINB>
__global__ void __launch_bounds__(32 * NW, MINB) k_rhs3d_march(
    Geo<R> g, const R *__restrict__ u, const R *__restrict__ v, const R *__restrict__ Huon,
    const R *__restrict__ Hvom, const R *__restrict__ W, const R *__restrict__ Hz,
    R *__restrict__ ru, R *__restrict__ rv) {
    rhs3d_march_body<R, NW, RW, STG, SX, SPLIT>(g, u, v, Huon, Hvom, W, Hz, ru, rv,
                                                (int)blockIdx.x, (int)blockIdx.y);
}
template <typename R, int TX, int TY>
__global__ void __launch_bounds__(TX *TY) kb_rhs3d(const Member<R> *mt, const int2 *bm, int var,
                                                   const R *__restrict__ u, const R *__restrict__ v, const R *Huon,
                                                   const R *Hvom, const R *__restrict__ W, const R *__restrict__ Hz,
                                                   R *__restrict__ ru, R *__restrict__ rv) {
    SF_MEMBER(bm)
    const int ntx = M_.ntx[var];
    rhs3d_body<R, TX, TY, false>(g, O3(u), O3(v), O3(Huon), O3(Hvom), O3(W), ON(Hz), O3(ru), O3(rv),
                                 mb_.y % ntx, mb_.y / ntx);
}

template <typename R, int C>
__global__ void __launch_bounds__(kBlock) k_maxflux_omega(
    Geo<R> g, const R *__restrict__ u, const R *__restrict__ v, R *Huon, R *Hvom, const R *__restrict__ Hz, R *__restrict__ W, const R *__restrict__ z_w,
    int do_flux, int do_omega, R *__restrict__ zeta1, R *__restrict__ zeta2, const double *__restrict__ Zt) {
    maxflux_omega_body<R, C>(g, u, v, Huon, Hvom, Hz, W, z_w, do_flux, do_omega, zeta1, zeta2, Zt,
                             (long)tid_flat());
}
template <typename R>
__global__ void __launch_bounds__(kBlock) kb_maxflux_omega(
    const Member<R> *mt, const int2 *bm, const R *__restrict__ u, const R *__restrict__ v, R *Huon, R *Hvom, const R *__restrict__ Hz,
    R *__restrict__ W, const R *__restrict__ z_w, int do_flux, int do_omega, R *__restrict__ zeta1, R *__restrict__ zeta2, const double *__restrict__ Zt) {
    SF_MEMBER(bm)
    maxflux_omega_body(g, O3(u), O3(v), O3(Huon), O3(Hvom), ON(Hz), O3(W), O3(z_w), do_flux,
                       do_omega, O2(zeta1), O2(zeta2), O2(Zt), (long)mb_.y * kBlock + threadIdx.x);
}

template <typename R>
__global__ void __launch_bounds__(kBlock) k_set_depth(Geo<R> g, const double *__restrict__ Zt, R *__restrict__ z_w, R *__restrict__ z_r,
                                                      R *__restrict__ Hz) {
    set_depth_body(g, Zt, z_w, z_r, Hz, (long)tid_flat());
}
template <typename R>
__global__ void __launch_bounds__(kBlock) kb_set_depth(const Member<R> *mt, const int2 *bm,
                                                       const double *__restrict__ Zt, R *__restrict__ z_w, R *__restrict__ z_r, R *__restrict__ Hz) {
    SF_MEMBER(bm)
    set_depth_body(g, O2(Zt), O3(z_w), ON(z_r), ON(Hz), (long)mb_.y * kBlock + threadIdx.x);
}

template <typename R>
__global__ void __launch_bounds__(128) k_step3d_uv(
    Geo<R> g, R *__restrict__ u, R *__restrict__ v, const R *__restrict__ ru, const R *__restrict__ rv, R *__restrict__ ubar_t1, R *__restrict__ vbar_t1, R *__restrict__ ubar_t2,
    R *__restrict__ vbar_t2, const R *__restrict__ Hz, const R *__restrict__ Akv, const R *__restrict__ z_r, const double *__restrict__ DU, const double *__restrict__ DV,
    const R *tmpU, const R *tmpV, R cff, R lambda, R Dt, int do_bc, R bcval) {
    step3d_uv_body(g, u, v, ru, rv, ubar_t1, vbar_t1, ubar_t2, vbar_t2, Hz, Akv, z_r, DU, DV,
                   tmpU, tmpV, cff, lambda, Dt, do_bc, bcval, (long)tid_flat());
}
template <typename R>
__global__ void __launch_bounds__(128) kb_step3d_uv(
    const Member<R> *mt, const int2 *bm, R *__restrict__ u, R *__restrict__ v, const R *__restrict__ ru, const R *__restrict__ rv, R *__restrict__ ubar_t1,
    R *__restrict__ vbar_t1, R *__restrict__ ubar_t2, R *__restrict__ vbar_t2, const R *__restrict__ Hz, const R *__restrict__ Akv, const R *__restrict__ z_r,
    const double *__restrict__ DU, const double *__restrict__ DV, const R *tmpU, const R *tmpV, R cff, R lambda, R Dt,
    int do_bc, R bcval) {
    SF_MEMBER(bm)
    step3d_uv_body(g, O3(u), O3(v), O3(ru), O3(rv), O2(ubar_t1), O2(vbar_t1), O2(ubar_t2),
                   O2(vbar_t2), ON(Hz), O3(Akv), ON(z_r), O2(DU), O2(DV), O3(tmpU), O3(tmpV), cff,
                   lambda, Dt, do_bc, bcval, (long)mb_.y * 128 + threadIdx.x);
}

template <typename R>
__global__ void __launch_bounds__(kPipeThreads, 5) k_step3d_uv_pipe(
    Geo<R> g, float *__restrict__ u, float *__restrict__ v, const float *__restrict__ ru, const float *__restrict__ rv, float *__restrict__ ubar_t1,
    float *__restrict__ vbar_t1, float *__restrict__ ubar_t2, float *__restrict__ vbar_t2, const float *__restrict__ Hz, const float *__restrict__ Akv,
    const float *__restrict__ z_r, const double *__restrict__ DU, const double *__restrict__ DV, const float *tmpU, const float *tmpV,
    float cff, float lambda, float Dt, int do_bc, float bcval, int stage) {
    // span staging (stage 1: bulk copies, 2: 16-byte cp.async) where the tile's spans (down to
    // p0 - I - r, up to p0 + 63) lie in the plane; per-element staging elsewhere
    const long p0 = (long)blockIdx.x * kPipeCols, rB = (4 - (g.I & 3)) & 3;
    const bool inside = p0 - g.I - rB >= 0 && p0 + kPipeCols <= g.s2;
    if (stage == 1 && inside)
        step3d_uv_pipe_body<R, 1>(g, u, v, ru, rv, ubar_t1, vbar_t1, ubar_t2, vbar_t2, Hz, Akv,
                                  z_r, DU, DV, tmpU, tmpV, cff, lambda, Dt, do_bc, bcval,
                                  (long)blockIdx.x);
    else if (stage == 2 && inside)
        step3d_uv_pipe_body<R, 2>(g, u, v, ru, rv, ubar_t1, vbar_t1, ubar_t2, vbar_t2, Hz, Akv,
                                  z_r, DU, DV, tmpU, tmpV, cff, lambda, Dt, do_bc, bcval,
                                  (long)blockIdx.x);
    else
        step3d_uv_pipe_body<R, 0>(g, u, v, ru, rv, ubar_t1, vbar_t1, ubar_t2, vbar_t2, Hz, Akv,
                                  z_r, DU, DV, tmpU, tmpV, cff, lambda, Dt, do_bc, bcval,
                                  (long)blockIdx.x);
}
template <typename R>
__global__ void __launch_bounds__(kPipeThreads, 5) kb_step3d_uv_pipe(
    const Member<R> *mt, const int2 *bm, float *__restrict__ u, float *__restrict__ v, const float *__restrict__ ru, const float *__restrict__ rv,
    float *__restrict__ ubar_t1, float *__restrict__ vbar_t1, float *__restrict__ ubar_t2, float *__restrict__ vbar_t2, const float *__restrict__ Hz,
    const float *__restrict__ Akv, const float *__restrict__ z_r, const double *__restrict__ DU, const double *__restrict__ DV, const float *tmpU,
    const float *tmpV, float cff, float lambda, float Dt, int do_bc, float bcval) {
    SF_MEMBER(bm)
    step3d_uv_pipe_body<R, 0>(g, O3(u), O3(v), O3(ru), O3(rv), O2(ubar_t1), O2(vbar_t1), O2(ubar_t2),
                        O2(vbar_t2), ON(Hz), O3(Akv), ON(z_r), O2(DU), O2(DV), O3(tmpU), O3(tmpV),
                        cff, lambda, Dt, do_bc, bcval, (long)mb_.y);
}
#undef ON
#undef O3
#undef O2
#undef SF_MEMBER

// ------------------------------------------------------------------------------------------
// Launchers
// ------------------------------------------------------------------------------------------
inline unsigned blocks_for(long n, int b) { return (unsigned)((n + b - 1) / b); }
template <typename R>
inline const Member<R> *mt(const sf_ctx *c) { return static_cast<const Member<R> *>(c->members); }

template <typename R>
Geo<R> Ops<R>::geo(const sf_ctx *c) {
    Geo<R> g;
    g.I = c->I;
    g.J = c->J;
    g.dI = make_fastdiv(c->I);
    g.dJ = make_fastdiv(c->J);
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
    g.err = c->dev_err;
    return g;
}

template <typename R>
cudaError_t Ops<R>::zeta_rhs(const sf_ctx *c, const R *zeta, const R *ubar, const R *vbar,
                             R *rzeta, int mode, double cff1, double *Zt, double *DU, double *DV,
                             const R *zeta_t0, R *zeta_t2, double Dt, cudaStream_t s) {
    if (c->nmem > 1) {
        return launch_dep(c, kb_zeta_rhs<R>, c->nbm_pt, kBlock, 0, s, mt<R>(c), c->bm_pt, zeta,
                          ubar, vbar, rzeta, mode, cff1, Zt, DU, DV, zeta_t0, zeta_t2, (R)Dt);
    }
    return launch_dep(c, k_zeta_rhs<R>, blocks_for((c->s2 + 3) / 4, kBlock), kBlock, 0, s, geo(c), zeta,
                      ubar, vbar, rzeta, mode, cff1, Zt, DU, DV, zeta_t0, zeta_t2, (R)Dt);
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
    if (c->nmem > 1) {
        return launch_dep(c, kb_momentum<R>, c->nbm_pt, kBlock, 0, s, mt<R>(c), c->bm_pt, rhs_u,
                          rhs_v, za, zb, (R)g, (R)w1, (R)weight, do_rhs, do_pred, (R)Dt, u_t1,
                          u_t2, v_t1, v_t2, z1, z2);
    }
    return launch_dep(c, k_momentum<R>, blocks_for((c->s2 + 3) / 4, kBlock), kBlock, 0, s, geo(c), rhs_u,
                      rhs_v, za, zb, (R)g, (R)w1, (R)weight, do_rhs, do_pred, (R)Dt, u_t1, u_t2,
                      v_t1, v_t2, z1, z2);
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
    if (c->nmem > 1) {
        return launch_dep(c, kb_corr_point<R>, c->nbm_pt, kBlock, 0, s, mt<R>(c), c->bm_pt, (R)Dt,
                          zeta_t2, rz0, rz1, rz2, ubar_t1, vbar_t1, rub0, rub1, vbar_t2);
    }
    return launch_dep(c, k_corr_point<R>, blocks_for((c->s2 + 3) / 4, kBlock), kBlock, 0, s, geo(c), (R)Dt,
                      zeta_t2, rz0, rz1, rz2, ubar_t1, vbar_t1, rub0, rub1, vbar_t2);
}
template <typename R>
cudaError_t Ops<R>::bc_apply(const sf_ctx *c, const BcProgram &p1, R *f1, const BcProgram &p2,
                             R *f2, double val, cudaStream_t s, const double *valp) {
    long n = (long)p1.n + p2.n;
    if (n == 0 && p1.nch == 0 && p2.nch == 0) return cudaSuccess;
    const long nw = 32L * ((long)p1.ngr + p2.ngr);   // one warp per chained group
    if (n < nw) n = nw;
    return launch_dep(c, k_bc_apply<R>, blocks_for(n > 0 ? n : 1, 256), 256, 0, s, p1, f1, p2, f2,
                      (R)val, valp);
}
template <typename R>
cudaError_t Ops<R>::rhs3d(const sf_ctx *c, const R *u, const R *v, const R *Huon, const R *Hvom,
                          const R *W, const R *Hz, R *ru, R *rv, cudaStream_t s) {
    // pair staging: even rows, fields on 2-element boundaries, 32-bit flat offsets
    const uintptr_t al = 2 * sizeof(R);
    const bool p2 = c->I % 2 == 0 && (long)c->I * c->J < (1L << 30) &&
                    (uintptr_t)u % al == 0 && (uintptr_t)v % al == 0 &&
                    (uintptr_t)Huon % al == 0 && (uintptr_t)Hvom % al == 0 &&
                    (uintptr_t)W % al == 0 && (uintptr_t)Hz % al == 0;
    // marching form (sf_ctx_tune SF_TUNE_RHS_MARCH): 1 = 4 warps x 4 rows (levels 2 .. N-4 in
    // the walk's branch-free form), 2 = 8 warps x 2 rows (the same, two blocks per SM), 3 = 8
    // warps x 2 rows (the general walk on every level, three blocks per SM)
    if (c->nmem == 1 && c->rhs_march > 0 && c->N >= 6 && (long)c->I * c->J < (1L << 30)) {
        // staging: 16-byte chunks (FP32, even rows, levels of a multiple of 4 elements, fields
        // on 16-byte boundaries; sf_ctx_tune SF_TUNE_RHS_CHUNKS), else pairs, else elements
        const bool c16 = sizeof(R) == 4 && c->rhs_chunks && c->I % 2 == 0 && c->s2 % 4 == 0 &&
                         (uintptr_t)u % 16 == 0 && (uintptr_t)v % 16 == 0 &&
                         (uintptr_t)Huon % 16 == 0 && (uintptr_t)Hvom % 16 == 0 &&
                         (uintptr_t)W % 16 == 0 && (uintptr_t)Hz % 16 == 0;
        auto march = [&](auto nw, auto rw, auto split, auto minb) {
            constexpr int NW = decltype(nw)::value, RW = decltype(rw)::value;
            constexpr bool SP = decltype(split)::value;
            auto go = [&](auto stg, auto sx) {
                constexpr int STG = decltype(stg)::value, SX = decltype(sx)::value;
                constexpr int MB = decltype(minb)::value > 0 ? decltype(minb)::value
                                                             : march_min_blocks<R, NW, RW, SX>();
                constexpr size_t smem = march_smem_bytes<R, NW, RW, SX>();
                static bool attr_set[64] = {};
                int dev = 0;
                cudaGetDevice(&dev);
                if (dev >= 0 && dev < 64 && !attr_set[dev]) {
                    cudaFuncSetAttribute(k_rhs3d_march<R, NW, RW, STG, SX, SP, MB>,
                                         cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
                    attr_set[dev] = true;
                }
                const dim3 grid((c->I + kMarchX - 1) / kMarchX, (c->J + NW * RW - 1) / (NW * RW));
                const dim3 block(32, NW);
                k_rhs3d_march<R, NW, RW, STG, SX, SP, MB><<<grid, block, smem, s>>>(
                    geo(c), u, v, Huon, Hvom, W, Hz, ru, rv);
            };
            using S0 = std::integral_constant<int, 0>;
            using S1 = std::integral_constant<int, 1>;
            using S2 = std::integral_constant<int, 2>;
            using X38 = std::integral_constant<int, 38>;
            using X44 = std::integral_constant<int, 44>;
            using X46 = std::integral_constant<int, 46>;
            if constexpr (sizeof(R) == 4) {
                if (c16) {
                    if (c->I % 4 == 0) go(S2{}, X44{});
                    else go(S2{}, X46{});
                    return;
                }
            }
            if (p2) go(S1{}, X38{});
            else go(S0{}, X38{});
        };
        using M0 = std::integral_constant<int, 0>;
        using M2 = std::integral_constant<int, 2>;
        using M4 = std::integral_constant<int, 4>;
        using M8 = std::integral_constant<int, 8>;
        using ST = std::true_type;
        using SF = std::false_type;
        switch (c->rhs_march) {
        case 1: march(M4{}, M4{}, ST{}, M0{}); break;
        case 2: march(M8{}, M2{}, ST{}, M2{}); break;
        default: march(M8{}, M2{}, SF{}, M0{}); break;
        }
        return cudaGetLastError();
    }
    // tile variant: 0 = 32 x 8, 1 = 32 x 4, 2 = 64 x 4, 3 = 32 x 16
    const int var = c->rhs_tile;
    auto run = [&](auto tx, auto ty) {
        constexpr int TX = decltype(tx)::value, TY = decltype(ty)::value;
        constexpr size_t smem = rhs_smem_bytes<R, TX, TY>();
        static bool attr_set[64] = {};
        int dev = 0;
        cudaGetDevice(&dev);
        if (dev >= 0 && dev < 64 && !attr_set[dev]) {
            cudaFuncSetAttribute(k_rhs3d<R, TX, TY, false>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)smem);
            cudaFuncSetAttribute(k_rhs3d<R, TX, TY, true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)smem);
            cudaFuncSetAttribute(kb_rhs3d<R, TX, TY>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)smem);
            attr_set[dev] = true;
        }
        if (c->nmem > 1) {
            kb_rhs3d<R, TX, TY><<<c->nbm_tile[var], dim3(TX, TY), smem, s>>>(
                mt<R>(c), c->bm_tile[var], var, u, v, Huon, Hvom, W, Hz, ru, rv);
        } else {
            const dim3 grid((c->I + TX - 1) / TX, (c->J + TY - 1) / TY), block(TX, TY);
            if (p2)
                k_rhs3d<R, TX, TY, true><<<grid, block, smem, s>>>(geo(c), u, v, Huon, Hvom, W, Hz, ru, rv);
            else
                k_rhs3d<R, TX, TY, false><<<grid, block, smem, s>>>(geo(c), u, v, Huon, Hvom, W, Hz, ru, rv);
        }
    };
    using I32 = std::integral_constant<int, 32>;
    using I8 = std::integral_constant<int, 8>;
    using I4 = std::integral_constant<int, 4>;
    using I64 = std::integral_constant<int, 64>;
    using I16 = std::integral_constant<int, 16>;
    if (var == 3) {
        run(I32{}, I16{});
    } else if (var == 1) {
        run(I32{}, I4{});
    } else if (var == 2) {
        run(I64{}, I4{});
    } else {
        run(I32{}, I8{});
    }
    return cudaGetLastError();
}
template <typename R>
cudaError_t Ops<R>::maxflux_omega(const sf_ctx *c, const R *u, const R *v, R *Huon, R *Hvom,
                                  const R *Hz, R *W, const R *z_w, int do_flux, int do_omega,
                                  R *zeta1, R *zeta2, const double *Zt, cudaStream_t s) {
    const size_t smem = do_omega ? sizeof(R) * (size_t)kBlock * (c->nmem > 1 ? c->maxN : c->N) : 0;
    static bool attr_set[64] = {};
    int dev = 0;
    cudaGetDevice(&dev);
    if (dev >= 0 && dev < 64 && !attr_set[dev]) {
        const int most = (int)(sizeof(R) * kBlock * kNMax);
        cudaFuncSetAttribute(k_maxflux_omega<R, -1>, cudaFuncAttributeMaxDynamicSharedMemorySize, most);
        cudaFuncSetAttribute(k_maxflux_omega<R, 0>, cudaFuncAttributeMaxDynamicSharedMemorySize, most);
        cudaFuncSetAttribute(k_maxflux_omega<R, 4>, cudaFuncAttributeMaxDynamicSharedMemorySize, most);
        cudaFuncSetAttribute(k_maxflux_omega<R, 8>, cudaFuncAttributeMaxDynamicSharedMemorySize, most);
        cudaFuncSetAttribute(k_maxflux_omega<R, 5>, cudaFuncAttributeMaxDynamicSharedMemorySize, most);
        cudaFuncSetAttribute(kb_maxflux_omega<R>, cudaFuncAttributeMaxDynamicSharedMemorySize, most);
        attr_set[dev] = true;
    }
    if (c->nmem > 1) {
        kb_maxflux_omega<R><<<c->nbm_pt, kBlock, smem, s>>>(mt<R>(c), c->bm_pt, u, v, Huon, Hvom, Hz,
                                                           W, z_w, do_flux, do_omega, zeta1, zeta2,
                                                           Zt);
        return cudaGetLastError();
    }
    // the chunked forms address with 32-bit element offsets
    const bool fits = (long)(c->N + 1) * c->s2 < (1L << 31);
    auto k = !do_flux ? k_maxflux_omega<R, -1>
             : !fits ? k_maxflux_omega<R, 0>
             : c->mo_chunk == 8 ? k_maxflux_omega<R, 8>
             : c->mo_chunk == 5 ? k_maxflux_omega<R, 5>
             : c->mo_chunk == 4 ? k_maxflux_omega<R, 4> : k_maxflux_omega<R, 0>;
    k<<<blocks_for(c->s2, kBlock), kBlock, smem, s>>>(
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
    if (c->nmem > 1) {
        kb_set_depth<R><<<c->nbm_pt, kBlock, 0, s>>>(mt<R>(c), c->bm_pt, Zt, z_w, z_r, Hz);
        return cudaGetLastError();
    }
    k_set_depth<R><<<blocks_for(c->s2, kBlock), kBlock, 0, s>>>(geo(c), Zt, z_w, z_r, Hz);
    return cudaGetLastError();
}
template <typename R>
cudaError_t Ops<R>::step3d_uv(const sf_ctx *c, R *u, R *v, const R *ru, const R *rv, R *ubar_t1,
                              R *vbar_t1, R *ubar_t2, R *vbar_t2, const R *Hz, const R *Akv,
                              const R *z_r, const double *DU, const double *DV, const R *tmpU,
                              const R *tmpV, double cff, double lambda, double Dt, int do_bc,
                              double bcval, cudaStream_t s) {
    const int B = 128;
    if constexpr (std::is_same<R, float>::value) {
        static bool attr_set[64] = {};
        int dev = 0;
        cudaGetDevice(&dev);
        if (dev >= 0 && dev < 64 && !attr_set[dev]) {
            cudaError_t e = cudaFuncSetAttribute(k_step3d_uv_pipe<float>,
                                                 cudaFuncAttributeMaxDynamicSharedMemorySize,
                                                 (int)pipe_smem_bytes(kNMax));
            if (e == cudaSuccess)
                e = cudaFuncSetAttribute(kb_step3d_uv_pipe<float>,
                                         cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)pipe_smem_bytes(kNMax));
            if (e != cudaSuccess) return e;
            attr_set[dev] = true;
        }
        // the pipelined form addresses a field with 32-bit element offsets
        const bool fits = (long)(kNMax + 1) * c->s2 < (1L << 31);
        if (fits && c->nmem > 1) {
            kb_step3d_uv_pipe<float><<<c->nbm_pipe, kPipeThreads, pipe_smem_bytes(c->maxN), s>>>(
                mt<R>(c), c->bm_pipe, u, v, ru, rv, ubar_t1, vbar_t1, ubar_t2, vbar_t2, Hz, Akv, z_r,
                DU, DV, tmpU, tmpV, (float)cff, (float)lambda, (float)Dt, do_bc, (float)bcval);
            return cudaGetLastError();
        }
        if (fits) {
            // span staging needs 16-byte aligned spans: every level starts on a 16-byte
            // boundary (s2 a multiple of 4) in 16-byte aligned fields
            auto al = [](const void *q) { return q == nullptr || ((uintptr_t)q & 15) == 0; };
            const bool aligned = c->s2 % 4 == 0 && al(u) && al(v) && al(ru) && al(rv) && al(Hz) &&
                                 al(Akv) && al(z_r) && al(tmpU) && al(tmpV);
            const int stage = !aligned ? 0 : c->use_bulk ? 1 : c->s3_vec ? 2 : 0;
            k_step3d_uv_pipe<float><<<blocks_for(c->s2, kPipeCols), kPipeThreads,
                                      pipe_smem_bytes(c->N), s>>>(
                geo(c), u, v, ru, rv, ubar_t1, vbar_t1, ubar_t2, vbar_t2, Hz, Akv, z_r, DU, DV,
                tmpU, tmpV, (float)cff, (float)lambda, (float)Dt, do_bc, (float)bcval, stage);
            return cudaGetLastError();
        }
    }
    if (c->nmem > 1) {
        kb_step3d_uv<R><<<c->nbm_128, B, 0, s>>>(mt<R>(c), c->bm_128, u, v, ru, rv, ubar_t1, vbar_t1,
                                                ubar_t2, vbar_t2, Hz, Akv, z_r, DU, DV, tmpU, tmpV,
                                                (R)cff, (R)lambda, (R)Dt, do_bc, (R)bcval);
        return cudaGetLastError();
    }
    k_step3d_uv<R><<<blocks_for(c->s2, B), B, 0, s>>>(
        geo(c), u, v, ru, rv, ubar_t1, vbar_t1, ubar_t2, vbar_t2, Hz, Akv, z_r, DU, DV, tmpU, tmpV,
        (R)cff, (R)lambda, (R)Dt, do_bc, (R)bcval);
    return cudaGetLastError();
}
template <typename R>
__global__ void __launch_bounds__(kBlock) kb_lateral_uv_bc(const Member<R> *mt, const int2 *bm,
                                                           R *__restrict__ u, R *__restrict__ v,
                                                           R bcval) {
    const int2 mb = bm[blockIdx.x];
    const Member<R> &M = mt[mb.x];
    lateral_uv_bc_at(M.g, u + M.off3, v + M.off3, bcval, (long)mb.y * kBlock + threadIdx.x);
}
template <typename R>
cudaError_t Ops<R>::lateral_uv_bc(const sf_ctx *c, R *u, R *v, double val, cudaStream_t s) {
    if (c->nmem > 1)
        kb_lateral_uv_bc<R><<<c->nbm_pt, kBlock, 0, s>>>(mt<R>(c), c->bm_pt, u, v, (R)val);
    else
        k_lateral_uv_bc<R><<<blocks_for(c->s2, kBlock), kBlock, 0, s>>>(geo(c), u, v, (R)val);
    return cudaGetLastError();
}

template <typename R>
cudaError_t Ops<R>::gls_corrector(const sf_ctx *c, const sf_gls_params &P, double dt, const R *u,
                                  const R *v, const R *z_r, const R *Hz, const R *bvf,
                                  const R *sustr, const R *svstr, R *tke, R *gls, R *Akv, R *Akt,
                                  R *Akk, R *Akp, R *Lscale, const R *tkn0,
                                  const R *gln0, const uint8_t *sel, const int *list,
                                  const int *count, cudaStream_t s) {
    k_gls_corrector<R><<<blocks_for(c->s2, 128), 128, 0, s>>>(
        geo(c), P, (R)dt, u, v, z_r, Hz, bvf, sustr, svstr, tke, gls, Akv, Akt, Akk, Akp, Lscale,
        tkn0, gln0, sel, list, count);
    return cudaGetLastError();
}


// Buoyancy frequency squared at every W level for a linear equation of state in temperature
// alone, with T(z) = T0 + dT exp(z / zscale): N^2 = g alpha dT/dz.  The stratification of the
// analytic basins (their tracers are not stepped, so N^2 follows z_w).
template <typename R>
__global__ void k_analytic_bvf(long n, const R *__restrict__ z_w, double dT, double zscale,
                               double galpha, R *__restrict__ bvf) {
    const long e = tid_flat();
    if (e >= n) return;
    bvf[e] = (R)(galpha * (dT / zscale) * exp((double)z_w[e] / zscale));
}
template <typename R>
cudaError_t Ops<R>::analytic_bvf(const sf_ctx *c, const R *z_w, double dT, double zscale,
                                 double galpha, R *bvf, cudaStream_t s) {
    const long n = (long)(c->N + 1) * c->s2;
    k_analytic_bvf<R><<<blocks_for(n, kBlock), kBlock, 0, s>>>(n, z_w, dT, zscale, galpha, bvf);
    return cudaGetLastError();
}

}  // namespace sf

#include "sf_roms.cuh"
