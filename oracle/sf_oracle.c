/*
 * sf_oracle.c -- CPU restatement of the reference's time-step kernels (TEST INFRASTRUCTURE).
 *
 * This file is the oracle: plain C, FP64, one loop iteration per CUDA thread of the
 * reference launch, evaluating every expression in the same order as the reference's
 * expression templates (modules/mod_cppkernels.h:185-1490) evaluate it, so that with
 * floating-point contraction disabled (-ffp-contract=off) its results are bit-identical
 * to the reference kernels compiled for the host (oracle/_ref, see build_ref.py).
 * Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg use it; the
 * product never links it.
 *
 * Conventions (the reference's): every field is a flat C-order array, 2D fields are
 * (M+1) x (L+1) = J rows of I points (I = L+1 is the xi stride), 3D fields are levels of
 * s2 = I*J points.  A "thread" p is a flat 2D index; i = p % I, j = p / I.  Neighbour reads
 * use flat offsets (p-1, p+I, ...) exactly like the reference, so at the first/last column
 * they wrap into the neighbouring row.  Reads that leave an array (possible only at the
 * boundary ring, e.g. rhs_kernels.cpp:86-130 has no guard) are the caller's business: the
 * Python harness allocates zero guards around every array, which is what makes those
 * reference reads deterministic.
 */
#include <math.h>
#include <stddef.h>

typedef struct {
    int I, J, N;               /* xi points (L+1), eta points (M+1), levels */
    const double *on_u, *om_v, *pn, *pm;   /* device globals of mod_cppkernels.h:40-41 */
} orc_grid;

#define S2(g) ((long)(g)->I * (long)(g)->J)

/* Node predicates, mod_cppkernels.h:101-152. */
static int is_inner(const orc_grid *g, long p) {
    if (p >= S2(g)) return 0;
    int i = (int)(p % g->I), j = (int)(p / g->I);
    return (i > 1) && (i < g->I - 2) && (j > 1) && (j < g->J - 2);
}
static int is_rnode(const orc_grid *g, long p) {
    if (p >= S2(g)) return 0;
    int i = (int)(p % g->I), j = (int)(p / g->I);
    return (i > 0) && (i < g->I) && (j > 0) && (j < g->J);
}
static int is_unode(const orc_grid *g, long p) {
    if (p >= S2(g)) return 0;
    int i = (int)(p % g->I), j = (int)(p / g->I);
    return (i > 1) && (i < g->I) && (j > 0) && (j < g->J);
}
static int is_vnode(const orc_grid *g, long p) {
    if (p >= S2(g)) return 0;
    int i = (int)(p % g->I), j = (int)(p / g->I);
    return (i > 0) && (i < g->I) && (j > 1) && (j < g->J - 1);
}
/* Interior rho points of the 2D kernels: mod_cppkernels.cpp:20,55,89. */
static int is_rint(const orc_grid *g, long p) {
    if (p >= S2(g)) return 0;
    int i = (int)(p % g->I), j = (int)(p / g->I);
    return !(i == 0 || i == g->I - 1 || j == 0 || j == g->J - 1);
}

/* ------------------------------------------------------------------------------------ */
/* 2D barotropic kernels, modules/mod_cppkernels.cpp                                     */
/* ------------------------------------------------------------------------------------ */

/* computeZetaRHS, mod_cppkernels.cpp:81-128. */
void orc_zeta_rhs(const orc_grid *g, const double *zeta, const double *h, const double *ubar,
                  const double *vbar, double *DU_avg1, double *DV_avg1, double *Zt_avg1,
                  int isPredictor, const double *weight1, int iif, double *res) {
    const long I = g->I, s2 = S2(g);
    for (long p = 0; p < s2; ++p) {
        if (!is_rint(g, p)) continue;
#define D_(q) (zeta[q] + h[q])
#define DU_(q) (ubar[q] * ((D_(q) + D_((q) - 1)) * 0.5))
#define DV_(q) (vbar[q] * ((D_(q) + D_((q) - I)) * 0.5))
        res[p] = (((DU_(p + 1) * g->on_u[p + 1] - DU_(p) * g->on_u[p]) +
                   (DV_(p + I) * g->om_v[p + I] - DV_(p) * g->om_v[p])) * g->pm[p]) * g->pn[p];
        if (!isPredictor) {
            const double cff1 = weight1[iif - 1];
            Zt_avg1[p] = Zt_avg1[p] + cff1 * zeta[p];
            DU_avg1[p] = DU_avg1[p] + (cff1 * DU_(p)) * g->on_u[p];
            DV_avg1[p] = DV_avg1[p] + (cff1 * DV_(p)) * g->om_v[p];
        }
#undef DU_
#undef DV_
#undef D_
    }
}

/* computeZetaPred, mod_cppkernels.cpp:134-150 (the reference's leapfrog uses Dt, :146). */
void orc_zeta_pred(const orc_grid *g, double Dt, const double *zeta_t0, double *zeta_t2,
                   const double *rzeta_t1) {
    const long I = g->I, s2 = S2(g);
    for (long p = 0; p < s2; ++p) {
        if ((p % I) == 0 || (p / I) == 0) continue;
        zeta_t2[p] = zeta_t0[p] + Dt * rzeta_t1[p];
    }
}

/* computeMomentumRHSPred (:13-42) and computeMomentumRHSCorr (:46-77):
 * gzeta = (1-w)*za + w*zb, rhs = g*on_u*(RtoU(h)*Dxi(gzeta) + 0.5*Dxi(gzeta^2)). */
void orc_momentum_rhs(const orc_grid *g, const double *h, double *rhs_ubar, double *rhs_vbar,
                      const double *za, const double *zb, double grav, double weight) {
    const long I = g->I, s2 = S2(g);
    const double w1 = 1 - weight;
    for (long p = 0; p < s2; ++p) {
        if (!is_rint(g, p)) continue;
#define GZ(q) (w1 * za[q] + weight * zb[q])
#define GZ2(q) (GZ(q) * GZ(q))
        rhs_ubar[p] = (grav * g->on_u[p]) *
                      (((h[p] + h[p - 1]) * 0.5) * (GZ(p) - GZ(p - 1)) + 0.5 * (GZ2(p) - GZ2(p - 1)));
        rhs_vbar[p] = (grav * g->om_v[p]) *
                      (((h[p] + h[p - I]) * 0.5) * (GZ(p) - GZ(p - I)) + 0.5 * (GZ2(p) - GZ2(p - I)));
#undef GZ2
#undef GZ
    }
}

/* computeMomentumPred, mod_cppkernels.cpp:156-186.  Its guard tests the flat index against
 * szJ (the number of rows), not szI (:162). */
void orc_momentum_pred(const orc_grid *g, double Dt, const double *u_t1, double *u_t2,
                       const double *v_t1, double *v_t2, const double *rhsu, const double *rhsv,
                       const double *h, const double *zeta_t1, const double *zeta_t2) {
    const long I = g->I, J = g->J, s2 = S2(g);
    for (long p = 0; p < s2; ++p) {
        if ((p % J) == 0 || (p / J) == 0) continue;
        const double D1p = zeta_t1[p] + h[p], D2p = zeta_t2[p] + h[p];
        const double D1U = (D1p + (zeta_t1[p - 1] + h[p - 1])) * 0.5;
        const double D1V = (D1p + (zeta_t1[p - I] + h[p - I])) * 0.5;
        const double D2U = (D2p + (zeta_t2[p - 1] + h[p - 1])) * 0.5;
        const double D2V = (D2p + (zeta_t2[p - I] + h[p - I])) * 0.5;
        u_t2[p] = (u_t1[p] * D1U + ((Dt * rhsu[p]) * g->pm[p]) * g->pn[p]) / D2U;
        v_t2[p] = (v_t1[p] * D1V + ((Dt * rhsv[p]) * g->pm[p]) * g->pn[p]) / D2V;
    }
}

/* AdamsMoultonCorr3rd, mod_cppkernels.cpp:191-209: v_t2 += Dt*(5/12 r2 + 8/12 r1 - 1/12 r0).
 * The reference also launches this kernel for the momentum corrector, because
 * modules/mod_operators.py:146 binds AdamsMoultonCorr3rd2 to it; nonlinear/step2d.py:120 then
 * passes (Dt, ubar_t1, vbar_t1, rubar_t0, rubar_t1, ...) of which the kernel reads five. */
void orc_am3(const orc_grid *g, double Dt, double *v_t2, const double *r0, const double *r1,
             const double *r2) {
    const long s2 = S2(g);
    const double A2 = 5.0 / 12.0, A1 = 8.0 / 12.0, A0 = -1.0 / 12.0;
    for (long p = 0; p < s2; ++p)
        v_t2[p] = v_t2[p] + Dt * ((A2 * r2[p] + A1 * r1[p]) + A0 * r0[p]);
}

/* AdamsMoultonCorr3rd2 as written (mod_cppkernels.cpp:214-250); never launched by the
 * reference (see orc_am3), kept for completeness of the kernel set. */
void orc_am3_momentum(const orc_grid *g, double Dt, double *u_t2, double *v_t2,
                      const double *ru0, const double *ru1, const double *ru2,
                      const double *rv0, const double *rv1, const double *rv2,
                      const double *h, const double *zeta_t1, const double *zeta_t2) {
    const long I = g->I, s2 = S2(g);
    const double A2 = 5.0 / 12.0, A1 = 8.0 / 12.0, A0 = -1.0 / 12.0;
    for (long p = 0; p < s2; ++p) {
        const double D1p = zeta_t1[p] + h[p], D2p = zeta_t2[p] + h[p];
        const double D1U = (D1p + (zeta_t1[p - 1] + h[p - 1])) * 0.5;
        const double D1V = (D1p + (zeta_t1[p - I] + h[p - I])) * 0.5;
        const double D2U = (D2p + (zeta_t2[p - 1] + h[p - 1])) * 0.5;
        const double D2V = (D2p + (zeta_t2[p - I] + h[p - I])) * 0.5;
        const double pmn_u = (Dt * g->pm[p]) * g->pn[p];
        u_t2[p] = (u_t2[p] * D1U + pmn_u * ((A2 * ru2[p] + A1 * ru1[p]) + A0 * ru0[p])) / D2U;
        v_t2[p] = (v_t2[p] * D1V + pmn_u * ((A2 * rv2[p] + A1 * rv1[p]) + A0 * rv0[p])) / D2V;
    }
}

/* setBC / copyBC, modules/mod_BC.c:6-23, executed in thread order. */
void orc_set_bc(double *var, const int *idx, long n, double val) {
    for (long k = 0; k < n; ++k) var[idx[k]] = val;
}
void orc_copy_bc(double *var, const int *idx1, const int *idx2, long n) {
    for (long k = 0; k < n; ++k) var[idx1[k]] = var[idx2[k]];
}

/* ------------------------------------------------------------------------------------ */
/* 3D right-hand side, nonlinear/rhs_kernels.cpp                                          */
/* ------------------------------------------------------------------------------------ */

/* addCoriolis, rhs_kernels.cpp:7-35. */
void orc_add_coriolis(const orc_grid *g, const double *fomn, const double *u, const double *v,
                      double *ru, double *rv, const double *Hz) {
    const long I = g->I, s2 = S2(g);
    for (long p = 0; p < s2; ++p) {
        if (!is_rnode(g, p)) continue;
        for (int K = 0; K < g->N; ++K) {
            const long o = (long)K * s2;
#define CFF(q) (Hz[o + (q)] * fomn[q])
#define UF(q) (CFF(q) * ((v[o + (q)] + v[o + (q) + I]) * 0.5))
#define VF(q) (CFF(q) * ((u[o + (q)] + u[o + (q) + 1]) * 0.5))
            ru[o + p] = ru[o + p] + (UF(p) + UF(p - 1)) * 0.5;
            rv[o + p] = rv[o + p] - (VF(p) + VF(p - I)) * 0.5;
#undef VF
#undef UF
#undef CFF
        }
    }
}

/* horizontalAdvection, rhs_kernels.cpp:71-132 (Gadv = -0.5).  `nthreads` is the size of the
 * reference launch (grsz*GPUMUL blocks of bksz/GPUMUL threads, nonlinear/rhs.py:62): its
 * threads with p >= s2 store 0 into ru/rv at flat offset p (level 1), after the in-range
 * threads in thread order. */
void orc_horizontal_advection(const orc_grid *g, const double *u, const double *v,
                              const double *Hu, const double *Hv, double *ru, double *rv,
                              long nthreads) {
    const long I = g->I, s2 = S2(g);
    const double Gadv = -0.5;
    for (long p = 0; p < s2; ++p) {
        for (int K = 0; K < g->N; ++K) {
            const double *U = u + (long)K * s2, *V = v + (long)K * s2;
            const double *HU = Hu + (long)K * s2, *HV = Hv + (long)K * s2;
#define UR(q) ((U[q] + U[(q) + 1]) * 0.5)
#define UP(q) ((U[q] + U[(q) - 1]) * 0.5)
#define VR(q) ((V[q] + V[(q) + I]) * 0.5)
#define VP(q) ((V[q] + V[(q) - I]) * 0.5)
#define HUR(q) ((HU[q] + HU[(q) + 1]) * 0.5)
#define HUP(q) ((HU[q] + HU[(q) - 1]) * 0.5)
#define HVP(q) ((HV[q] + HV[(q) - I]) * 0.5)
#define HVR(q) ((HV[q] + HV[(q) + I]) * 0.5)
#define DXX(X, q) (((X)[(q) - 1] - 2.0 * (X)[q]) + (X)[(q) + 1])
#define DEE(X, q) (((X)[(q) - I] - 2.0 * (X)[q]) + (X)[(q) + I])
#define UXXR(q) ((UR(q) + UR((q) + 1) >= 0) ? DXX(U, q) : DXX(U, (q) + 1))
#define UEEP(q) ((HVP(q) + HVP((q) - I) >= 0) ? DEE(U, q) : DEE(U, (q) - I))
#define HUXXR(q) ((DXX(HU, q) + DXX(HU, (q) + 1)) * 0.5)
#define HUEEP(q) ((DEE(HU, q) + DEE(HU, (q) - 1)) * 0.5)
#define HVXXP(q) ((DXX(HV, q) + DXX(HV, (q) - I)) * 0.5)
#define HVEER(q) ((DEE(HV, q) + DEE(HV, (q) + I)) * 0.5)
#define UFXR(q) (UR(q) + (Gadv * UXXR(q)) * (HUR(q) + Gadv * HUXXR(q)))
#define UFEP(q) (UP(q) + (Gadv * UEEP(q)) * (HVP(q) + Gadv * HVXXP(q)))
#define VFXP(q) (VP(q) + (Gadv * UEEP(q)) * (HUP(q) + Gadv * HUEEP(q)))
#define VFER(q) (VR(q) + (Gadv * UXXR(q)) * (HVR(q) + Gadv * HVEER(q)))
            const long o = (long)K * s2 + p;
            ru[o] = ru[o] - ((UFXR(p) - UFXR(p - 1)) + (UFEP(p) - UFEP(p - I)));
            rv[o] = rv[o] - ((VFXP(p) - VFXP(p - 1)) + (VFER(p) - VFER(p - I)));
        }
    }
    for (long p = s2; p < nthreads; ++p) {
        ru[p] = 0.0;
        rv[p] = 0.0;
    }
}

/* verticalAdvection, rhs_kernels.cpp:136-196. */
void orc_vertical_advection(const orc_grid *g, const double *u, const double *v, const double *W,
                            double *ru, double *rv, const int *BC) {
    const long I = g->I, s2 = S2(g);
    const int N = g->N;
    const double c9 = 9.0 / 16.0, c1 = 1.0 / 16.0;
    for (long p = 0; p < s2; ++p) {
        if (BC[p] >= 0) continue;
        if (!is_inner(g, p)) continue;
#define AT(X, k) ((X)[(long)(k) * s2 + p])
#define W_(k, q) (W[(long)(k) * s2 + (q)])
#define U4(X, k) (c9 * (AT(X, k) + AT(X, (k) + 1)) - c1 * (AT(X, (k) - 1) + AT(X, (k) + 2)))
#define WU4(k) (c9 * (W_(k, p) + W_(k, p + 1)) - c1 * (W_(k, p - 1) + W_(k, p + 2)))
#define WV4(k) (c9 * (W_(k, p) + W_(k, p + I)) - c1 * (W_(k, p - I) + W_(k, p + 2 * I)))
#define FU(k) (U4(u, k) * WU4(k))
#define FV(k) (U4(v, k) * WV4(k))
        for (int K = 2; K < N - 2; ++K) {
            AT(ru, K) = AT(ru, K) - (FU(K + 1) - FU(K));
            AT(rv, K) = AT(rv, K) - (FV(K + 1) - FV(K));
        }
        AT(rv, 1) -= c9 * (FV(1) + FV(2)) - c1 * (FV(1) + FV(3));
        const double uuu = (c9 * (AT(u, 0) + AT(u, 1)) - c1 * (0 + AT(u, 2))) * WU4(1);
        const double uuu2 = (c9 * (0 + AT(u, 0)) - c1 * (0 + AT(u, 1))) * WU4(0);
        AT(ru, 1) = AT(ru, 1) - (FU(2) - uuu);
        AT(ru, 0) = AT(ru, 0) - (uuu - uuu2);
        /* ru[N-2] -= ... and rv[N-2] -= ... (:179-180) are overwritten at :189-190 before
         * anything reads them, so they are not evaluated here. */
        AT(rv, 0) = AT(rv, 1);
        AT(ru, N - 2) = AT(ru, N - 3);
        AT(rv, N - 2) = AT(rv, N - 3);
        AT(ru, N - 1) = AT(ru, N - 2);
        AT(rv, N - 1) = AT(rv, N - 2);
        AT(ru, N) = AT(ru, N - 2);
        AT(rv, N) = AT(rv, N - 2);
#undef FV
#undef FU
#undef WV4
#undef WU4
#undef U4
#undef W_
#undef AT
    }
}

/* ------------------------------------------------------------------------------------ */
/* 3D step kernels, nonlinear/step3D_uv.kernels.cpp                                       */
/* ------------------------------------------------------------------------------------ */

/* set_maxflux, step3D_uv.kernels.cpp:372-405. */
void orc_set_maxflux(const orc_grid *g, const double *u, const double *v, double *Huon,
                     double *Hvom, const double *Hz) {
    const long I = g->I, s2 = S2(g);
    for (long p = 0; p < s2; ++p) {
        if (is_unode(g, p))
            for (int K = 0; K < g->N; ++K) {
                const long o = (long)K * s2 + p;
                Huon[o] = (((Hz[o] + Hz[o - 1]) * 0.5) * u[o]) * g->on_u[p];
            }
        if (is_vnode(g, p))
            for (int K = 0; K < g->N; ++K) {
                const long o = (long)K * s2 + p;
                Hvom[o] = (((Hz[o] + Hz[o - I]) * 0.5) * v[o]) * g->om_v[p];
            }
    }
}

/* omega, step3D_uv.kernels.cpp:62-165. */
void orc_omega(const orc_grid *g, double *W, const double *Huon, const double *Hvom,
               const double *z_w, const int *BC) {
    const long I = g->I, s2 = S2(g);
    const int N = g->N;
    for (long p = 0; p < s2; ++p) {
        if (BC[p] >= 0) continue;
        W[p] = 0.0;
        for (int K = 1; K < N; ++K) {
            const long o = (long)K * s2 + p;
            W[o] = W[o - s2] - ((Huon[o + 1] - Huon[o]) + (Hvom[o + I] - Hvom[o]));
        }
        const double zbed = z_w[p];
        const double h = z_w[(long)(N - 1) * s2 + p] - zbed;
        const double Ws = W[(long)(N - 1) * s2 + p];
        for (int K = N - 1; K > 0; --K) {
            const long o = (long)K * s2 + p;
            W[o] = W[o] - (Ws * (z_w[o] - zbed)) / h;
        }
        W[(long)N * s2 + p] = 0.0;
    }
}

/* set_zeta, step3D_uv.kernels.cpp:294-310. */
void orc_set_zeta(const orc_grid *g, double *zeta1, double *zeta2, const double *Zt_avg1) {
    const long s2 = S2(g);
    for (long p = 0; p < s2; ++p) {
        if (!is_rnode(g, p)) continue;
        zeta2[p] = Zt_avg1[p];
        zeta1[p] = Zt_avg1[p];
    }
}

/* set_depth, step3D_uv.kernels.cpp:225-291. */
void orc_set_depth(const orc_grid *g, int Vtransform, const double *Zt, double *z_w, double *z_r,
                   const double *h, double hc, double *Hz, const double *sc_r, const double *sc_w,
                   const double *Cs_r, const double *Cs_w) {
    const long s2 = S2(g);
    const int N = g->N;
    for (long p = 0; p < s2; ++p) {
        if (Vtransform == 1) {
            for (int K = 0; K < N; ++K) {
                const double z_r0 = hc * (sc_r[K] - Cs_r[K]) + Cs_r[K] * h[p];
                const double z_w0 = hc * (sc_w[K] - Cs_w[K]) + Cs_w[K] * h[p];
                z_w[(long)K * s2 + p] = z_w0 + Zt[p] * (1.0 + z_w0 / h[p]);
                z_r[(long)K * s2 + p] = z_r0 + Zt[p] * (1.0 + z_r0 / h[p]);
            }
            z_w[(long)N * s2 + p] = Zt[p];
        } else if (Vtransform == 2) {
            z_w[(long)N * s2 + p] = 0.0;
            for (int K = 0; K < N; ++K) {
                const double cff2_r = (hc * sc_r[K] + Cs_r[K] * h[p]) / (hc + h[p]);
                const double cff2_w = (hc * sc_w[K] + Cs_w[K] * h[p]) / (hc + h[p]);
                z_w[(long)K * s2 + p] = Zt[p] + (Zt[p] + h[p]) * cff2_w;
                z_r[(long)K * s2 + p] = Zt[p] + (Zt[p] + h[p]) * cff2_r;
            }
            z_w[(long)N * s2 + p] = Zt[p];
        }
        for (int K = 0; K < N; ++K)
            Hz[(long)K * s2 + p] = z_w[(long)(K + 1) * s2 + p] - z_w[(long)K * s2 + p];
    }
}

/* setLateralUVBCs, step3D_uv.kernels.cpp:314-368, with val = 0.05*sin(t*0.0002) (:338-339). */
void orc_lateral_uv_bc(const orc_grid *g, double t, double *u, double *v, const int *vIdx2,
                       const int *uType, const int *vType) {
    const long s2 = S2(g);
    const int N = g->N;
    const int bcClosed = 1 << 4, bcClamped = 1 << 3, bcGradient = 1 << 6;
    for (long p = 0; p < s2; ++p) {
        const int ut = uType[p], vt = vType[p];
        if (ut <= 0 && vt <= 0) continue;
        if (ut > 0) {
            if ((ut & bcClosed) != 0) {
            } else if ((ut & bcClamped) != 0) {
                double omega = 0.0002;
                double val = 0.05 * sin(t * omega);
                for (int k = 0; k < N; ++k) u[p + (long)k * s2] = val;
            }
        }
        if (vt > 0) {
            if ((vt & bcClosed) != 0) {
                for (int k = 0; k < N; ++k) v[p + (long)k * s2] = 0.0;
            } else if ((vt & bcClamped) != 0) {
                for (int k = 0; k < N; ++k) v[p + (long)k * s2] = 0.0;
            } else if ((vt & bcGradient) != 0) {
                for (int k = 0; k < N; ++k) v[p + (long)k * s2] = v[vIdx2[p + (long)k * s2]];
            }
        }
    }
}

/* step3d_UV and its helpers, step3D_uv.kernels.cpp:408-707.  SD/D/RHS are the reference's
 * tridiagonal scratch (VerticalVelEq, mod_cppkernels.h:89-96), each (N+1)*s2. */
static void orc_build_matrix(const orc_grid *g, long p, int isV, double cff, double Dt,
                             double lambda, double *FC, double *BCd, double *RHS,
                             const double *Hz, const double *Akv, const double *z_r,
                             const double *u, const double *ru) {
    const long s2 = S2(g), d = isV ? g->I : 1;
    const int N = g->N;
    const double pmU = (g->pm[p] + g->pm[p - d]) * 0.5, pnU = (g->pn[p] + g->pn[p - d]) * 0.5;
    const double cdt = cff * Dt;
#define HZU(k) ((Hz[(long)(k) * s2 + p] + Hz[(long)(k) * s2 + p - d]) * 0.5)
#define AKU(k) ((Akv[(long)(k) * s2 + p] + Akv[(long)(k) * s2 + p - d]) * 0.5)
#define DZ(k) (((z_r[(long)(k) * s2 + p] - z_r[(long)((k) - 1) * s2 + p]) + \
                (z_r[(long)(k) * s2 + p - d] - z_r[(long)((k) - 1) * s2 + p - d])) * 0.5)
#define X(A, k) ((A)[(long)(k) * s2 + p])
    const double c = -lambda * Dt;
    X(FC, N - 1) = 0.0;
    X(BCd, 0) = HZU(0);
    X(RHS, 0) = 0.0;
    for (int K = 0; K < N - 1; ++K) X(FC, K) = (c * AKU(K)) / DZ(K + 1);
    for (int K = 1; K < N; ++K) {
        X(RHS, K) = HZU(K) * (X(u, K) + (cdt * (pmU * pnU)) * X(ru, K));
        X(BCd, K) = (HZU(K) - X(FC, K)) - X(FC, K - 1);
    }
    X(BCd, N - 1) = HZU(N - 1) - X(FC, N - 2);
    X(FC, 0) = (c * AKU(0)) / DZ(1);
    X(BCd, 0) = HZU(0) - 2.0 * X(FC, 0);
#undef X
#undef DZ
#undef AKU
#undef HZU
}

static void orc_solve_tri(const orc_grid *g, long p, double *FC, double *BCd, double *RHS,
                          double *u) {
    const long s2 = S2(g);
    const int N = g->N;
#define X(A, k) ((A)[(long)(k) * s2 + p])
    for (int k = 1; k < N; ++k) {
        const double w = X(FC, k - 1) / X(BCd, k - 1);
        X(BCd, k) = X(BCd, k) - w * X(FC, k - 1);
        X(RHS, k) = X(RHS, k) - w * X(RHS, k - 1);
    }
    X(u, N - 1) = X(RHS, N - 1) / X(BCd, N - 1);
    for (int k = N - 2; k >= 0; --k) X(u, k) = (X(RHS, k) - X(FC, k) * X(u, k + 1)) / X(BCd, k);
#undef X
}

static void orc_correct_mean(const orc_grid *g, long p, int isV, double *u, const double *Hz,
                             const double *DU_avg1, const double *on, const double *tmp) {
    const long s2 = S2(g), d = isV ? g->I : 1;
    double H = 0.0, Hu = 0.0;
    for (int K = 0; K < g->N; ++K) {
        const long o = (long)K * s2 + p;
        const double hzu = (Hz[o] + Hz[o - d]) * 0.5;
        H += hzu;
        Hu += tmp[o] * hzu;
    }
    const double udiff = (Hu - DU_avg1[p] / on[p]) / H;
    for (int K = 0; K < g->N; ++K) u[(long)K * s2 + p] = u[(long)K * s2 + p] - udiff;
}

void orc_step3d_uv(const orc_grid *g, double *u, double *v, const double *ru, const double *rv,
                   double *ubar_t1, double *vbar_t1, double *ubar_t2, double *vbar_t2,
                   const double *Hz, const double *Akv, const double *z_r, const double *DU_avg1,
                   const double *DV_avg1, const double *tmpU, const double *tmpV, int iic,
                   int ntfirst, double lambda, double Dt, double *SD, double *Dg, double *RHS) {
    const long I = g->I, s2 = S2(g);
    const int N = g->N;
    double cff;
    if (iic == ntfirst) cff = 1.0;
    else if (iic == ntfirst + 1) cff = 3.0 / 2.0;
    else cff = 23.0 / 12.0;
    for (long p = 0; p < s2; ++p) {
        const int un = is_unode(g, p), vn = is_vnode(g, p);
        if (un) {
            orc_build_matrix(g, p, 0, cff, Dt, lambda, SD, Dg, RHS, Hz, Akv, z_r, tmpU, ru);
            orc_solve_tri(g, p, SD, Dg, RHS, u);
            orc_correct_mean(g, p, 0, u, Hz, DU_avg1, g->on_u, tmpU);
        }
        if (vn) orc_build_matrix(g, p, 1, cff, Dt, lambda, SD, Dg, RHS, Hz, Akv, z_r, tmpV, rv);
        if (un) orc_solve_tri(g, p, SD, Dg, RHS, v);      /* gated by isUNode, :525 */
        if (vn) orc_correct_mean(g, p, 1, v, Hz, DV_avg1, g->om_v, tmpV);
        if (un) {   /* adjustBarotropicVelocity, :408-469 */
            double HU = 0.0, HV = 0.0, HuU = 0.0, HvV = 0.0;
            for (int K = 0; K < N; ++K) {
                const long o = (long)K * s2 + p;
                const double hzu = (Hz[o] + Hz[o - 1]) * 0.5, hzv = (Hz[o] + Hz[o - I]) * 0.5;
                HU += hzu;
                HV += hzv;
                HuU += hzu * u[o];
                HvV += hzv * v[o];
            }
            const double uUpdate = (HuU - DU_avg1[p] / g->on_u[p]) / HU;
            const double vUpdate = (HvV - DV_avg1[p] / g->om_v[p]) / HV;
            ubar_t2[p] = (DU_avg1[p] / g->on_u[p]) / HU + uUpdate;
            vbar_t2[p] = (DV_avg1[p] / g->om_v[p]) / HV + vUpdate;
            ubar_t1[p] = ubar_t2[p];
            vbar_t1[p] = vbar_t2[p];
        }
    }
}
