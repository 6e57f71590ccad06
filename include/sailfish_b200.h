/*
 * sailfish_b200.h -- C ABI of libsailfish_b200.so, the B200 (sm_100a) time-step library.
 *
 * Every entry point replaces one launch (or one Python routine) of the reference's time
 * step and takes the same arrays, as raw device pointers in the reference's layout:
 * flat C-order fields, 2D fields (M+1) x (L+1) (xi fastest), 3D fields N or N+1 levels of
 * (M+1)*(L+1) points.  The element type of every state and metric array is the context's
 * precision (SF_FP64: double, SF_FP32: float); the fast-time accumulators Zt_avg1, DU_avg1
 * and DV_avg1 are double in both precisions.
 *
 * The reference keeps the grid in device globals set once by `initialize<<<1,1>>>`
 * (modules/mod_cppkernels.h:154-171, bound per module in modules/mod_operators.py:31-45);
 * here a context (sf_ctx) holds the same information plus the boundary programs.
 *
 * Conventions: 0 = SF_OK, negative = error (sf_last_error() describes the last one on the
 * calling thread).  Calls are stream-ordered and asynchronous (no hidden synchronisation),
 * buffers are caller-owned, per-context tables are context-owned.  A context is
 * thread-compatible, not thread-safe.  No C++ exception crosses this boundary.
 */
#ifndef SAILFISH_B200_H
#define SAILFISH_B200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct sf_ctx sf_ctx;
typedef void *sf_stream; /* a cudaStream_t; NULL = legacy default stream */

enum sf_status {
    SF_OK = 0,
    SF_EINVAL = -1,       /* bad size, pointer or argument */
    SF_EDTYPE = -2,       /* unsupported precision */
    SF_ECUDA = -3,        /* CUDA runtime error */
    SF_ENONFINITE = -4,   /* non-finite value detected by a check */
    SF_ETIMEOUT = -5,     /* a bounded device wait gave up */
    SF_ENOMEM = -6,       /* device allocation failed */
    SF_EUNSUPPORTED = -7  /* configuration the reference cannot run either */
};

enum sf_precision { SF_FP64 = 0, SF_FP32 = 1 };

/* Grid, vertical coordinate and boundary description; all pointers are HOST pointers and
 * are copied into the context by sf_ctx_create. */
typedef struct sf_grid_desc {
    int L, M, N;          /* rho points (M+1) x (L+1), N vertical levels (N >= 5) */
    int precision;        /* enum sf_precision */
    /* horizontal metrics, (M+1)*(L+1) doubles each (modules/mod_grid.py:197-243) */
    const double *h, *pm, *pn, *on_u, *om_v, *fomn;
    /* S-coordinate tables (nonlinear/set_coords.py:355-423): sc_r[N], sc_w[N+1], Cs_r[N],
     * Cs_w[N+1]; critical depth hc and Vtransform (1 or 2) */
    const double *sc_r, *sc_w, *Cs_r, *Cs_w;
    double hc;
    int Vtransform;
    /* Boundary arrays built by Boundary (modules/mod_boundary.py:103-297), int32: */
    const int32_t *zeta_field_idx2; /* zetaBC.bcIdxFieldIdx2, (M+1)*(L+1), >= 0 on the ring */
    const int32_t *uvel_field_type; /* uvelBC.bcIdxFieldType, (M+1)*(L+1) */
    const int32_t *vvel_field_type; /* vvelBC.bcIdxFieldType, (M+1)*(L+1) */
    const int32_t *zeta_copy_idx1, *zeta_copy_idx2; int n_zeta_copy; /* zetaClosedOrGradientBCIdx1/2 */
    const int32_t *ubar_closed_idx; int n_ubar_closed;                /* ubarClosedBCIdx1 */
    const int32_t *vbar_closed_idx; int n_vbar_closed;                /* vbarClosedBCIdx1 */
    const int32_t *ubar_clamped_idx; int n_ubar_clamped;              /* ubarClampedBCIdx1 */
    const int32_t *ubar_grad_idx1, *ubar_grad_idx2; int n_ubar_grad;  /* ubarGradientBCIdx1/2 */
    const int32_t *vbar_grad_idx1; int n_vbar_grad;                   /* vbarGradientBCIdx1 */
} sf_grid_desc;

/* GLS closure parameters (generic length scale, Umlauf and Burchard 2003): exponents p, m, n,
 * cmu0, c1, c2, c3- (stable), c3+ (unstable), Schmidt numbers sigk, sigp, floors Kmin, Pmin,
 * background viscosities/diffusivities, surface and bottom roughness Zos, Zob (m) and the
 * quadratic bottom-drag coefficient rdrag2.  The reference's input file sets the k-epsilon
 * values (utility/test.in:326-381). */
typedef struct sf_gls_params {
    double p, m, n, cmu0, c1, c2, c3m, c3p, sigk, sigp, Kmin, Pmin;
    double Akv_bak, Akt_bak, Akk_bak, Akp_bak, Zos, Zob, rdrag2;
} sf_gls_params;

/* Three time slots of the barotropic state, in (t0, t1, t2) order, as rotated by
 * T_OCEAN.cycleTimes2D (modules/mod_ocean.py:120-154), plus the fast-time accumulators. */
typedef struct sf_state2d {
    void *zeta[3], *ubar[3], *vbar[3], *rzeta[3], *rubar[3], *rvbar[3];
    double *Zt_avg1, *DU_avg1, *DV_avg1;
} sf_state2d;

/* ---- context ---------------------------------------------------------------------------
 * sf_ctx_create replaces mod_operators.initModule (modules/mod_operators.py:31-45, which
 * launches initialize, modules/mod_cppkernels.h:154-171) and the boundary index setup of
 * Boundary.__init__ (modules/mod_boundary.py:237-297).  It uses the current CUDA device. */
int sf_ctx_create(const sf_grid_desc *desc, sf_ctx **out);
int sf_ctx_destroy(sf_ctx *ctx);
/* An ensemble context: n independent grids (members) of possibly different sizes and N,
 * stepped together.  Their fields live in shared pools, member after member (layout from
 * sf_ctx_member_layout); the time-step entry points (sf_maxflux_omega, sf_rhs3d,
 * sf_barotropic_loop and its parts, sf_set_depth, sf_step3d_uv(_bc), sf_omega) then take the
 * pool pointers and run every member in each launch (each block finds its member from a block
 * map).  The reference runs one grid per process; this is config 2's fused ensemble.  All
 * members share the precision; nothing else needs to match. */
int sf_ctx_create_ensemble(const sf_grid_desc *descs, int n, sf_ctx **out);
/* Tile shape of the tiled 3D right-hand side (sf_rhs3d) for this context: 0 = 32 x 8 rho points
 * (default), 1 = 32 x 4, 2 = 64 x 4, 3 = 32 x 16.  Results do not
 * depend on it; the autotuner (sailfish_b200.autotune) times the variants and picks one. */
int sf_ctx_set_tile(sf_ctx *ctx, int variant);
/* Number of members (1 for sf_ctx_create). */
int sf_ctx_members(const sf_ctx *ctx);
/* Offsets (elements) of each member in the pools of 2D fields, of N+1-level fields and of
 * N-level fields, and the pool sizes totals[0..2]; any pointer may be NULL. */
int sf_ctx_member_layout(const sf_ctx *ctx, long *off2, long *off3, long *offN, long *totals);
const char *sf_last_error(void);
int sf_version(void);
int sf_ctx_precision(const sf_ctx *ctx);

/* ---- barotropic (2D) kernels, modules/mod_cppkernels.cpp ------------------------------- */

/* computeZetaRHS (mod_cppkernels.cpp:81-128).  cff1 = weight1[iif-1]; the accumulators are
 * updated when is_predictor == 0. */
int sf_zeta_rhs(sf_ctx *ctx, const void *zeta, const void *ubar, const void *vbar,
                double *DU_avg1, double *DV_avg1, double *Zt_avg1, int is_predictor, double cff1,
                void *rzeta, sf_stream stream);
/* computeZetaPred (mod_cppkernels.cpp:134-150). */
int sf_zeta_pred(sf_ctx *ctx, double Dt, const void *zeta_t0, void *zeta_t2, const void *rzeta_t1,
                 sf_stream stream);
/* computeMomentumRHSPred / computeMomentumRHSCorr (mod_cppkernels.cpp:13-77):
 * gzeta = (1-weight)*za + weight*zb. */
int sf_momentum_rhs(sf_ctx *ctx, void *rhs_ubar, void *rhs_vbar, const void *za, const void *zb,
                    double g, double weight, sf_stream stream);
/* computeMomentumPred (mod_cppkernels.cpp:156-186). */
int sf_momentum_pred(sf_ctx *ctx, double Dt, const void *u_t1, void *u_t2, const void *v_t1,
                     void *v_t2, const void *rhsu, const void *rhsv, const void *zeta_t1,
                     const void *zeta_t2, sf_stream stream);
/* AdamsMoultonCorr3rd (mod_cppkernels.cpp:191-209): v_t2 += Dt*(5/12 r2 + 8/12 r1 - 1/12 r0). */
int sf_am3(sf_ctx *ctx, double Dt, void *v_t2, const void *r0, const void *r1, const void *r2,
           sf_stream stream);
/* zetabc (nonlinear/zetabc.py:5-12, copyBC of modules/mod_BC.c:16-23). */
int sf_zetabc(sf_ctx *ctx, void *zeta, sf_stream stream);
/* barotropicVelocityBC (nonlinear/barotropicVelocityBC.py:7-31, setBC/copyBC of
 * modules/mod_BC.c:6-23); the clamped value is 0.05*sin(0.0002*time2D). */
int sf_barotropic_velocity_bc(sf_ctx *ctx, void *ubar, void *vbar, double time2D, sf_stream stream);
/* Blow-up check: scans zeta, ubar, vbar (2D, (M+1)(L+1)) and u, v (3D, (N+1)(M+1)(L+1)) for
 * NaN, infinities and magnitudes above surface_bound (zeta) or velocity_bound (the
 * velocities); any argument may be NULL to skip that field.  Synchronises `stream` and returns
 * SF_ENONFINITE, with the field and the (level, j, i) of its first bad value in
 * sf_last_error(), or SF_OK.  No counterpart in the reference, whose step has no such check
 * and runs on into non-finite values (the step that a driver runs every K steps). */
int sf_check_state(sf_ctx *ctx, const void *zeta, const void *ubar, const void *vbar,
                   const void *u, const void *v, double surface_bound, double velocity_bound,
                   sf_stream stream);
/* step2dPredictor (nonlinear/step2d.py:23-81): first_step selects its Forward-Euler branch.
 * The leapfrog branch runs as one fused launch where the context allows it
 * (sf_ctx_fused_available, sf_ctx_set_fused), with the same results as the four launches. */
int sf_step2d_predictor(sf_ctx *ctx, const sf_state2d *s, double dtfast, double time2D,
                        int first_step, sf_stream stream);
/* step2dCorrector (nonlinear/step2d.py:84-128), cff1 = weight1[iif-1]. */
int sf_step2d_corrector(sf_ctx *ctx, const sf_state2d *s, double dtfast, double time2D,
                        double cff1, sf_stream stream);

/* One substep of main3d's barotropic loop (nonlinear/main3d.py:168-189) with the slots of s
 * already rotated: step2dPredictor, step2dCorrector and vbar_t2[:] = 0 in five passes plus
 * boundary programs.  The corrector's momentum right-hand side (rubar_t2/rvbar_t2,
 * step2d.py:116) is overwritten by the next predictor before anything reads it, so it is
 * evaluated only when `last` is set; every other value is the reference's. */
int sf_barotropic_substep(sf_ctx *ctx, const sf_state2d *s, double dtfast, double time2D,
                          double cff1, int last, sf_stream stream);
/* The whole barotropic loop of one baroclinic step (nonlinear/main3d.py:166-189): nsub
 * substeps (nfast+1), zeroing the accumulators before the first, rotating the slots of *s
 * as cycleTimes2D does (the final order is written back into *s), with time2D advanced by
 * dtfast per substep from *time2D (written back) and cff1 = weight1[iif-1] taken from the
 * host array weight1. */
int sf_barotropic_loop(sf_ctx *ctx, sf_state2d *s, int nsub, const double *weight1,
                       double dtfast, double *time2D, sf_stream stream);
/* Turn the CUDA-graph replay of sf_barotropic_loop on (default) or off.  With graphs on, the
 * loop's launches are captured once per (slot pointers, weights, time step) — at most three
 * captures, as the slots rotate with period 3 — and replayed as one graph launch; the clamped
 * boundary values, which depend on time2D, are written to the device before each replay.
 * Results are identical either way.  No counterpart in the reference. */
int sf_ctx_set_graphs(sf_ctx *ctx, int enable);
/* Bulk-copy staging (cp.async.bulk into shared memory, completing on mbarriers) in the
 * kernels that have it (the FP32 column solve): 1 where the fields' alignment allows it, 0
 * (default, the faster on one B200) for per-element cp.async staging.  Results are identical
 * either way.  No counterpart in the reference. */
int sf_ctx_set_bulk(sf_ctx *ctx, int enable);
/* Tuning knobs of a context's kernels (no counterpart in the reference):
 * SF_TUNE_MO_CHUNK: 0, 4, 5 (default) or 8 levels whose loads the fused set_maxflux/omega kernel
 *   issues together on columns whose fluxes it all computes itself;
 * SF_TUNE_PRED_PAIR: the fused predictor's paired form (two nodes per thread, vector loads) on
 *   grids with an even row length and aligned fields, with blocks of 16 staged rows (1) or 8
 *   (2, default); 0 for the scalar form;
 * SF_TUNE_S3_VEC: 1 (default) for the FP32 column solve's levels staged as 16-byte-aligned
 *   spans with 16-byte cp.async where the fields allow it, 0 for per-element cp.async
 *   (sf_ctx_set_bulk(ctx, 1) takes the same spans through bulk copies instead);
 * SF_TUNE_RHS_MARCH: the 3D right-hand side (sf_rhs3d) of a single grid with N >= 6 in its
 *   marching form (each thread walks a few rows of one column; neighbouring face fluxes come
 *   from the west lane and from the row below): 1 = 4 rows per thread, 4 warps per block;
 *   2 = 2 rows, 8 warps, two blocks per SM; 3 = 2 rows, 8 warps, three blocks per SM (default
 *   for FP32); 0 for the tiled form of sf_ctx_set_tile (default for FP64);
 * SF_TUNE_RHS_CHUNKS: 1 (default) for the marching form's levels staged as 16-byte chunks
 *   where the fields allow it (FP32, even row length, levels a multiple of 4 elements, fields
 *   on 16-byte boundaries), 0 for aligned element pairs.
 * Results are identical for every value in FP64; in FP32 the compiler may contract products
 * into FMAs differently in the variants, so they agree to the rounding of FP32. */
#define SF_TUNE_MO_CHUNK 0
#define SF_TUNE_PRED_PAIR 1
#define SF_TUNE_S3_VEC 2
#define SF_TUNE_RHS_MARCH 3
#define SF_TUNE_RHS_CHUNKS 4
int sf_ctx_tune(sf_ctx *ctx, int knob, int value);
/* Turn programmatic dependent launch of the barotropic loop's kernels on (default) or off:
 * with it each kernel's blocks become resident while its predecessor's last wave runs and wait
 * on the device for its completion.  Results are identical either way. */
int sf_ctx_set_pdl(sf_ctx *ctx, int enable);
/* Use the fused barotropic predictor (default on): one kernel per substep for computeZetaRHS +
 * computeZetaPred, zetabc, the momentum predictor and barotropicVelocityBC, for single grids
 * whose boundary programs write only the outer two-cell ring (sf_ctx_fused_available).  FP64
 * results are identical either way. */
int sf_ctx_set_fused(sf_ctx *ctx, int enable);
/* 1 if the context can use the fused predictor, else 0. */
int sf_ctx_fused_available(const sf_ctx *ctx);

/* ---- ROMS-form barotropic step, obsolete/step2d_LF_AM3.h.py + nonlinear/set_vbc.py ------
 * The free-surface and depth-integrated momentum step of ROMS's LF-AM3 scheme, which the
 * reference carries only as untranslated Fortran (obsolete/step2d_LF_AM3.h.py: fast-time
 * averages :778-846, free surface :933-1020, pressure gradient :1120-1230, Coriolis
 * :1503-1530, bottom stress :2242-2262, surface stress :2598-2612, momentum step
 * :2640-2760; quadratic drag nonlinear/set_vbc.py:16-41), for closed rectangular basins:
 * ROMS signs, forward/backward Euler on a loop's first substep, leapfrog predictor with the
 * time-filtered surface 0.68 zeta(n) + 0.16 (zeta(n-1) + zeta(n+1*)), AM3 corrector, Coriolis,
 * surface stress and quadratic bottom drag in the momentum right-hand side, zero-gradient
 * free surface and zero normal velocity at the walls, and the FP64 fast-time averages
 * Zt_avg1, DU_avg1, DV_avg1, DU_avg2, DV_avg2.  Slots of the sf_state2d: zeta/ubar/vbar
 * [0] = n-1, [1] = n, [2] = scratch for the predicted n+1*; rzeta/rubar/rvbar [0] = n-1,
 * [1] = n.  Each substep writes n+1 over n-1 and swaps the two slot pointers in *s. */
/* nfast+1 substeps of one baroclinic step (the last one only accumulates the averages, as in
 * ROMS); W1, W2: ROMS-indexed averaging weights (W1[m] = weight(1, m), m = 0..nfast+1, W2
 * likewise); sustr, svstr: kinematic surface stress (m2/s2) at U and V faces; rdrag2:
 * quadratic drag coefficient. */
int sf_roms_barotropic_loop(sf_ctx *ctx, sf_state2d *s, double *DU_avg2, double *DV_avg2,
                            const void *sustr, const void *svstr, double rdrag2, int nfast,
                            const double *W1, const double *W2, double dtfast, sf_stream stream);
/* One 2D-only step (predictor + corrector, no averages): the ROMS-form counterpart of
 * main2d's step (nonlinear/main2d.py:9-88); first selects forward/backward Euler. */
int sf_roms_step2d(sf_ctx *ctx, sf_state2d *s, const void *sustr, const void *svstr,
                   double rdrag2, double dtfast, int first, sf_stream stream);
/* Surface and bottom stress on the 3D momentum right-hand side (ROMS's ru includes them):
 * ru[N-1] += sustr om_u on_u and ru[0] -= rdrag2 ub sqrt(ub^2 + v_u^2) om_u on_u at the interior
 * U faces (ub, v_u from the bottom level of u, v), rv likewise. */
int sf_roms_stress3d(sf_ctx *ctx, const void *u, const void *v, void *ru, void *rv,
                     const void *sustr, const void *svstr, double rdrag2, sf_stream stream);
/* The ROMS-form 3D momentum right-hand side (Hz-weighted, m^4/s^2) at the interior faces, 0
 * elsewhere: Coriolis (as rhs_kernels.cpp:7-35) and second-order centred horizontal advection of
 * momentum (the UV_C2ADVECTION fluxes of obsolete/step2d_LF_AM3.h.py:1244-1300, per level with
 * Huon/Hvom); the vertical advection is implicit in sf_roms_step3d_uv.  It replaces the
 * reference's rhs3d (nonlinear/rhs.py:16-93) in the ROMS-form step, whose runnable advection
 * (rhs_kernels.cpp:71-196) is not ROMS's. */
int sf_roms_rhs3d(sf_ctx *ctx, const void *u, const void *v, const void *Huon, const void *Hvom,
                  const void *Hz, void *ru, void *rv, sf_stream stream);
/* The ROMS-form step3d_uv (the reference's step3D_uv.kernels.cpp:512-530 with ROMS's units and
 * time stepping: right-hand side Hzu u + dt pm pn (c0 ru(n) + c1 ru(n-1) + c2 ru(n-2)) with the
 * Adams-Bashforth weights of step iic - ntfirst (Euler, AB2, AB3), every level solved, viscosity
 * on the w level between two rho levels, vertical advection by the volume fluxes W implicit in
 * the same tridiagonal system (backward-Euler upwind), the depth mean set to DU_avg1 / on_u
 * from the new u) at the interior faces, and the barotropic restart: ubar_n, ubar_s (vbar
 * likewise) = the new depth-mean velocity there, 0 elsewhere.  N <= 64. */
int sf_roms_step3d_uv(sf_ctx *ctx, void *u, void *v, const void *ru0, const void *ru1,
                      const void *ru2, const void *rv0, const void *rv1, const void *rv2,
                      void *ubar_n, void *vbar_n, void *ubar_s, void *vbar_s, const void *Hz,
                      const void *Akv, const void *z_r, const void *W, const double *DU_avg1,
                      const double *DV_avg1, int iic, int ntfirst, double lambda, double dt,
                      sf_stream stream);
/* Closed walls for the 3D velocities: u = 0 on the west and east U faces, v = 0 on the south
 * and north V faces, every level. */
int sf_roms_closed_walls(sf_ctx *ctx, void *u, void *v, sf_stream stream);

/* ---- 3D right-hand side, nonlinear/rhs.py:16-93 + nonlinear/rhs_kernels.cpp ------------ */
/* rhs3d: ru = rv = 0, addCoriolis (:7-35), horizontalAdvection (:71-132), verticalAdvection
 * (:136-196), fused in one pass.  u, v, Huon, Hvom, W, ru, rv have N+1 levels, Hz has N. */
int sf_rhs3d(sf_ctx *ctx, const void *u, const void *v, const void *Huon, const void *Hvom,
             const void *W, const void *Hz, void *ru, void *rv, sf_stream stream);

/* ---- 3D step kernels, nonlinear/step3D_uv.kernels.cpp ---------------------------------- */
/* set_maxflux (:372-405). */
int sf_set_maxflux(sf_ctx *ctx, const void *u, const void *v, void *Huon, void *Hvom,
                   const void *Hz, sf_stream stream);
/* omega (:62-165). */
int sf_omega(sf_ctx *ctx, void *W, const void *Huon, const void *Hvom, const void *z_w,
             sf_stream stream);
/* set_maxflux + omega + set_zeta (:294-310) in one pass, as main3d launches them in a row
 * (nonlinear/main3d.py:118-151).  zeta_t1/zeta_t2/Zt_avg1 may be NULL to skip set_zeta. */
int sf_maxflux_omega(sf_ctx *ctx, const void *u, const void *v, void *Huon, void *Hvom,
                     const void *Hz, void *W, const void *z_w, void *zeta_t1, void *zeta_t2,
                     const double *Zt_avg1, sf_stream stream);
/* set_zeta (:294-310). */
int sf_set_zeta(sf_ctx *ctx, void *zeta1, void *zeta2, const double *Zt_avg1, sf_stream stream);
/* set_depth (:225-291), evaluated in FP64 in both precisions. */
int sf_set_depth(sf_ctx *ctx, const double *Zt_avg1, void *z_w, void *z_r, void *Hz,
                 sf_stream stream);
/* step3d_UV (:646-707) with its helpers (:408-639).  tmpU/tmpV are the pre-step velocities
 * (nonlinear/main3d.py:298-299); NULL means "read u/v before overwriting them". */
int sf_step3d_uv(sf_ctx *ctx, void *u, void *v, const void *ru, const void *rv, void *ubar_t1,
                 void *vbar_t1, void *ubar_t2, void *vbar_t2, const void *Hz, const void *Akv,
                 const void *z_r, const double *DU_avg1, const double *DV_avg1, const void *tmpU,
                 const void *tmpV, int iic, int ntfirst, double lambda, double Dt,
                 sf_stream stream);
/* setLateralUVBCs (:314-368); the clamped value is 0.05*sin(0.0002*time). */
int sf_lateral_uv_bc(sf_ctx *ctx, double time, void *u, void *v, sf_stream stream);
/* step3d_UV followed by setLateralUVBCs in the same pass (nonlinear/main3d.py:304-311). */
int sf_step3d_uv_bc(sf_ctx *ctx, void *u, void *v, const void *ru, const void *rv,
                    void *ubar_t1, void *vbar_t1, void *ubar_t2, void *vbar_t2, const void *Hz,
                    const void *Akv, const void *z_r, const double *DU_avg1,
                    const double *DV_avg1, int iic, int ntfirst, double lambda, double Dt,
                    double time, sf_stream stream);

/* ---- vertical mixing ------------------------------------------------------------------- */
/* GLS corrector, column physics of nonlinear/gls_corrector_step.py:26-825 (ROMS pseudo-code in
 * the reference; see sf_gls.cuh for the parts restated), on rho-interior columns.  u, v: rho
 * levels (N+1 allocated), z_r, Hz: N levels, bvf (buoyancy frequency squared), tke, gls, Akv,
 * Akt, Akk, Akp, Lscale: N+1 W levels, updated in place; sustr/svstr: kinematic surface stress
 * at U/V points (m2/s2); dt: baroclinic step. */
int sf_gls_corrector(sf_ctx *ctx, const sf_gls_params *params, double dt, const void *u,
                     const void *v, const void *z_r, const void *Hz, const void *bvf,
                     const void *sustr, const void *svstr, void *tke, void *gls, void *Akv,
                     void *Akt, void *Akk, void *Akp, void *Lscale, sf_stream stream);
/* GLS predictor, nonlinear/gls_predictor_step.py:18-216 (ROMS pseudo-code in the reference):
 * the auxiliary advective half step of tke and gls at W levels 1..N-1 on the rho-interior
 * points — fourth-order centred horizontal advection (:62-127), the LF step interpolated
 * back half a step with AM3 weights (Gamma = 1/6; first_step: forward half step, :133-157)
 * and fourth-order vertical advection (:162-208) — into tke_aux/gls_aux (time level 3) with
 * the half-step box height Hz_half; tke_nnew/gls_nnew = Hz_w * tke/gls(nstp) (:153-154).  A
 * zero-gradient lateral condition is applied to the auxiliary level (tkebc_tile is not in the
 * reference; edges take the adjacent interior value, corners the diagonal one); its levels 0
 * and N take the nstp values at the interior points (the corrector's vertical fluxes read
 * them, gls_corrector_step.py:349-372).  Huon, Hvom:
 * U/V fluxes at rho levels (N used); W, tke*, gls*, Hz_half: N+1 W levels; Hz: N levels. */
int sf_gls_predictor(sf_ctx *ctx, double dt, int first_step, const void *Huon, const void *Hvom,
                     const void *W, const void *Hz, const void *tke_nstp, const void *tke_indx,
                     void *tke_aux, void *tke_nnew, const void *gls_nstp, const void *gls_indx,
                     void *gls_aux, void *gls_nnew, void *Hz_half, sf_stream stream);
/* GLS corrector's advective terms, nonlinear/gls_corrector_step.py:172-388 (ROMS pseudo-code in
 * the reference): tke_nnew/gls_nnew (the Hz_w-weighted new level from sf_gls_predictor) less
 * dt*pm*pn times the horizontal divergence of third-order upstream-biased fluxes of the
 * auxiliary level tke_aux/gls_aux (:181-298), floored at params->Kmin/Pmin (:300-317), then less
 * the fourth-order vertical flux divergence (:329-377) and floored again (:378-388); W levels
 * 1..N-1 on the rho-interior points, in place.  gadv weighs the upstream curvature term; the
 * reference's pseudo-code uses Gadv without defining it (:236, :290): 1/3 is the third-order
 * upstream-biased scheme the comment at :214-215 names.  The vertical fluxes at rho levels 1
 * and N read levels 0 and N of the auxiliary level, which sf_gls_predictor fills with the nstp
 * values.  Huon, Hvom: U/V fluxes at rho levels; W and the tke/gls levels: N+1 W levels. */
int sf_gls_advect(sf_ctx *ctx, const sf_gls_params *params, double dt, double gadv,
                  const void *Huon, const void *Hvom, const void *W, const void *tke_aux,
                  const void *gls_aux, void *tke_nnew, void *gls_nnew, sf_stream stream);
/* sf_gls_corrector whose new level starts from tke_nnew/gls_nnew (after sf_gls_advect: the
 * corrector's production terms add to tke(nnew), gls_corrector_step.py:447-450) instead of
 * Hz_w * tke/gls(nstp); tke/gls hold nstp on entry and the new level on return, as in
 * sf_gls_corrector.  With tke_nnew = Hz_w * tke (sf_gls_predictor's, no advection) the result
 * is sf_gls_corrector's.  tke_nnew/gls_nnew must not alias tke/gls. */
int sf_gls_corrector_nnew(sf_ctx *ctx, const sf_gls_params *params, double dt, const void *u,
                          const void *v, const void *z_r, const void *Hz, const void *bvf,
                          const void *sustr, const void *svstr, const void *tke_nnew,
                          const void *gls_nnew, void *tke, void *gls, void *Akv, void *Akt,
                          void *Akk, void *Akp, void *Lscale, sf_stream stream);
/* sf_gls_corrector on the rho-interior columns p with columns[p] != 0 only (the closure's
 * fallback columns); the other columns' fields are left as they are.  No counterpart in the
 * reference. */
int sf_gls_corrector_cols(sf_ctx *ctx, const sf_gls_params *params, double dt, const void *u,
                          const void *v, const void *z_r, const void *Hz, const void *bvf,
                          const void *sustr, const void *svstr, void *tke, void *gls, void *Akv,
                          void *Akt, void *Akk, void *Akp, void *Lscale, const uint8_t *columns,
                          sf_stream stream);
/* sf_gls_corrector on the columns list[0 .. *count) (flat indices; *count read on the device,
 * so a kernel earlier on the stream may produce both), e.g. the closure's fallback columns
 * compacted by sf_closure_step: the cost follows the number of columns, not where they are.
 * No counterpart in the reference. */
int sf_gls_corrector_list(sf_ctx *ctx, const sf_gls_params *params, double dt, const void *u,
                          const void *v, const void *z_r, const void *Hz, const void *bvf,
                          const void *sustr, const void *svstr, void *tke, void *gls, void *Akv,
                          void *Akt, void *Akk, void *Akp, void *Lscale, const int *list,
                          const int *count, sf_stream stream);
/* obc_volcons (nonlinear/obc_volcons.py:6-69, ROMS pseudo-code in the reference): the
 * cross-section area and volume flux through the open edges selected by `edges` (W=1, E=2,
 * S=4, N=8), out[0] = area, out[1] = flux (inflow positive), out[2] = ubar_xs = flux/area,
 * accumulated in FP64 with compensated summation in a fixed order (deterministic).  With
 * `correct`, conserve_mass_tile follows: ubar on W/E and vbar on S/N open edges corrected by
 * -/+ ubar_xs so that the net flux through them vanishes.  zeta: the time level in use;
 * the depths come from the context's h. */
int sf_obc_volcons(sf_ctx *ctx, const void *zeta, void *ubar, void *vbar, int edges, int correct,
                   double *out, sf_stream stream);
/* Buoyancy frequency squared at all N+1 W levels of a linear equation of state in temperature
 * (alpha, 1/degC) with the analytic profile T(z) = T0 + dT exp(z/zscale):
 * bvf = g alpha dT/zscale exp(z_w/zscale).  The stratification of the analytic basins, whose
 * tracers are not stepped (the reference's time step has no tracer equation either). */
int sf_analytic_bvf(sf_ctx *ctx, const void *z_w, double dT, double zscale, double alpha, double g,
                    void *bvf, sf_stream stream);

/* ---- learned closure (no counterpart in the reference) --------------------------------------
 * A per-column MLP standing in for the GLS corrector's Akv/Akt: SF_MLP_LAYERS dense layers of
 * width 128 (inputs and outputs zero-padded to 128), GELU or ReLU (`act`) between them, BF16
 * weights W[l]
 * ([out][in], row-major, device) and FP32 biases b[l] (device); products on the tensor cores
 * (tcgen05) with FP32 accumulation.  Rows are samples (one water column each), 128 FP32
 * values per row.  `err` is a device int set to 1 if a bounded wait on the tensor cores gave
 * up.  Error text of these entry points: sf_mlp_last_error(). */
#define SF_MLP_LAYERS 5
#define SF_MLP_WIDTH 128
#define SF_MLP_GELU 0   /* tanh form */
#define SF_MLP_RELU 1
typedef struct sf_mlp_params {
    const void *W[SF_MLP_LAYERS];
    const float *b[SF_MLP_LAYERS];
    int act;   /* SF_MLP_GELU (0, the zero-initialised default) or SF_MLP_RELU */
} sf_mlp_params;

const char *sf_mlp_last_error(void);
/* O[r, :] = act(A B^T + bias) for a 128-wide B (act 0: none, 1: GELU, 2: ReLU): A is element
 * (r, k) = A[r*a_rs + k*a_ks]
 * (n_rows x K, FP32 or BF16), B likewise (128 x K); K a multiple of 16; optional pre-activation
 * copy Z.  The dense-product building block of the forward and backward passes. */
int sf_mlp_gemm(int n_rows, int K, const void *A, int a_bf16, long a_rs, long a_ks,
                const void *B, int b_bf16, long b_rs, long b_ks, const float *bias, int act,
                float *O, long ldo, float *Z, long ldz, int *err, sf_stream stream);
/* Forward pass over n rows; `acts` ((LAYERS-1) x n x 128) and `pre` (LAYERS x n x 128) keep the
 * hidden activations and pre-activations for the backward pass (acts required). */
int sf_mlp_forward(const sf_mlp_params *w, int n, const float *X, float *Y, float *acts,
                   float *pre, int *err, sf_stream stream);
/* Inference only: the same outputs as sf_mlp_forward (up to the GELU's hardware tanh) from one
 * fused pass that keeps every layer's weights and the tile's activations on chip, reading X
 * and writing Y only (n x 128 FP32 each, 16-byte aligned rows). */
int sf_mlp_infer(const sf_mlp_params *w, int n, const float *X, float *Y, int *err,
                 sf_stream stream);
/* Backward pass: weight and bias gradients dW[l] (128 x 128 FP32), db[l] (128) for output
 * gradient dY; `work` is 2 x n x 128 FP32 scratch; n a multiple of 16. */
int sf_mlp_backward(const sf_mlp_params *w, int n, const float *X, const float *acts,
                    const float *pre, const float *dY, float *const *dW, float *const *db,
                    float *work, int *err, sf_stream stream);
/* sf_mlp_backward without the `work` argument, for callers that cannot allocate device memory
 * where they train (an application that owns all device memory through its own pool, or a
 * latency-critical loop that may not call an allocator).  No counterpart in the reference.
 * Its scratch is a fixed 2 MiB device array inside the library, held by every GPU that loads
 * it until the process exits; n <= 2048 rows, larger n is rejected with SF_EINVAL.  The first
 * call on a device looks up that array's device address (cudaGetSymbolAddress), so make it
 * before any stream capture.  Each device has its own 2 MiB copy of the array; on one device
 * all calls share it and leave their intermediate values in it (every value read is written
 * first by the same call), so calls that overlap on the same device (on different streams,
 * for example) race. */
int sf_mlp_backward_static(const sf_mlp_params *w, int n, const float *X, const float *acts,
                           const float *pre, const float *dY, float *const *dW, float *const *db,
                           int *err, sf_stream stream);
/* Mean squared error over the first nvalid outputs of each row; adds the loss into *loss. */
int sf_mlp_mse(int n, int nvalid, const float *Y, const float *T, float *dY, float *loss,
               sf_stream stream);
/* Adam step on n FP32 master weights (bias-corrected, step >= 1); refreshes the BF16 copy. */
int sf_mlp_adam(long n, float *w, const float *g, float *m, float *v, void *w_bf16, float lr,
                float b1, float b2, int step, float eps, sf_stream stream);
/* One feature row per water column (s2 x 128 FP32), nl = N-1 interior W levels (N <= 63):
 * log-scaled shear^2 in [0, nl), log-scaled N^2 in [nl, 2nl), then log10 surface friction
 * velocity squared, surface buoyancy flux and log10 depth; non-interior columns are 0. */
int sf_closure_features(sf_ctx *ctx, const void *u, const void *v, const void *z_r,
                        const void *bvf, const void *sustr, const void *svstr, float *X,
                        sf_stream stream);
/* mask[p] = 1 for each rho-interior column whose feature row (from sf_closure_features) has
 * any of its first nfeat features outside [lo[k], hi[k]] (NaN included): the columns the
 * network was not trained for, which plain GLS handles (sf_gls_corrector_cols); else 0. */
int sf_closure_range_mask(sf_ctx *ctx, const float *X, int nfeat, const float *lo,
                          const float *hi, uint8_t *mask, sf_stream stream);
/* The closure for one step in one fused pass: for every rho-interior column, its feature row
 * (as sf_closure_features), the range check against [lo, hi] over the first nfeat features
 * (as sf_closure_range_mask, written to `fallback`), the network (as sf_mlp_infer) and, for
 * the columns in range, Akv/Akt at levels 1..N-1 (as sf_closure_apply).  Columns flagged in
 * `fallback` keep their Akv/Akt for plain GLS; if fallback_list/fallback_count are given (s2
 * ints, one int), the flagged columns are also listed there, in no particular order, with
 * *fallback_count zeroed first, for sf_gls_corrector_list.  No counterpart in the reference. */
int sf_closure_step(sf_ctx *ctx, const sf_mlp_params *w, const void *u, const void *v,
                    const void *z_r, const void *bvf, const void *sustr, const void *svstr,
                    int nfeat, const float *lo, const float *hi, uint8_t *fallback,
                    int *fallback_list, int *fallback_count, void *Akv, void *Akt, int *err,
                    sf_stream stream);
/* Akv and Akt at the interior W levels 1..N-1 from the network outputs [0, nl) and [nl, 2nl)
 * (log10, clipped to [1e-6, 1e-1] m2/s), except on columns flagged in `fallback` (may be
 * NULL). */
int sf_closure_apply(sf_ctx *ctx, const float *Y, const uint8_t *fallback, void *Akv, void *Akt,
                     sf_stream stream);

#ifdef __cplusplus
}
#endif
#endif /* SAILFISH_B200_H */
