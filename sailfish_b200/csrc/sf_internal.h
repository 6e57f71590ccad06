// Internal types shared by the C-ABI layer (sf_capi.cu) and the kernel translation units
// (sf_kernels_f64.cu, sf_kernels_f32.cu).
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include "../../include/sailfish_b200.h"

namespace sf {

// A boundary "program": the sequential effect of the reference's boundary scatter launches
// (setBC / copyBC, modules/mod_BC.c:6-23, run one after the other in thread order) reduced to
// a gather dst[k] <- src[k], where src >= 0 is a node of the field as it was before the
// program ran, src == -1 is the constant 0 and src == -2 is the time-dependent value.
// Entries whose source is another entry's destination (and those destinations) form the
// short "chained" list, applied by one thread that reads all its sources before writing;
// all other entries are independent and applied by one thread each.
constexpr int kMaxChained = 32;
// Per-node boundary-program maps of the fused predictor: kBcNone (no destination) or
// (source + 2) | kBcChained when the entry belongs to the chained group.
constexpr int kBcNone = 0x7FFFFFFF;
constexpr int kBcChained = 1 << 30;
struct BcProgram {
    int n = 0;                 // independent entries
    int *dst = nullptr;        // device
    int *src = nullptr;        // device
    int nch = 0;               // chained entries
    int *dst_ch = nullptr;     // device
    int *src_ch = nullptr;     // device
    int ngr = 0;               // groups of chained entries (one per ensemble member that has
    int *gofs = nullptr;       // any): group g is [gofs[g], gofs[g+1]), device
};

// Coefficients of the GLS predictor's half step: cff1, cff2 of the LF/AM3 interpolation and
// cff3, the time step of the advective terms (gls_predictor_step.py:133-146).
struct GlsPre {
    double c1, c2, c3;
};

// floor(n / d) for 0 <= n < 2^31 by one 64-bit multiply and a shift: with 2^(l-1) < d <= 2^l
// and m = ceil(2^(31+l) / d), floor(n * m / 2^(31+l)) = floor(n / d) (Granlund and
// Montgomery, "Division by invariant integers using multiplication", PLDI 1994, the N+l-bit
// multiplier form).  Used for the flat index's row and column in the 2D kernels.
struct FastDiv {
    unsigned long long m;
    int shift;   // 31 + l
};
inline FastDiv make_fastdiv(int d) {
    int l = 0;
    while ((1LL << l) < d) ++l;
    FastDiv f;
    f.shift = 31 + l;
    f.m = ((1ULL << f.shift) + (unsigned long long)d - 1) / (unsigned long long)d;
    return f;
}
__host__ __device__ __forceinline__ int fdiv(int n, FastDiv f) {
    return (int)(((unsigned long long)(unsigned)n * f.m) >> f.shift);
}

// Grid view handed to kernels by value.
template <typename R>
struct Geo {
    int I, J, N;  // xi points (L+1), eta points (M+1), levels
    FastDiv dI, dJ;   // division by I and by J
    long s2;      // I*J
    const R *on_u, *om_v, *pm, *pn, *h, *fomn;
    const double *hd;                          // h in FP64 (set_depth)
    const double *sc_r, *sc_w, *Cs_r, *Cs_w;   // S-coordinate tables
    double hc;
    int Vtransform;
    const int *bcfield;   // zetaBC.bcIdxFieldIdx2
    const int *utype, *vtype;
    long ref_threads;     // threads of the reference's rhs3d launches (rhs_kernels.cpp:86-91)
    int *err = nullptr;   // context's device error word: a bounded wait that gave up sets it
};

// Launch geometry shared by the kernels and the host code that builds block maps.
constexpr int kPointBlock = 256;           // threads per block of the point kernels
constexpr int kTileX = 32, kTileY = 8;     // tile of the tiled 3D right-hand side
constexpr int kPipeTile = 64;              // columns per block of the pipelined column solve

// One member of an ensemble context: its grid view (metric pointers into the context's
// pools) and the offsets of its fields in the state pools: 2D fields (off2), fields of N+1
// levels (off3) and of N levels (offN); ntx = tiles along xi of the tiled kernels.
constexpr int kRhsTiles = 4;
constexpr int kRhsTileX[kRhsTiles] = {32, 32, 64, 32}, kRhsTileY[kRhsTiles] = {8, 4, 4, 16};
template <typename R>
struct Member {
    Geo<R> g;
    long off2, off3, offN;
    int ntx[kRhsTiles];   // tiles along xi for each tile variant of the 3D right-hand side
};

}  // namespace sf

// A captured barotropic loop (sf_barotropic_loop): valid for the slot pointers, weights and
// time step it was captured with.
struct sf_loop_graph {
    cudaGraphExec_t exec = nullptr;
    int nsub = 0;
    double dtfast = 0.0;
    void *slots[18] = {};
    double *acc[3] = {};
    double w[256] = {};
};

struct sf_ctx {
    int prec;
    int L, M, N, I, J;
    long s2;
    int device;
    void *metrics[6];       // h, pm, pn, on_u, om_v, fomn in the context precision
    double *hd;             // h in FP64
    double *vert;           // sc_r[N] | sc_w[N+1] | Cs_r[N] | Cs_w[N+1]
    double hc;
    int Vtransform;
    int *bcfield, *utype, *vtype;
    sf::BcProgram zbc, ubc, vbc;
    long ref_threads;
    // CUDA-graph replay of the barotropic loop: a capture stream, the per-substep clamped
    // boundary values (device, written before each replay), and up to 3 captured loops (the
    // slot rotation cycles with period 3).
    int use_graphs = 1;
    // Programmatic dependent launch of the barotropic kernels (sf_ctx_set_pdl): each kernel
    // lets its successor's blocks become resident while its own last wave runs; the successor
    // waits (griddepcontrol.wait) for its completion before touching any field.
    int use_pdl = 1;
    // The fused barotropic predictor (sf::Ops::pred2d) for single grids whose boundary
    // programs write only the outer two-cell ring: per-node program maps (zeta, ubar, vbar;
    // device, 3 * s2), the last-block counter, and whether the fused form is used.
    int *bcmap = nullptr;
    int *pred_counter = nullptr;
    int pred_ok = 0;
    int use_fused = 1;
    // bulk-copy staging (cp.async.bulk) in the kernels that have it (sf_ctx_set_bulk); off
    // by default: on basin4 the column solve took 2.08 ms with it against 1.65 ms with
    // per-element cp.async staging
    int use_bulk = 0;
    // levels whose loads the fused flux/omega kernel issues together (sf_ctx_tune; basin4:
    // 0.82, 0.77 and 1.16 ms with 4, 5 and 8: 80, 80 and 128 registers)
    int mo_chunk = 5;
    // fused predictor in its paired form (two nodes per thread) where the grid allows it: 1
    // with 16-row blocks, 2 with 8-row blocks (basin4 loop 4.27 and 4.18 ms), 0 scalar (4.49)
    int pred_pair = 2;
    // FP32 column solve staged with 16-byte cp.async where aligned (else per element): on one
    // B200 basin4 takes 1.43 ms with it and 1.56 ms without
    int s3_vec = 1;
    // 3D right-hand side in its marching form (sf_ctx_tune SF_TUNE_RHS_MARCH; set at context
    // creation: 3 for FP32 single grids); 0: the tiled form of rhs_tile
    int rhs_march = 0;
    // the marching form's levels staged as 16-byte chunks where the fields allow it (FP32)
    int rhs_chunks = 1;
    cudaStream_t cap = nullptr;
    double *d_bcval = nullptr;
    sf_loop_graph graphs[3];
    int graph_next = 0;
    // the learned closure's feature-row tiles (sf_closure_step), allocated on first use
    void *closure_x = nullptr;
    size_t closure_x_bytes = 0;
    // Ensembles (sf_ctx_create_ensemble): nmem > 1 members whose fields live in shared pools;
    // the step kernels take the pools and find their member from a block map (member, local
    // block).  For a single grid nmem = 1 and the kernels take the arrays directly.
    int nmem = 1;
    int maxN = 0;
    void *members = nullptr;     // device sf::Member<R>[nmem]
    int2 *bm_pt = nullptr;       // blocks of kBlock points
    int nbm_pt = 0;
    int2 *bm_128 = nullptr;      // blocks of 128 points
    int nbm_128 = 0;
    int2 *bm_tile[sf::kRhsTiles] = {};   // tiles of the tiled 3D right-hand side, per variant
    int nbm_tile[sf::kRhsTiles] = {};
    int rhs_tile = 0;            // variant of the tiled 3D right-hand side (sf_ctx_set_tile)
    int2 *bm_pipe = nullptr;     // 64-point tiles of the pipelined column solve
    int nbm_pipe = 0;
    long tot2 = 0, tot3 = 0, totN = 0;   // pool sizes
    long *h_off2 = nullptr, *h_off3 = nullptr, *h_offN = nullptr;   // host copies
    // sf_check_state: the smallest (field, flat index) key of a bad value (device) and its
    // pinned host copy, allocated on first use
    unsigned long long *check_dev = nullptr;
    unsigned long long *check_host = nullptr;
    // device error word of the kernels with bounded waits (Geo::err); sf_check_state reports
    // and clears it
    int *dev_err = nullptr;
};

namespace sf {

// Kernels launched through launch_dep (programmatic dependent launch) start with pdl_enter():
// it lets the next kernel on the stream begin launching its blocks, then waits until this
// kernel's predecessor has completed and its writes are visible.  Both are no-ops when the
// kernel was launched without the attribute.
__device__ __forceinline__ void pdl_enter() {
    asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
    asm volatile("griddepcontrol.wait;" ::: "memory");
}

template <typename... KArgs, typename... Args>
inline cudaError_t launch_dep(const sf_ctx *c, void (*kern)(KArgs...), dim3 grid, dim3 block,
                              size_t smem, cudaStream_t s, Args... args) {
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = grid;
    cfg.blockDim = block;
    cfg.dynamicSmemBytes = smem;
    cfg.stream = s;
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    at[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = at;
    cfg.numAttrs = c->use_pdl ? 1 : 0;
    return cudaLaunchKernelEx(&cfg, kern, static_cast<KArgs>(args)...);
}

// Levels the ROMS-form step3d_uv holds per column (sf_roms_step3d_uv rejects more).
constexpr int kRomsMaxN = 64;

// Arguments of one phase of the ROMS-form barotropic substep (kernels in sf_roms.cuh).
template <typename R>
struct RomsArgs {
    const R *zb, *zn, *zp;          // zeta at n-1, n and the predicted n+1*
    const R *ub, *un, *up;
    const R *vb, *vn, *vp;
    R *zout, *uout, *vout;          // the phase's output slots (p in the predictor, b in the corrector)
    const R *zkstp, *ukstp, *vkstp; // the momentum step's old level (kstp)
    const R *zrhs, *urhs, *vrhs;    // the level the right-hand side is evaluated at (krhs)
    R *rz_n, *ru_n, *rv_n;          // tendencies of level n (written by the predictor)
    const R *rz_b, *ru_b, *rv_b;    // tendencies of level n-1
    const R *sustr, *svstr;         // kinematic surface stress at U / V faces (m2/s2)
    double *Zt, *DU1, *DV1, *DU2, *DV2;
    double rdrag2, dtfast;
    double c1, c2;                  // accumulation weights of this phase
    int phase;                      // 0 predictor, 1 corrector
    int first;                      // first substep of a loop: forward / backward Euler
    int acc;                        // 0 none, 1 accumulate, 2 reset (predictor of substep 1)
    int step;                       // 0: the predictor only accumulates (substep nfast+1)
};


// Launchers, one explicit instantiation per precision (FP64 in a translation unit built
// without FMA contraction, so that it reproduces the reference's IEEE evaluation).
template <typename R>
struct Ops {
    static Geo<R> geo(const sf_ctx *c);
    static cudaError_t zeta_rhs(const sf_ctx *c, const R *zeta, const R *ubar, const R *vbar,
                                R *rzeta, int mode, double cff1, double *Zt, double *DU, double *DV,
                                const R *zeta_t0, R *zeta_t2, double Dt, cudaStream_t s);
    static cudaError_t zeta_pred(const sf_ctx *c, double Dt, const R *z0, R *z2, const R *rz1,
                                 cudaStream_t s);
    static cudaError_t zeta_euler(const sf_ctx *c, double Dt, const R *z1, R *z2, const R *rz1,
                                  cudaStream_t s);
    static cudaError_t momentum(const sf_ctx *c, R *rhs_u, R *rhs_v, const R *za, const R *zb,
                                double g, double weight, int do_rhs, int do_pred, double Dt,
                                const R *u_t1, R *u_t2, const R *v_t1, R *v_t2, const R *z1,
                                const R *z2, cudaStream_t s);
    static cudaError_t am3(const sf_ctx *c, double Dt, R *v, const R *r0, const R *r1,
                           const R *r2, cudaStream_t s);
    static cudaError_t corr_point(const sf_ctx *c, double Dt, R *zeta_t2, const R *rz0,
                                  const R *rz1, const R *rz2, R *ubar_t1, const R *vbar_t1,
                                  const R *rub0, const R *rub1, R *vbar_t2, cudaStream_t s);
    static cudaError_t bc_apply(const sf_ctx *c, const BcProgram &p1, R *f1,
                                const BcProgram &p2, R *f2, double val, cudaStream_t s,
                                const double *valp = nullptr);
    static cudaError_t rhs3d(const sf_ctx *c, const R *u, const R *v, const R *Huon,
                             const R *Hvom, const R *W, const R *Hz, R *ru, R *rv,
                             cudaStream_t s);
    static cudaError_t maxflux_omega(const sf_ctx *c, const R *u, const R *v, R *Huon, R *Hvom,
                                     const R *Hz, R *W, const R *z_w, int do_flux, int do_omega,
                                     R *zeta1, R *zeta2, const double *Zt, cudaStream_t s);
    static cudaError_t set_zeta(const sf_ctx *c, R *z1, R *z2, const double *Zt, cudaStream_t s);
    static cudaError_t set_depth(const sf_ctx *c, const double *Zt, R *z_w, R *z_r, R *Hz,
                                 cudaStream_t s);
    static cudaError_t step3d_uv(const sf_ctx *c, R *u, R *v, const R *ru, const R *rv,
                                 R *ubar_t1, R *vbar_t1, R *ubar_t2, R *vbar_t2, const R *Hz,
                                 const R *Akv, const R *z_r, const double *DU, const double *DV,
                                 const R *tmpU, const R *tmpV, double cff, double lambda,
                                 double Dt, int do_bc, double bcval, cudaStream_t s);
    static cudaError_t lateral_uv_bc(const sf_ctx *c, R *u, R *v, double val, cudaStream_t s);
    static cudaError_t gls_corrector(const sf_ctx *c, const sf_gls_params &P, double dt,
                                     const R *u, const R *v, const R *z_r, const R *Hz,
                                     const R *bvf, const R *sustr, const R *svstr, R *tke, R *gls,
                                     R *Akv, R *Akt, R *Akk, R *Akp, R *Lscale,
                                     const R *tkn0, const R *gln0, const uint8_t *sel,
                                     const int *list, const int *count, cudaStream_t s);
    static cudaError_t gls_advect(const sf_ctx *c, double dt, double gadv, double Kmin,
                                  double Pmin, const R *Huon, const R *Hvom, const R *W,
                                  const R *tke3, const R *gls3, R *tken, R *glsn, cudaStream_t s);
    static cudaError_t gls_prestep(const sf_ctx *c, GlsPre pc, const R *Huon, const R *Hvom,
                                   const R *W, const R *Hz, const R *tke0, const R *tkei, R *tke3,
                                   R *tken, const R *gls0, const R *glsi, R *gls3, R *glsn,
                                   R *Hz_half, cudaStream_t s);
    // vb1_zero: vbar_t1 is known to be all +0 (the loop's substeps after the first)
    static cudaError_t pred2d(const sf_ctx *c, R *z0, R *z1, R *z2, R *ub1, R *vb1, R *ub2,
                              R *vb2, R *rz, R *ru, R *rv, double Dt, double weight, double val,
                              const double *valp, cudaStream_t s, int vb1_zero = 0);
    static cudaError_t obc_volcons(const sf_ctx *c, const R *zeta, R *ubar, R *vbar, int edges,
                                   int correct, double *out, cudaStream_t s);
    static cudaError_t analytic_bvf(const sf_ctx *c, const R *z_w, double dT, double zscale,
                                    double galpha, R *bvf, cudaStream_t s);
    // the ROMS-form barotropic step (sf_roms.cuh)
    static cudaError_t roms_phase(const sf_ctx *c, const RomsArgs<R> &a, cudaStream_t s);
    static cudaError_t roms_stress3d(const sf_ctx *c, const R *u, const R *v, R *ru, R *rv,
                                     const R *sustr, const R *svstr, double rdrag2, cudaStream_t s);
    static cudaError_t roms_rhs3d(const sf_ctx *c, const R *u, const R *v, const R *Huon,
                                  const R *Hvom, const R *Hz, R *ru, R *rv, cudaStream_t s);
    static cudaError_t roms_step3d(const sf_ctx *c, R *u, R *v, const R *const *ru,
                                   const R *const *rv, const double *coef, R *ubar_n, R *vbar_n,
                                   R *ubar_s, R *vbar_s, const R *Hz, const R *Akv, const R *z_r,
                                   const R *W, const double *DU, const double *DV, double dt,
                                   double lamdt, cudaStream_t s);
    static cudaError_t roms_walls3d(const sf_ctx *c, R *u, R *v, cudaStream_t s);
};

extern template struct Ops<double>;
extern template struct Ops<float>;

}  // namespace sf
