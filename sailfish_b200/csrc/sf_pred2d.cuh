// The barotropic predictor of one substep as one kernel (single grids): computeZetaRHS +
// computeZetaPred, zetabc, computeMomentumRHSPred + computeMomentumPred, barotropicVelocityBC
// (nonlinear/step2d.py:23-81 with the kernels of mod_cppkernels.cpp:13-186), replacing four
// launches whose intermediate fields each went through DRAM.
//
// A block owns a tile of 31 x 15 rho points.  Phase 1 computes the predicted zeta on the tile
// and on a halo of one row (south) and one column (west) into shared memory, 32 x 16 nodes on
// 32 x 8 threads (two rows each: every warp does the same work); phase 2 computes the momentum
// right-hand side and the predicted ubar/vbar of the tile's nodes from it.  Interior points with two cells of margin (the "deep" region,
// 2 <= i <= I-3, 2 <= j <= J-3) hold no boundary destination, so they take the fast path.
// Points of the outer two-cell ring evaluate everything as pure functions of the step's inputs:
// a field's value after its boundary program at node x is, by the program's gather semantics
// (all sources read before any destination is written), its pre-program value at the source
// node of x (or 0, or the clamped value), and a pre-program value is either computed from the
// inputs or, where the predictor does not write the node, the node's old content.  So no block
// waits for another.  Destinations are written with their final values, except those of
// chained entries (a destination that is also a source, e.g. at corners), whose old content
// other blocks may still read: block 0 evaluates them first (into a small buffer, while every
// old content is intact) and the last "edge" block to finish copies them into place.  Old
// contents are read only where a node off the deep region is evaluated, i.e. by the ring blocks
// and by the tiles whose nodes or halo reach the outer ring (the edge blocks); tiles wholly
// inside (tile and halo deep) read only the step's inputs, so they leave without taking part
// in the count.
#pragma once
#include "sf_internal.h"

namespace sf {

// A tile of 31 x 15 nodes; its block of 32 x 8 threads stages the tile with its south halo row
// and west halo column (32 x 16 nodes), two staged rows per thread.
constexpr int kPredTX = 31, kPredTY = 15;

template <typename R>
struct PredArgs {
    Geo<R> g;
    const R *z0, *z1, *ub1, *vb1;   // inputs (zeta_t0, zeta_t1, ubar_t1, vbar_t1)
    R *z2, *rz, *ru, *rv, *ub2, *vb2;   // outputs (zeta_t2, rzeta_t1, rubar_t1, rvbar_t1, ...)
    const int *mz, *mu, *mv;        // per-node program maps (kBcNone or code)
    R Dt, w1, w, grav;
    R val;                          // clamped value of the ubar/vbar programs
    const double *valp;             // ... or read from the device (graph replay)
    BcProgram pz, pu, pv;           // for the chained entries
    int *counter;                   // blocks done (last-block detection), reset by the last
    R *chv;                         // chained entries' values [3][kMaxChained], from block 0
    int vb1_zero;                   // vbar_t1 is all +0: the paired tiles use 0 without loading it
};

__device__ __forceinline__ int bc_src(int m) { return (m & (kBcChained - 1)) - 2; }

// computeZetaRHS at an interior node (mod_cppkernels.cpp:81-128), as zeta_rhs_body.
template <typename R>
__device__ __forceinline__ R prd_rz(const PredArgs<R> &a, long x) {
    const Geo<R> &g = a.g;
    const long I = g.I;
    const R *h = g.h, *zeta = a.z1;
    const R Dp = zeta[x] + h[x], Dw = zeta[x - 1] + h[x - 1], De = zeta[x + 1] + h[x + 1];
    const R Ds = zeta[x - I] + h[x - I], Dn = zeta[x + I] + h[x + I];
    const R DUp = a.ub1[x] * ((Dp + Dw) * R(0.5));
    const R DUe = a.ub1[x + 1] * ((De + Dp) * R(0.5));
    const R DVp = a.vb1[x] * ((Dp + Ds) * R(0.5));
    const R DVn = a.vb1[x + I] * ((Dn + Dp) * R(0.5));
    return (((DUe * g.on_u[x + 1] - DUp * g.on_u[x]) + (DVn * g.om_v[x + I] - DVp * g.om_v[x])) *
            g.pm[x]) * g.pn[x];
}

// zeta_t2 at x before zetabc: zeta_t0 + Dt * rzeta where i != 0 and j != 0 (rzeta as the
// node's old value off the interior), else the node's old content (not written).
template <typename R>
__device__ __forceinline__ R prd_z2p(const PredArgs<R> &a, long x) {
    const int j = fdiv((int)x, a.g.dI), i = (int)x - j * a.g.I;
    if (i == 0 || j == 0) return a.z2[x];
    const R r = rint_(i, j, a.g.I, a.g.J) ? prd_rz(a, x) : a.rz[x];
    return a.z0[x] + a.Dt * r;
}

// zeta_t2 at x after zetabc (its program has no clamped entries: value 0).
template <typename R>
__device__ __forceinline__ R prd_z2b(const PredArgs<R> &a, long x) {
    const int m = a.mz[x];
    if (m == kBcNone) return prd_z2p(a, x);
    const int s = bc_src(m);
    return s >= 0 ? prd_z2p(a, s) : R(0);
}

// zeta_t2 after zetabc at x from the block's shared tile when x lies in it (the tile and its
// south/west halo hold exactly these values), else through the pure functions.
template <typename R>
struct PrdTile {
    const R (*s)[kPredTX + 1];
    int i0, j0;
};
template <typename R>
__device__ __forceinline__ R prd_zb(const PredArgs<R> &a, const PrdTile<R> &t, long x) {
    const int j = fdiv((int)x, a.g.dI), i = (int)x - j * a.g.I;
    const int r = j - t.j0 + 1, c = i - t.i0 + 1;
    if (r >= 0 && r <= kPredTY && c >= 0 && c <= kPredTX && (r | c) != 0) return t.s[r][c];
    return prd_z2b(a, x);
}

// computeMomentumRHSPred + computeMomentumPred at x (momentum_body) with zeta_t2 after zetabc.
template <typename R>
struct PrdMom {
    R ru, rv, u2, v2;
    bool in, pd;
};
template <typename R>
__device__ __forceinline__ PrdMom<R> prd_mom(const PredArgs<R> &a, const PrdTile<R> &t, long x) {
    const Geo<R> &g = a.g;
    const long I = g.I, J = g.J;
    const int j = fdiv((int)x, g.dI), i = (int)x - j * g.I;
    const R *h = g.h;
    PrdMom<R> o;
    o.ru = o.rv = o.u2 = o.v2 = R(0);
    o.in = rint_(i, j, g.I, g.J);
    o.pd = (int)x - fdiv((int)x, g.dJ) * g.J != 0 && x >= J;
    if (!o.in && !o.pd) return o;
    // x >= 1 here (interior, or x % J != 0)
    const R zp = prd_zb(a, t, x), zw = prd_zb(a, t, x - 1);
    const R zs = x - I >= 0 ? prd_zb(a, t, x - I) : R(0);
    if (o.in) {
        const R gp = a.w1 * zp + a.w * a.z0[x];
        const R gw = a.w1 * zw + a.w * a.z0[x - 1];
        const R gs = a.w1 * zs + a.w * a.z0[x - I];
        o.ru = (a.grav * g.on_u[x]) * (((h[x] + h[x - 1]) * R(0.5)) * (gp - gw) + R(0.5) * (gp * gp - gw * gw));
        o.rv = (a.grav * g.om_v[x]) * (((h[x] + h[x - I]) * R(0.5)) * (gp - gs) + R(0.5) * (gp * gp - gs * gs));
    }
    if (o.pd) {
        R ru = o.ru, rv = o.rv;
        if (!o.in) {
            ru = a.ru[x];
            rv = a.rv[x];
        }
        const R D1p = a.z1[x] + h[x], D2p = zp + h[x];
        const R D1U = (D1p + (a.z1[x - 1] + h[x - 1])) * R(0.5);
        const R D2U = (D2p + (zw + h[x - 1])) * R(0.5);
        const R hs = ldz(h, x - I);
        const R D1V = (D1p + (ldz(a.z1, x - I) + hs)) * R(0.5);
        const R D2V = (D2p + (zs + hs)) * R(0.5);
        o.u2 = ddiv(a.ub1[x] * D1U + ((a.Dt * ru) * g.pm[x]) * g.pn[x], D2U);
        o.v2 = ddiv(a.vb1[x] * D1V + ((a.Dt * rv) * g.pm[x]) * g.pn[x], D2V);
    }
    return o;
}

// ubar_t2 / vbar_t2 at x before barotropicVelocityBC (the old content where not predicted).
template <typename R>
__device__ __forceinline__ R prd_u2p(const PredArgs<R> &a, const PrdTile<R> &t, long x, int comp) {
    const PrdMom<R> m = prd_mom(a, t, x);
    if (m.pd) return comp ? m.v2 : m.u2;
    return comp ? a.vb2[x] : a.ub2[x];
}

template <typename R>
__device__ __forceinline__ R prd_val(const PredArgs<R> &a) {
    return a.valp ? (R)a.valp[0] : a.val;
}

// Value after the program of field f (0 zeta, 1 ubar, 2 vbar) at a destination whose source
// code is s.
template <typename R>
__device__ __noinline__ R prd_bc_value(const PredArgs<R> &a, const PrdTile<R> &t, int f, int s) {
    if (s == -1) return R(0);
    if (s == -2) return f == 0 ? R(0) : prd_val(a);
    return f == 0 ? prd_z2p(a, s) : prd_u2p(a, t, s, f - 1);
}

// An edge-ring node: everything through the pure functions (or the tile); writes its own
// outputs.
template <typename R>
__device__ __noinline__ void prd_edge_node(const PredArgs<R> &a, const PrdTile<R> &t, long x) {
    const Geo<R> &g = a.g;
    const int j = fdiv((int)x, g.dI), i = (int)x - j * g.I;
    const bool in = rint_(i, j, g.I, g.J);
    // zeta: rzeta (interior), zeta_t2 (i, j != 0), then zetabc
    R rzx = R(0);
    if (in) rzx = prd_rz(a, x);
    const int mz = a.mz[x];
    R z2v;
    bool wz;
    if (mz == kBcNone) {
        wz = i != 0 && j != 0;
        z2v = wz ? a.z0[x] + a.Dt * (in ? rzx : a.rz[x]) : R(0);
    } else {
        wz = !(mz & kBcChained);
        z2v = wz ? prd_bc_value(a, t, 0, bc_src(mz)) : R(0);
    }
    const PrdMom<R> m = prd_mom(a, t, x);
    const int mu = a.mu[x], mv = a.mv[x];
    R u2 = m.u2, v2 = m.v2;
    bool wu = m.pd, wv = m.pd;
    if (mu != kBcNone) {
        wu = !(mu & kBcChained);
        if (wu) u2 = prd_bc_value(a, t, 1, bc_src(mu));
    }
    if (mv != kBcNone) {
        wv = !(mv & kBcChained);
        if (wv) v2 = prd_bc_value(a, t, 2, bc_src(mv));
    }
    // every read of old contents above; the writes touch only this node
    if (in) a.rz[x] = rzx;
    if (wz) a.z2[x] = z2v;
    if (m.in) {
        a.ru[x] = m.ru;
        a.rv[x] = m.rv;
    }
    if (wu) a.ub2[x] = u2;
    if (wv) a.vb2[x] = v2;
}

__device__ __forceinline__ bool prd_deep(int i, int j, int I, int J) {
    return i >= 2 && i <= I - 3 && j >= 2 && j <= J - 3;
}

// A deep node's inputs that both phases use, read once in phase 1 and kept in registers across
// the block's barrier: zeta_t1 and h at the node and its west and south neighbours, ubar_t1,
// vbar_t1, the metrics and zeta_t0 at the node.
template <typename R>
struct PrdNode {
    R z1p, z1w, z1s, hp, hw, hs, ub, vb, pm, pn, ou, ov, z0p;
};

// computeZetaRHS at a deep node (the operations of prd_rz in its order) through per-node base
// pointers, the neighbours at constant offsets, filling the node's kept inputs.
template <typename R>
__device__ __forceinline__ R prd_rz_keep(const PredArgs<R> &a, long x, PrdNode<R> &n) {
    const Geo<R> &g = a.g;
    const int I = g.I;
    const R *z = a.z1 + x, *h = g.h + x, *ub = a.ub1 + x, *vb = a.vb1 + x, *ou = g.on_u + x,
            *ov = g.om_v + x;
    n.z1p = z[0];
    n.z1w = z[-1];
    n.z1s = z[-I];
    n.hp = h[0];
    n.hw = h[-1];
    n.hs = h[-I];
    n.ub = ub[0];
    n.vb = vb[0];
    n.ou = ou[0];
    n.ov = ov[0];
    n.pm = g.pm[x];
    n.pn = g.pn[x];
    n.z0p = a.z0[x];
    const R Dp = n.z1p + n.hp, Dw = n.z1w + n.hw, De = z[1] + h[1];
    const R Ds = n.z1s + n.hs, Dn = z[I] + h[I];
    const R DUp = n.ub * ((Dp + Dw) * R(0.5));
    const R DUe = ub[1] * ((De + Dp) * R(0.5));
    const R DVp = n.vb * ((Dp + Ds) * R(0.5));
    const R DVn = vb[I] * ((Dn + Dp) * R(0.5));
    return (((DUe * ou[1] - DUp * n.ou) + (DVn * ov[I] - DVp * n.ov)) * n.pm) * n.pn;
}

// The fast path of a deep node: computeMomentumRHSPred + computeMomentumPred (the operations of
// prd_mom in its order) from the tile's zeta_t2 at x, x-1 and x-I and the node's kept inputs.
template <typename R>
__device__ __forceinline__ void prd_deep_mom_kept(const PredArgs<R> &a, long x, bool pd, R zp,
                                                  R zw, R zs, const PrdNode<R> &n) {
    const int I = a.g.I;
    const R *z0 = a.z0 + x;
    const R gp = a.w1 * zp + a.w * n.z0p;
    const R gw = a.w1 * zw + a.w * z0[-1];
    const R gs = a.w1 * zs + a.w * z0[-I];
    const R ru = (a.grav * n.ou) * (((n.hp + n.hw) * R(0.5)) * (gp - gw) + R(0.5) * (gp * gp - gw * gw));
    const R rv = (a.grav * n.ov) * (((n.hp + n.hs) * R(0.5)) * (gp - gs) + R(0.5) * (gp * gp - gs * gs));
    a.ru[x] = ru;
    a.rv[x] = rv;
    if (pd) {
        const R D1p = n.z1p + n.hp, D2p = zp + n.hp;
        const R D1U = (D1p + (n.z1w + n.hw)) * R(0.5);
        const R D2U = (D2p + (zw + n.hw)) * R(0.5);
        const R D1V = (D1p + (n.z1s + n.hs)) * R(0.5);
        const R D2V = (D2p + (zs + n.hs)) * R(0.5);
        a.ub2[x] = ddiv(n.ub * D1U + ((a.Dt * ru) * n.pm) * n.pn, D2U);
        a.vb2[x] = ddiv(n.vb * D1V + ((a.Dt * rv) * n.pm) * n.pn, D2V);
    }
}

// The ring nodes: 4 I nodes of rows 0, 1, J-2, J-1, then 4 (J-4) of columns 0, 1, I-2, I-1.
__device__ __forceinline__ long prd_ring_node(int e, int I, int J) {
    if (e < 4 * I) {
        const int r = e / I, i = e - r * I;
        const int j = r < 2 ? r : J - 4 + r;
        return (long)j * I + i;
    }
    const int f = e - 4 * I, c = f / (J - 4);
    const int i = c < 2 ? c : I - 4 + c;
    return (long)(2 + f - c * (J - 4)) * I + i;
}

// The first `ring_blocks` blocks take one ring node per thread through the pure functions;
// the others own tiles of 31 x 15 nodes, lane tx taking column i0-1+tx of the staged rows
// j0-1+ty and j0-1+ty+8 (lane 0 the west halo column, row 0 the south halo row), so every
// load of a warp is 32 consecutive nodes of one row.  A tile block fills its shared zeta_t2 for
// halo and ring nodes too (the deep nodes next to them read them) but writes only its own
// nodes' outputs, and leaves the ring nodes' outputs to the ring blocks.
__host__ __device__ __forceinline__ bool prd_inner_tile(int i0, int j0, int I, int J) {
    return i0 >= 3 && j0 >= 3 && i0 + kPredTX + 2 <= I && j0 + kPredTY + 2 <= J;
}

// Chained destinations: the last edge block, after every edge block's reads.  A thread
// reaches the barrier only after each of its loads has returned (every loaded value feeds a
// store or a branch before it), so once a block has counted itself, none of its reads of old
// contents is pending and the last edge block may overwrite them.
template <typename R>
__device__ __forceinline__ void prd_chained_tail(const PredArgs<R> &a, int tid, int edge_blocks) {
    __shared__ int s_last;
    __syncthreads();
    if (tid == 0) s_last = atomicAdd(a.counter, 1) == edge_blocks - 1;
    __syncthreads();
    if (!s_last) return;
    __threadfence();
    const BcProgram *ps[3] = {&a.pz, &a.pu, &a.pv};
    R v[3] = {R(0), R(0), R(0)};
    int d[3] = {-1, -1, -1};
#pragma unroll
    for (int f = 0; f < 3; ++f) {
        const BcProgram &p = *ps[f];
        if (tid < p.nch) {
            d[f] = p.dst_ch[tid];
            v[f] = __ldcg(a.chv + f * kMaxChained + tid);
        }
    }
    if (d[0] >= 0) a.z2[d[0]] = v[0];
    if (d[1] >= 0) a.ub2[d[1]] = v[1];
    if (d[2] >= 0) a.vb2[d[2]] = v[2];
    if (tid == 0) *a.counter = 0;
}

// Block 0 evaluates the chained entries' values first (the last edge block stores them).
template <typename R>
__device__ __forceinline__ void prd_chained_head(const PredArgs<R> &a, int tid, R (*sZ)[kPredTX + 1]) {
    const BcProgram *ps[3] = {&a.pz, &a.pu, &a.pv};
#pragma unroll
    for (int f = 0; f < 3; ++f)
        if (tid < ps[f]->nch)
            a.chv[f * kMaxChained + tid] =
                prd_bc_value(a, PrdTile<R>{sZ, -kPredTX - 2, -kPredTY - 2}, f, ps[f]->src_ch[tid]);
    __threadfence();   // ... visible before this block counts itself
}

template <typename R>
__global__ void __launch_bounds__(256, 5) k_pred2d(const __grid_constant__ PredArgs<R> a,
                                                int ring_blocks, int tiles_x, int edge_blocks) {
    pdl_enter();
    __shared__ R sZ[kPredTY + 1][kPredTX + 1];   // zeta_t2 after zetabc, (j0-1.., i0-1..)
    const Geo<R> &g = a.g;
    const int I = g.I, J = g.J;
    const int tx = threadIdx.x, ty = threadIdx.y;
    const int tid = ty * 32 + tx;
    const int bid = (int)blockIdx.x;
    int i0 = -kPredTX - 2, j0 = -kPredTY - 2;   // ring blocks: a tile no node falls in
    if (bid == 0) prd_chained_head(a, tid, sZ);
    if (bid < ring_blocks) {
        const int e = bid * 256 + tid;
        if (e < 4 * I + 4 * (J - 4)) prd_edge_node(a, PrdTile<R>{sZ, i0, j0}, prd_ring_node(e, I, J));
    } else {
        const int tb = bid - ring_blocks;
        i0 = (tb % tiles_x) * kPredTX;
        j0 = (tb / tiles_x) * kPredTY;
        const int i = i0 - 1 + tx;   // staged column tx (0: the west halo)
        // ---- phase 1: zeta_t2 (after zetabc) on the tile and its south/west halo ------------
        PrdNode<R> kept[2];   // a deep node's inputs, for phase 2
#pragma unroll
        for (int h = 0; h < 16; h += 8) {
            const int r = ty + h;   // staged row (0: the south halo)
            const int j = j0 - 1 + r;
            if (i >= 0 && j >= 0 && i < I && j < J) {
                const long x = (long)j * I + i;
                R z;
                if (prd_deep(i, j, I, J)) {
                    const R rz = prd_rz_keep(a, x, kept[h / 8]);
                    z = kept[h / 8].z0p + a.Dt * rz;
                    if (tx >= 1 && r >= 1) {   // the tile's own node (a halo node is its tile's)
                        a.rz[x] = rz;
                        a.z2[x] = z;
                    }
                } else {
                    z = prd_z2b(a, x);
                }
                sZ[r][tx] = z;
            }
        }
        __syncthreads();
        // ---- phase 2: momentum of the tile's deep nodes ----------------------------------------
#pragma unroll
        for (int h = 0; h < 16; h += 8) {
            const int r = ty + h;
            const int j = j0 - 1 + r;
            if (tx >= 1 && r >= 1 && i < I && j < J && prd_deep(i, j, I, J)) {
                const int q = j * I + i;
                const bool pd = q - fdiv(q, g.dJ) * J != 0 && q >= J;   // q % J != 0 (szJ)
                prd_deep_mom_kept(a, (long)q, pd, sZ[r][tx], sZ[r][tx - 1], sZ[r - 1][tx], kept[h / 8]);
            }
        }
        if (prd_inner_tile(i0, j0, I, J)) return;   // uniform over the block: no barrier below
    }

    prd_chained_tail(a, tid, edge_blocks);
}

// ---- the paired form (grids with an even row length) -------------------------------------
// Lane tx of a 32 x 16 block takes the node pair (x, x+1), x = j I + i with i even, of staged
// row ty: with I even every such pair starts on an 8-byte (FP32) or 16-byte (FP64) boundary, so
// each array's two values arrive in one vector load, and the pair shares the neighbours that
// the scalar form loads twice (x's east node is x+1's own, x+1's west node is x's own).  Each
// node's arithmetic is prd_rz_keep's and prd_deep_mom_kept's, operation for operation (the
// shared terms are the same expressions on the same operands), so the FP64 build reproduces
// the scalar form bit for bit.  A tile is 62 x 15 nodes, staged with two west halo columns
// (the first keeps the pairs aligned; only the second is read) and one south halo row: 64 x 16
// nodes, one staged row per warp.  With I even a pair is deep in both nodes or in neither.
constexpr int kPairTX = 62, kPairTY = 15;   // (the 8-row form's tiles are 62 x 7)

template <typename R>
struct Vec2;
template <>
struct Vec2<float> {
    using T = float2;
};
template <>
struct Vec2<double> {
    using T = double2;
};
template <typename R>
__device__ __forceinline__ void ld2(const R *__restrict__ q, R &a, R &b) {
    const typename Vec2<R>::T t = *reinterpret_cast<const typename Vec2<R>::T *>(q);
    a = t.x;
    b = t.y;
}
template <typename R>
__device__ __forceinline__ void st2(R *__restrict__ q, R a, R b) {
    typename Vec2<R>::T t;
    t.x = a;
    t.y = b;
    *reinterpret_cast<typename Vec2<R>::T *>(q) = t;
}

// A deep pair's inputs that both phases use (node a = x, node b = x+1).
template <typename R>
struct PrdPair {
    R z1w, z1a, z1b, z1sa, z1sb, hw, ha, hb, hsa, hsb;
    R uba, ubb, vba, vbb, pma, pmb, pna, pnb, oua, oub, ova, ovb, z0a, z0b;
    R z0w, z0sa, z0sb;   // zeta_t0 west and south of the pair (the momentum's), loaded with the rest
};

// computeZetaRHS at both nodes of a deep pair; fills the pair's kept inputs.
template <typename R>
__device__ __forceinline__ void prd_rz_pair(const PredArgs<R> &a, long x, PrdPair<R> &n, R &rza,
                                            R &rzb) {
    const Geo<R> &g = a.g;
    const int I = g.I;
    const R *z = a.z1 + x, *h = g.h + x, *ub = a.ub1 + x, *vb = a.vb1 + x, *ou = g.on_u + x,
            *ov = g.om_v + x;
    ld2(z, n.z1a, n.z1b);
    n.z1w = z[-1];
    const R z1e = z[2];
    ld2(z - I, n.z1sa, n.z1sb);
    R zna, znb;
    ld2(z + I, zna, znb);
    ld2(h, n.ha, n.hb);
    n.hw = h[-1];
    const R he = h[2];
    ld2(h - I, n.hsa, n.hsb);
    R hna, hnb;
    ld2(h + I, hna, hnb);
    ld2(ub, n.uba, n.ubb);
    const R ube = ub[2];
    R vna, vnb;
    if (a.vb1_zero) {
        n.vba = n.vbb = vna = vnb = R(0);
    } else {
        ld2(vb, n.vba, n.vbb);
        ld2(vb + I, vna, vnb);
    }
    ld2(ou, n.oua, n.oub);
    const R oue = ou[2];
    ld2(ov, n.ova, n.ovb);
    R ovna, ovnb;
    ld2(ov + I, ovna, ovnb);
    ld2(g.pm + x, n.pma, n.pmb);
    ld2(g.pn + x, n.pna, n.pnb);
    ld2(a.z0 + x, n.z0a, n.z0b);
    n.z0w = a.z0[x - 1];
    ld2(a.z0 + x - I, n.z0sa, n.z0sb);
    // node a
    const R Dpa = n.z1a + n.ha, Dwa = n.z1w + n.hw, Dpb = n.z1b + n.hb;
    const R Dsa = n.z1sa + n.hsa, Dna = zna + hna;
    const R DUpa = n.uba * ((Dpa + Dwa) * R(0.5));
    const R DUpb = n.ubb * ((Dpb + Dpa) * R(0.5));   // node a's east flux, node b's west
    const R DVpa = n.vba * ((Dpa + Dsa) * R(0.5));
    const R DVna = vna * ((Dna + Dpa) * R(0.5));
    rza = (((DUpb * n.oub - DUpa * n.oua) + (DVna * ovna - DVpa * n.ova)) * n.pma) * n.pna;
    // node b
    const R Deb = z1e + he, Dsb = n.z1sb + n.hsb, Dnb = znb + hnb;
    const R DUeb = ube * ((Deb + Dpb) * R(0.5));
    const R DVpb = n.vbb * ((Dpb + Dsb) * R(0.5));
    const R DVnb = vnb * ((Dnb + Dpb) * R(0.5));
    rzb = (((DUeb * oue - DUpb * n.oub) + (DVnb * ovnb - DVpb * n.ovb)) * n.pmb) * n.pnb;
}

// The momentum of a deep pair from the tile's zeta_t2: za, zb at the nodes, zw west of a, zsa
// and zsb south of them.
template <typename R>
__device__ __forceinline__ void prd_mom_pair(const PredArgs<R> &a, long x, bool pda, bool pdb,
                                             R za, R zb, R zw, R zsa, R zsb, const PrdPair<R> &n) {
    const R gpa = a.w1 * za + a.w * n.z0a;
    const R gw = a.w1 * zw + a.w * n.z0w;
    const R gsa = a.w1 * zsa + a.w * n.z0sa;
    const R gpb = a.w1 * zb + a.w * n.z0b;
    const R gsb = a.w1 * zsb + a.w * n.z0sb;
    const R rua = (a.grav * n.oua) * (((n.ha + n.hw) * R(0.5)) * (gpa - gw) + R(0.5) * (gpa * gpa - gw * gw));
    const R rva = (a.grav * n.ova) * (((n.ha + n.hsa) * R(0.5)) * (gpa - gsa) + R(0.5) * (gpa * gpa - gsa * gsa));
    const R rub = (a.grav * n.oub) * (((n.hb + n.ha) * R(0.5)) * (gpb - gpa) + R(0.5) * (gpb * gpb - gpa * gpa));
    const R rvb = (a.grav * n.ovb) * (((n.hb + n.hsb) * R(0.5)) * (gpb - gsb) + R(0.5) * (gpb * gpb - gsb * gsb));
    st2(a.ru + x, rua, rub);
    st2(a.rv + x, rva, rvb);
    if (!pda && !pdb) return;
    const R D1pa = n.z1a + n.ha, D2pa = za + n.ha, D1pb = n.z1b + n.hb, D2pb = zb + n.hb;
    const R ua = ddiv(n.uba * ((D1pa + (n.z1w + n.hw)) * R(0.5)) + ((a.Dt * rua) * n.pma) * n.pna,
                      (D2pa + (zw + n.hw)) * R(0.5));
    const R va = ddiv(n.vba * ((D1pa + (n.z1sa + n.hsa)) * R(0.5)) + ((a.Dt * rva) * n.pma) * n.pna,
                      (D2pa + (zsa + n.hsa)) * R(0.5));
    const R ub = ddiv(n.ubb * ((D1pb + D1pa) * R(0.5)) + ((a.Dt * rub) * n.pmb) * n.pnb,
                      (D2pb + D2pa) * R(0.5));
    const R vb = ddiv(n.vbb * ((D1pb + (n.z1sb + n.hsb)) * R(0.5)) + ((a.Dt * rvb) * n.pmb) * n.pnb,
                      (D2pb + (zsb + n.hsb)) * R(0.5));
    if (pda && pdb) {
        st2(a.ub2 + x, ua, ub);
        st2(a.vb2 + x, va, vb);
    } else if (pda) {
        a.ub2[x] = ua;
        a.vb2[x] = va;
    } else {
        a.ub2[x + 1] = ub;
        a.vb2[x + 1] = vb;
    }
}

__host__ __device__ __forceinline__ bool prd_inner_pair_tile(int i0, int j0, int I, int J,
                                                             int ty_own = kPairTY) {
    // every staged node (columns i0-2 .. i0+61, rows j0-1 .. j0+ty_own-1) deep
    return i0 >= 4 && j0 >= 3 && i0 + kPairTX + 2 <= I && j0 + ty_own + 2 <= J;
}

// The kept inputs stay in registers across the block's barrier (64 registers, two blocks per
// SM): a form that read them again after the barrier (40 registers, three blocks per SM) took
// the basin4 loop to 4.72 ms against 4.30.
// ROWS staged rows per block (one per warp): 16 (tiles 62 x 15, two blocks per SM) or 8 (62 x 7,
// four blocks per SM).
template <typename R, int ROWS>
__global__ void __launch_bounds__(32 * ROWS, ROWS == 16 ? 2 : 4) k_pred2d_pair(
        const __grid_constant__ PredArgs<R> a, int ring_blocks, int tiles_x, int edge_blocks) {
    pdl_enter();
    constexpr int TY = ROWS - 1;
    __shared__ R sZ[ROWS][kPairTX + 2];   // zeta_t2 after zetabc, (j0-1.., i0-2..)
    __shared__ R sDummy[kPredTY + 1][kPredTX + 1];
    const Geo<R> &g = a.g;
    const int I = g.I, J = g.J;
    const int tx = threadIdx.x, ty = threadIdx.y;
    const int tid = ty * 32 + tx;
    const int bid = (int)blockIdx.x;
    if (bid == 0) prd_chained_head(a, tid, sDummy);
    if (bid < ring_blocks) {
        const int e = bid * (32 * ROWS) + tid;
        if (e < 4 * I + 4 * (J - 4))
            prd_edge_node(a, PrdTile<R>{sDummy, -kPredTX - 2, -kPredTY - 2}, prd_ring_node(e, I, J));
    } else {
        const int tb = bid - ring_blocks;
        const int i0 = (tb % tiles_x) * kPairTX, j0 = (tb / tiles_x) * TY;
        const int i = i0 - 2 + 2 * tx;   // the pair (i, i+1) of staged columns 2 tx, 2 tx + 1
        const int r = ty;                // staged row (0: the south halo)
        const int j = j0 - 1 + r;
        const bool live = i >= 0 && j >= 0 && i < I && j < J;   // I even: i + 1 < I too
        const bool deep = live && prd_deep(i, j, I, J);       // ... and i + 1 deep alike
        const long x = (long)j * I + i;
        PrdPair<R> kept;
        // ---- phase 1: zeta_t2 (after zetabc) on the tile and its halo -----------------------
        if (deep) {
            R rza, rzb;
            prd_rz_pair(a, x, kept, rza, rzb);
            const R za = kept.z0a + a.Dt * rza, zb = kept.z0b + a.Dt * rzb;
            if (tx >= 1 && r >= 1) {   // the tile's own pair
                st2(a.rz + x, rza, rzb);
                st2(a.z2 + x, za, zb);
            }
            sZ[r][2 * tx] = za;
            sZ[r][2 * tx + 1] = zb;
        } else if (live) {
            sZ[r][2 * tx] = prd_z2b(a, x);
            sZ[r][2 * tx + 1] = prd_z2b(a, x + 1);
        }
        __syncthreads();
        // ---- phase 2: momentum of the tile's deep pairs ---------------------------------------
        if (deep && tx >= 1 && r >= 1) {
            const int qa = j * I + i, qb = qa + 1;
            const bool pda = qa - fdiv(qa, g.dJ) * J != 0 && qa >= J;   // q % J != 0 (szJ)
            const bool pdb = qb - fdiv(qb, g.dJ) * J != 0 && qb >= J;
            prd_mom_pair(a, x, pda, pdb, sZ[r][2 * tx], sZ[r][2 * tx + 1], sZ[r][2 * tx - 1],
                         sZ[r - 1][2 * tx], sZ[r - 1][2 * tx + 1], kept);
        }
        if (prd_inner_pair_tile(i0, j0, I, J, TY)) return;   // uniform over the block
    }
    prd_chained_tail(a, tid, edge_blocks);
}

template <typename R>
cudaError_t Ops<R>::pred2d(const sf_ctx *c, R *z0, R *z1, R *z2, R *ub1, R *vb1, R *ub2, R *vb2,
                           R *rz, R *ru, R *rv, double Dt, double weight, double val,
                           const double *valp, cudaStream_t s, int vb1_zero) {
    PredArgs<R> a;
    a.vb1_zero = vb1_zero;
    a.g = geo(c);
    a.z0 = z0;
    a.z1 = z1;
    a.ub1 = ub1;
    a.vb1 = vb1;
    a.z2 = z2;
    a.rz = rz;
    a.ru = ru;
    a.rv = rv;
    a.ub2 = ub2;
    a.vb2 = vb2;
    a.mz = c->bcmap;
    a.mu = c->bcmap + c->s2;
    a.mv = c->bcmap + 2 * c->s2;
    a.Dt = (R)Dt;
    a.w1 = (R)(1.0 - weight);
    a.w = (R)weight;
    a.grav = (R)10.0;
    a.val = (R)val;
    a.valp = valp;
    a.pz = c->zbc;
    a.pu = c->ubc;
    a.pv = c->vbc;
    a.counter = c->pred_counter;
    a.chv = reinterpret_cast<R *>(reinterpret_cast<char *>(c->pred_counter) + 256);
    // the paired form where every row starts on a vector boundary in every array
    bool pair = c->pred_pair && (c->I % 2) == 0;
    {
        const void *ptrs[] = {z0, z1, z2, ub1, vb1, ub2, vb2, rz, ru, rv, a.g.h, a.g.pm, a.g.pn,
                              a.g.on_u, a.g.om_v};
        for (const void *q : ptrs) pair = pair && (reinterpret_cast<uintptr_t>(q) % (2 * sizeof(R))) == 0;
    }
    if (pair) {
        const int rows = c->pred_pair == 2 ? 8 : 16, TY = rows - 1, nt = 32 * rows;
        const int tiles_x = (c->I + kPairTX - 1) / kPairTX, tiles_y = (c->J + TY - 1) / TY;
        const int ring_blocks = (4 * c->I + 4 * (c->J - 4) + nt - 1) / nt;
        int inner_x = 0, inner_y = 0;
        for (int tx = 0; tx < tiles_x; ++tx)
            inner_x += prd_inner_pair_tile(tx * kPairTX, 3, c->I, 3 + TY + 2, TY);
        for (int ty = 0; ty < tiles_y; ++ty)
            inner_y += prd_inner_pair_tile(4, ty * TY, 4 + kPairTX + 2, c->J, TY);
        const int edge_blocks = ring_blocks + tiles_x * tiles_y - inner_x * inner_y;
        const dim3 grid((unsigned)(ring_blocks + tiles_x * tiles_y));
        if (rows == 8)
            return launch_dep(c, k_pred2d_pair<R, 8>, grid, dim3(32, 8), 0, s, a, ring_blocks,
                              tiles_x, edge_blocks);
        return launch_dep(c, k_pred2d_pair<R, 16>, grid, dim3(32, 16), 0, s, a, ring_blocks,
                          tiles_x, edge_blocks);
    }
    const int tiles_x = (c->I + kPredTX - 1) / kPredTX, tiles_y = (c->J + kPredTY - 1) / kPredTY;
    const int ring_blocks = (4 * c->I + 4 * (c->J - 4) + 255) / 256;
    // the blocks counted before the chained writes: the ring blocks and the tiles that are not
    // inner (the condition is separable: inner columns of tiles times inner rows of tiles)
    int inner_x = 0, inner_y = 0;
    for (int tx = 0; tx < tiles_x; ++tx) inner_x += prd_inner_tile(tx * kPredTX, 3, c->I, 3 + kPredTY + 2);
    for (int ty = 0; ty < tiles_y; ++ty) inner_y += prd_inner_tile(3, ty * kPredTY, 3 + kPredTX + 2, c->J);
    const int edge_blocks = ring_blocks + tiles_x * tiles_y - inner_x * inner_y;
    return launch_dep(c, k_pred2d<R>, dim3((unsigned)(ring_blocks + tiles_x * tiles_y)), dim3(32, 8),
                      0, s, a, ring_blocks, tiles_x, edge_blocks);
}

}  // namespace sf
