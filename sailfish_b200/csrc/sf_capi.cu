// C ABI of libsailfish_b200.so (declarations and reference citations: include/sailfish_b200.h).
//
// Host-side runtime: context creation (grid snapshot, boundary programs), argument checks,
// precision dispatch and error reporting.  No C++ exception crosses the boundary.
#include <cuda_runtime.h>

#include <cmath>
#include <cstdio>
#include <cstring>
#include <new>
#include <type_traits>
#include <string>
#include <unordered_map>
#include <vector>

#include "sf_internal.h"

namespace {

thread_local std::string g_err;

int fail(int code, const std::string &msg) {
    g_err = msg;
    return code;
}

int cuda_fail(cudaError_t e, const char *where) {
    return fail(SF_ECUDA, std::string(where) + ": " + cudaGetErrorString(e));
}

#define SF_TRY_CUDA(expr, where)                      \
    do {                                              \
        cudaError_t e_ = (expr);                      \
        if (e_ != cudaSuccess) return cuda_fail(e_, where); \
    } while (0)

template <typename T>
int upload(T **dst, const T *src, size_t n, const char *what) {
    *dst = nullptr;
    if (n == 0) return SF_OK;
    if (!src) return fail(SF_EINVAL, std::string("missing host array: ") + what);
    cudaError_t e = cudaMalloc((void **)dst, n * sizeof(T));
    if (e != cudaSuccess) return fail(SF_ENOMEM, std::string("cudaMalloc ") + what);
    e = cudaMemcpy(*dst, src, n * sizeof(T), cudaMemcpyHostToDevice);
    if (e != cudaSuccess) return cuda_fail(e, what);
    return SF_OK;
}

int upload_real(sf_ctx *c, void **dst, const double *src, size_t n, const char *what) {
    if (c->prec == SF_FP64) return upload(reinterpret_cast<double **>(dst), src, n, what);
    if (!src) return fail(SF_EINVAL, std::string("missing host array: ") + what);
    std::vector<float> tmp(n);
    for (size_t k = 0; k < n; ++k) tmp[k] = (float)src[k];
    return upload(reinterpret_cast<float **>(dst), tmp.data(), n, what);
}

// One boundary scatter of the reference: setBC (constant) or copyBC (node to node).
struct BcOp {
    const int32_t *idx1;
    const int32_t *idx2;   // nullptr for setBC
    int n;
    int code;              // setBC value: -1 -> 0.0, -2 -> time-dependent value
};

// Reduces a sequence of scatters, executed in order and each in thread order (what the
// reference's sequential launches amount to when no two threads of a launch conflict, and
// what its host-compiled form does when they do), to one gather program (sf::BcProgram).
int resolve(const std::vector<BcOp> &ops, long s2, std::vector<int> &dst, std::vector<int> &src) {
    std::unordered_map<int, int> cur;   // node -> symbolic value
    std::vector<int> order;
    auto get = [&](int node) {
        auto it = cur.find(node);
        return it == cur.end() ? node : it->second;
    };
    for (const BcOp &op : ops) {
        for (int k = 0; k < op.n; ++k) {
            const int d = op.idx1[k];
            if (d < 0 || d >= s2) return fail(SF_EINVAL, "boundary index out of range");
            int val;
            if (op.idx2) {
                const int s = op.idx2[k];
                if (s < 0 || s >= s2) return fail(SF_EINVAL, "boundary source index out of range");
                val = get(s);
            } else {
                val = op.code;
            }
            if (cur.find(d) == cur.end()) order.push_back(d);
            cur[d] = val;
        }
    }
    dst.clear();
    src.clear();
    for (int d : order) {
        const int v = cur[d];
        if (v == d) continue;
        dst.push_back(d);
        src.push_back(v);
    }
    return SF_OK;
}

// A boundary program on the host: independent entries (di <- si), chained entries (dc <- sc)
// in groups [gofs[g], gofs[g+1]).
struct ProgHost {
    std::vector<int> di, si, dc, sc, gofs;
};

int upload_program(sf::BcProgram &p, const ProgHost &h) {
    p.n = (int)h.di.size();
    p.nch = (int)h.dc.size();
    p.ngr = h.gofs.empty() ? 0 : (int)h.gofs.size() - 1;
    int rc = upload(&p.dst, h.di.data(), h.di.size(), "boundary program");
    if (!rc) rc = upload(&p.src, h.si.data(), h.si.size(), "boundary program");
    if (!rc) rc = upload(&p.dst_ch, h.dc.data(), h.dc.size(), "boundary program");
    if (!rc) rc = upload(&p.src_ch, h.sc.data(), h.sc.size(), "boundary program");
    if (!rc && p.ngr > 0) rc = upload(&p.gofs, h.gofs.data(), h.gofs.size(), "boundary program");
    return rc;
}

int build_program(ProgHost &out, const std::vector<BcOp> &ops, long s2) {
    std::vector<int> d, s;
    int rc = resolve(ops, s2, d, s);
    if (rc) return rc;
    // Partition (see sf::BcProgram): chained = entries reading another entry's destination,
    // plus the entries writing those destinations.
    std::unordered_map<int, int> dst_of;
    for (size_t k = 0; k < d.size(); ++k) dst_of[d[k]] = (int)k;
    std::vector<char> ch(d.size(), 0);
    for (size_t k = 0; k < d.size(); ++k)
        if (s[k] >= 0 && dst_of.count(s[k])) {
            ch[k] = 1;
            ch[dst_of[s[k]]] = 1;
        }
    std::vector<int> di, si, dc, sc;
    for (size_t k = 0; k < d.size(); ++k) {
        if (ch[k]) {
            dc.push_back(d[k]);
            sc.push_back(s[k]);
        } else {
            di.push_back(d[k]);
            si.push_back(s[k]);
        }
    }
    if ((int)dc.size() > sf::kMaxChained)
        return fail(SF_EUNSUPPORTED, "boundary lists with more than 32 chained entries");
    out.di = std::move(di);
    out.si = std::move(si);
    out.dc = std::move(dc);
    out.sc = std::move(sc);
    out.gofs.clear();
    if (!out.dc.empty()) out.gofs = {0, (int)out.dc.size()};
    return SF_OK;
}

// Appends a member's program to an ensemble's, its node indices offset into the pools.
void append_program(ProgHost &all, const ProgHost &m, long off) {
    auto sh = [&](int v) { return v >= 0 ? (int)(v + off) : v; };
    for (size_t k = 0; k < m.di.size(); ++k) {
        all.di.push_back(sh(m.di[k]));
        all.si.push_back(sh(m.si[k]));
    }
    if (m.dc.empty()) return;
    if (all.gofs.empty()) all.gofs.push_back(0);
    for (size_t k = 0; k < m.dc.size(); ++k) {
        all.dc.push_back(sh(m.dc[k]));
        all.sc.push_back(sh(m.sc[k]));
    }
    all.gofs.push_back((int)all.dc.size());
}

void free_ctx(sf_ctx *c) {
    if (!c) return;
    for (void *m : c->metrics) cudaFree(m);
    cudaFree(c->hd);
    cudaFree(c->vert);
    cudaFree(c->bcfield);
    cudaFree(c->utype);
    cudaFree(c->vtype);
    for (auto &g : c->graphs)
        if (g.exec) cudaGraphExecDestroy(g.exec);
    if (c->cap) cudaStreamDestroy(c->cap);
    cudaFree(c->d_bcval);
    cudaFree(c->closure_x);
    cudaFree(c->bcmap);
    cudaFree(c->pred_counter);
    for (sf::BcProgram *p : {&c->zbc, &c->ubc, &c->vbc}) {
        cudaFree(p->dst);
        cudaFree(p->src);
        cudaFree(p->dst_ch);
        cudaFree(p->src_ch);
        cudaFree(p->gofs);
    }
    cudaFree(c->members);
    cudaFree(c->bm_pt);
    cudaFree(c->bm_128);
    for (int2 *b : c->bm_tile) cudaFree(b);
    cudaFree(c->bm_pipe);
    delete[] c->h_off2;
    delete[] c->h_off3;
    delete[] c->h_offN;
    cudaFree(c->check_dev);
    if (c->check_host) cudaFreeHost(c->check_host);
    cudaFree(c->dev_err);
    delete c;
}

inline cudaStream_t S(sf_stream s) { return reinterpret_cast<cudaStream_t>(s); }

// Dispatch a launcher on the context precision; `body` is a generic lambda taking a type tag.
template <typename F>
int dispatch(const sf_ctx *c, const char *name, F body) {
    if (!c) return fail(SF_EINVAL, "null context");
    cudaError_t e;
    if (c->prec == SF_FP64) e = body((double *)nullptr);
    else e = body((float *)nullptr);
    if (e != cudaSuccess) return cuda_fail(e, name);
    return SF_OK;
}

const double kBcOmega = 0.0002;   // fake clamped boundary (barotropicVelocityBC.py:21-22,
                                  // step3D_uv.kernels.cpp:338-339)

}  // namespace

extern "C" {

int sf_version(void) { return 1; }

const char *sf_last_error(void) { return g_err.c_str(); }

int sf_ctx_precision(const sf_ctx *ctx) { return ctx ? ctx->prec : SF_EINVAL; }

}  // extern "C"

namespace {
int validate_desc(const sf_grid_desc *d) {
    if (d->precision != SF_FP64 && d->precision != SF_FP32)
        return fail(SF_EDTYPE, "precision must be SF_FP64 or SF_FP32");
    if (d->L < 4 || d->M < 4) return fail(SF_EINVAL, "grid too small (need L, M >= 4)");
    if (d->N < 5 || d->N > 64)
        return fail(SF_EINVAL, "N must be in [5, 64]: the reference's verticalAdvection reads "
                               "levels up to 5 (rhs_kernels.cpp:172) and columns are held per thread");
    if (d->Vtransform != 1 && d->Vtransform != 2) return fail(SF_EINVAL, "Vtransform must be 1 or 2");
    if (!d->h || !d->pm || !d->pn || !d->on_u || !d->om_v || !d->fomn)
        return fail(SF_EINVAL, "missing metric arrays");
    if (!d->sc_r || !d->sc_w || !d->Cs_r || !d->Cs_w) return fail(SF_EINVAL, "missing S-coordinate tables");
    if (!d->zeta_field_idx2 || !d->uvel_field_type || !d->vvel_field_type)
        return fail(SF_EINVAL, "missing boundary maps");
    const long s2 = (long)(d->L + 1) * (d->M + 1);
    if (s2 >= (1L << 31)) return fail(SF_EINVAL, "grid too large: (L+1)(M+1) must be below 2^31");
    for (long k = 0; k < s2; ++k)
        if (d->vvel_field_type[k] > 0 && (d->vvel_field_type[k] & (1 << 4)) == 0 &&
            (d->vvel_field_type[k] & (1 << 3)) == 0 && (d->vvel_field_type[k] & (1 << 6)) != 0)
            return fail(SF_EUNSUPPORTED, "gradient 3D v boundary: the reference reads past the "
                                         "boundary map (step3D_uv.kernels.cpp:363)");
    if (d->n_vbar_grad > d->n_ubar_grad)
        return fail(SF_EUNSUPPORTED, "vbar gradient list longer than the ubar list the reference "
                                     "copies it from (barotropicVelocityBC.py:30-31)");
    return SF_OK;
}

// The three boundary programs of one grid, on the host.
int build_programs(const sf_grid_desc *d, long s2, ProgHost &z, ProgHost &u, ProgHost &v) {
    int rc = build_program(z, {{d->zeta_copy_idx1, d->zeta_copy_idx2, d->n_zeta_copy, 0}}, s2);
    if (!rc)
        rc = build_program(u,
                           {{d->ubar_closed_idx, nullptr, d->n_ubar_closed, -1},
                            {d->ubar_clamped_idx, nullptr, d->n_ubar_clamped, -2},
                            {d->ubar_grad_idx1, d->ubar_grad_idx2, d->n_ubar_grad, 0}},
                           s2);
    if (!rc)
        rc = build_program(v,
                           {{d->vbar_closed_idx, nullptr, d->n_vbar_closed, -1},
                            {d->vbar_grad_idx1, d->ubar_grad_idx2, d->n_vbar_grad, 0}},
                           s2);
    return rc;
}

// Per-node maps of the three boundary programs for the fused predictor (sf_pred2d.cuh): code
// (source + 2) | chained flag at each destination, kBcNone elsewhere.  The fused form is used
// only when every destination lies in the outer two-cell ring of the grid and no node is a
// destination twice; otherwise the context keeps the four-launch predictor.
int build_pred_maps(sf_ctx *c, const ProgHost &Z, const ProgHost &U, const ProgHost &V) {
    c->pred_ok = 0;
    const long s2 = c->s2;
    const int I = c->I, J = c->J;
    if (s2 >= (1L << 29) || I < 6 || J < 6) return SF_OK;
    std::vector<int> map(3 * (size_t)s2, sf::kBcNone);
    const ProgHost *ps[3] = {&Z, &U, &V};
    for (int f = 0; f < 3; ++f) {
        const ProgHost &p = *ps[f];
        for (int ch = 0; ch < 2; ++ch) {
            const std::vector<int> &dd = ch ? p.dc : p.di, &ss = ch ? p.sc : p.si;
            for (size_t k = 0; k < dd.size(); ++k) {
                const int x = dd[k], i = x % I, j = x / I;
                if (i >= 2 && i <= I - 3 && j >= 2 && j <= J - 3) return SF_OK;
                int &m = map[(size_t)f * s2 + x];
                if (m != sf::kBcNone) return SF_OK;
                m = (ss[k] + 2) | (ch ? sf::kBcChained : 0);
            }
        }
    }
    int rc = upload(&c->bcmap, map.data(), map.size(), "boundary maps");
    if (rc == SF_OK) {
        // the counter, then (at byte 256) the chained entries' values, 3 x kMaxChained
        if (cudaMalloc(&c->pred_counter, 256 + 3 * sf::kMaxChained * sizeof(double)) != cudaSuccess)
            return fail(SF_ENOMEM, "cudaMalloc predictor counter");
        if (cudaMemset(c->pred_counter, 0, sizeof(int)) != cudaSuccess)
            return fail(SF_ECUDA, "cudaMemset predictor counter");
        c->pred_ok = 1;
    }
    return rc;
}

template <typename R>
int upload_members(sf_ctx *c, const sf_grid_desc *d, int n, const std::vector<long> &off2,
                   const std::vector<long> &off3, const std::vector<long> &offN,
                   const std::vector<long> &voff) {
    std::vector<sf::Member<R>> mt(n);
    for (int m = 0; m < n; ++m) {
        sf::Geo<R> &g = mt[m].g;
        g.I = d[m].L + 1;
        g.J = d[m].M + 1;
        g.dI = sf::make_fastdiv(g.I);
        g.dJ = sf::make_fastdiv(g.J);
        g.N = d[m].N;
        g.s2 = (long)g.I * g.J;
        const R *const *mp = reinterpret_cast<const R *const *>(c->metrics);
        g.h = mp[0] + off2[m];
        g.pm = mp[1] + off2[m];
        g.pn = mp[2] + off2[m];
        g.on_u = mp[3] + off2[m];
        g.om_v = mp[4] + off2[m];
        g.fomn = mp[5] + off2[m];
        g.hd = c->hd + off2[m];
        g.sc_r = c->vert + voff[m];
        g.sc_w = g.sc_r + g.N;
        g.Cs_r = g.sc_w + g.N + 1;
        g.Cs_w = g.Cs_r + g.N;
        g.hc = d[m].hc;
        g.Vtransform = d[m].Vtransform;
        g.bcfield = c->bcfield + off2[m];
        g.utype = c->utype + off2[m];
        g.vtype = c->vtype + off2[m];
        g.ref_threads = 512L * (g.s2 / 512 + 1);
        mt[m].off2 = off2[m];
        mt[m].off3 = off3[m];
        mt[m].offN = offN[m];
        for (int v = 0; v < sf::kRhsTiles; ++v)
            mt[m].ntx[v] = (g.I + sf::kRhsTileX[v] - 1) / sf::kRhsTileX[v];
    }
    return upload(reinterpret_cast<sf::Member<R> **>(&c->members), mt.data(), mt.size(), "members");
}
}  // namespace

extern "C" {

int sf_ctx_create_ensemble(const sf_grid_desc *d, int n, sf_ctx **out) {
    if (!d || !out || n < 1) return fail(SF_EINVAL, "null argument");
    *out = nullptr;
    for (int m = 0; m < n; ++m) {
        if (d[m].precision != d[0].precision) return fail(SF_EDTYPE, "members differ in precision");
        if (const int rc = validate_desc(&d[m])) return rc;
    }
    sf_ctx *c = new (std::nothrow) sf_ctx();
    if (!c) return fail(SF_ENOMEM, "host allocation");
    c->prec = d[0].precision;
    c->nmem = n;
    cudaGetDevice(&c->device);
    // pool layout: members one after another, each region padded to 32 elements
    auto pad = [](long x) { return (x + 31) / 32 * 32; };
    std::vector<long> off2(n), off3(n), offN(n), voff(n);
    long t2 = 0, t3 = 0, tN = 0, tv = 0;
    for (int m = 0; m < n; ++m) {
        const long s2 = (long)(d[m].L + 1) * (d[m].M + 1);
        off2[m] = t2;
        off3[m] = t3;
        offN[m] = tN;
        voff[m] = tv;
        t2 += pad(s2);
        t3 += pad((d[m].N + 1) * s2);
        tN += pad(d[m].N * s2);
        tv += 4 * d[m].N + 2;
        if (d[m].N > c->maxN) c->maxN = d[m].N;
    }
    c->tot2 = t2;
    c->tot3 = t3;
    c->totN = tN;
    c->s2 = t2;            // pool-wide operations (accumulator clears) cover every member
    c->N = c->maxN;
    c->I = c->J = 0;
    c->L = c->M = 0;
    c->h_off2 = new long[n];
    c->h_off3 = new long[n];
    c->h_offN = new long[n];
    for (int m = 0; m < n; ++m) {
        c->h_off2[m] = off2[m];
        c->h_off3[m] = off3[m];
        c->h_offN[m] = offN[m];
    }
    int rc = SF_OK;
    {   // metric pools
        const char *mn[6] = {"h", "pm", "pn", "on_u", "om_v", "fomn"};
        for (int k = 0; k < 6 && rc == SF_OK; ++k) {
            std::vector<double> pool(t2, 0.0);
            for (int m = 0; m < n; ++m) {
                const double *src[6] = {d[m].h, d[m].pm, d[m].pn, d[m].on_u, d[m].om_v, d[m].fomn};
                const long s2 = (long)(d[m].L + 1) * (d[m].M + 1);
                std::copy(src[k], src[k] + s2, pool.begin() + off2[m]);
            }
            rc = upload_real(c, &c->metrics[k], pool.data(), (size_t)t2, mn[k]);
            if (k == 0 && rc == SF_OK) rc = upload(&c->hd, pool.data(), (size_t)t2, "h");
        }
    }
    if (rc == SF_OK) {
        std::vector<double> v;
        for (int m = 0; m < n; ++m) {
            const int N = d[m].N;
            v.insert(v.end(), d[m].sc_r, d[m].sc_r + N);
            v.insert(v.end(), d[m].sc_w, d[m].sc_w + N + 1);
            v.insert(v.end(), d[m].Cs_r, d[m].Cs_r + N);
            v.insert(v.end(), d[m].Cs_w, d[m].Cs_w + N + 1);
        }
        rc = upload(&c->vert, v.data(), v.size(), "S-coordinate tables");
    }
    if (rc == SF_OK) {
        std::vector<int> bf(t2, 0), ut(t2, 0), vt(t2, 0);
        for (int m = 0; m < n; ++m) {
            const long s2 = (long)(d[m].L + 1) * (d[m].M + 1);
            std::copy(d[m].zeta_field_idx2, d[m].zeta_field_idx2 + s2, bf.begin() + off2[m]);
            std::copy(d[m].uvel_field_type, d[m].uvel_field_type + s2, ut.begin() + off2[m]);
            std::copy(d[m].vvel_field_type, d[m].vvel_field_type + s2, vt.begin() + off2[m]);
        }
        rc = upload(&c->bcfield, bf.data(), bf.size(), "zeta_field_idx2");
        if (rc == SF_OK) rc = upload(&c->utype, ut.data(), ut.size(), "uvel_field_type");
        if (rc == SF_OK) rc = upload(&c->vtype, vt.data(), vt.size(), "vvel_field_type");
    }
    if (rc == SF_OK) {
        ProgHost Z, U, V;
        for (int m = 0; m < n && rc == SF_OK; ++m) {
            ProgHost z, u, v;
            const long s2 = (long)(d[m].L + 1) * (d[m].M + 1);
            rc = build_programs(&d[m], s2, z, u, v);
            append_program(Z, z, off2[m]);
            append_program(U, u, off2[m]);
            append_program(V, v, off2[m]);
        }
        if (rc == SF_OK) rc = upload_program(c->zbc, Z);
        if (rc == SF_OK) rc = upload_program(c->ubc, U);
        if (rc == SF_OK) rc = upload_program(c->vbc, V);
    }
    if (rc == SF_OK)
        rc = c->prec == SF_FP64 ? upload_members<double>(c, d, n, off2, off3, offN, voff)
                                : upload_members<float>(c, d, n, off2, off3, offN, voff);
    if (rc == SF_OK) {   // block maps
        std::vector<int2> pt, b128, pipe, tile[sf::kRhsTiles];
        for (int m = 0; m < n; ++m) {
            const int I = d[m].L + 1, J = d[m].M + 1;
            const long s2 = (long)I * J;
            for (long b = 0; b < (s2 + sf::kPointBlock - 1) / sf::kPointBlock; ++b) pt.push_back({m, (int)b});
            for (long b = 0; b < (s2 + 127) / 128; ++b) b128.push_back({m, (int)b});
            for (int v = 0; v < sf::kRhsTiles; ++v) {
                const int ntx = (I + sf::kRhsTileX[v] - 1) / sf::kRhsTileX[v];
                const int nty = (J + sf::kRhsTileY[v] - 1) / sf::kRhsTileY[v];
                for (int b = 0; b < ntx * nty; ++b) tile[v].push_back({m, b});
            }
            for (long b = 0; b < (s2 + sf::kPipeTile - 1) / sf::kPipeTile; ++b) pipe.push_back({m, (int)b});
        }
        c->nbm_pt = (int)pt.size();
        c->nbm_128 = (int)b128.size();
        c->nbm_pipe = (int)pipe.size();
        rc = upload(&c->bm_pt, pt.data(), pt.size(), "block map");
        if (rc == SF_OK) rc = upload(&c->bm_128, b128.data(), b128.size(), "block map");
        if (rc == SF_OK) rc = upload(&c->bm_pipe, pipe.data(), pipe.size(), "block map");
        for (int v = 0; v < sf::kRhsTiles && rc == SF_OK; ++v) {
            c->nbm_tile[v] = (int)tile[v].size();
            rc = upload(&c->bm_tile[v], tile[v].data(), tile[v].size(), "block map");
        }
    }
    if (rc != SF_OK) {
        free_ctx(c);
        return rc;
    }
    *out = c;
    return SF_OK;
}

int sf_ctx_members(const sf_ctx *c) { return c ? c->nmem : 0; }

int sf_ctx_set_tile(sf_ctx *c, int variant) {
    if (!c) return fail(SF_EINVAL, "null context");
    if (variant < 0 || variant >= sf::kRhsTiles) return fail(SF_EINVAL, "tile variant is 0, 1, 2 or 3");
    c->rhs_tile = variant;
    return SF_OK;
}

int sf_ctx_member_layout(const sf_ctx *c, long *off2, long *off3, long *offN, long *totals) {
    if (!c) return fail(SF_EINVAL, "null context");
    for (int m = 0; m < c->nmem; ++m) {
        if (off2) off2[m] = c->nmem > 1 ? c->h_off2[m] : 0;
        if (off3) off3[m] = c->nmem > 1 ? c->h_off3[m] : 0;
        if (offN) offN[m] = c->nmem > 1 ? c->h_offN[m] : 0;
    }
    if (totals) {
        totals[0] = c->nmem > 1 ? c->tot2 : c->s2;
        totals[1] = c->nmem > 1 ? c->tot3 : (long)(c->N + 1) * c->s2;
        totals[2] = c->nmem > 1 ? c->totN : (long)c->N * c->s2;
    }
    return SF_OK;
}

int sf_ctx_create(const sf_grid_desc *d, sf_ctx **out) {
    if (!d || !out) return fail(SF_EINVAL, "null argument");
    *out = nullptr;
    if (d->precision != SF_FP64 && d->precision != SF_FP32)
        return fail(SF_EDTYPE, "precision must be SF_FP64 or SF_FP32");
    if (d->L < 4 || d->M < 4) return fail(SF_EINVAL, "grid too small (need L, M >= 4)");
    if (d->N < 5 || d->N > 64)
        return fail(SF_EINVAL, "N must be in [5, 64]: the reference's verticalAdvection reads "
                               "levels up to 5 (rhs_kernels.cpp:172) and columns are held per thread");
    if (d->Vtransform != 1 && d->Vtransform != 2) return fail(SF_EINVAL, "Vtransform must be 1 or 2");
    sf_ctx *c = new (std::nothrow) sf_ctx();
    if (!c) return fail(SF_ENOMEM, "host allocation");
    c->prec = d->precision;
    // the 3D right-hand side's marching form in FP32 (basin4: 1.45 ms against 1.53 ms tiled);
    // FP64 keeps the tiled form (the marching form's FP64 registers spill)
    c->rhs_march = c->prec == SF_FP64 ? 0 : 3;
    c->L = d->L;
    c->M = d->M;
    c->N = d->N;
    c->I = d->L + 1;
    c->J = d->M + 1;
    c->s2 = (long)c->I * c->J;
    c->hc = d->hc;
    c->Vtransform = d->Vtransform;
    // horizontalAdvection is launched with (grsz*GPUMUL, bksz//GPUMUL) = 512*(s2/512 + 1)
    // threads (nonlinear/rhs.py:62, modules/mod_operators.py:40-41, utility/misc.py:10,17).
    c->ref_threads = 512L * (c->s2 / 512 + 1);
    cudaGetDevice(&c->device);
    const size_t s2 = (size_t)c->s2;
    int rc = SF_OK;
    const double *m[6] = {d->h, d->pm, d->pn, d->on_u, d->om_v, d->fomn};
    const char *mn[6] = {"h", "pm", "pn", "on_u", "om_v", "fomn"};
    for (int k = 0; k < 6 && rc == SF_OK; ++k) rc = upload_real(c, &c->metrics[k], m[k], s2, mn[k]);
    if (rc == SF_OK) rc = upload(&c->hd, d->h, s2, "h");
    if (rc == SF_OK) {
        const int N = d->N;
        if (!d->sc_r || !d->sc_w || !d->Cs_r || !d->Cs_w) rc = fail(SF_EINVAL, "missing S-coordinate tables");
        else {
            std::vector<double> v;
            v.insert(v.end(), d->sc_r, d->sc_r + N);
            v.insert(v.end(), d->sc_w, d->sc_w + N + 1);
            v.insert(v.end(), d->Cs_r, d->Cs_r + N);
            v.insert(v.end(), d->Cs_w, d->Cs_w + N + 1);
            rc = upload(&c->vert, v.data(), v.size(), "S-coordinate tables");
        }
    }
    if (rc == SF_OK) rc = upload(&c->bcfield, (const int *)d->zeta_field_idx2, s2, "zeta_field_idx2");
    if (rc == SF_OK) rc = upload(&c->utype, (const int *)d->uvel_field_type, s2, "uvel_field_type");
    if (rc == SF_OK) rc = upload(&c->vtype, (const int *)d->vvel_field_type, s2, "vvel_field_type");
    if (rc == SF_OK) {
        // setLateralUVBCs's gradient branch reads bcVIdxFieldIdx2[i + k*sz2D] for k >= 1, past
        // the end of that 2D map (step3D_uv.kernels.cpp:363); it is refused here.
        for (size_t k = 0; k < s2; ++k)
            if (d->vvel_field_type[k] > 0 && (d->vvel_field_type[k] & (1 << 4)) == 0 &&
                (d->vvel_field_type[k] & (1 << 3)) == 0 && (d->vvel_field_type[k] & (1 << 6)) != 0) {
                rc = fail(SF_EUNSUPPORTED, "gradient 3D v boundary: the reference reads past the "
                                           "boundary map (step3D_uv.kernels.cpp:363)");
                break;
            }
    }
    if (rc == SF_OK && d->n_vbar_grad > d->n_ubar_grad)
        rc = fail(SF_EUNSUPPORTED, "vbar gradient list longer than the ubar list the reference "
                                   "copies it from (barotropicVelocityBC.py:30-31)");
    ProgHost Z, U, V;
    if (rc == SF_OK) rc = build_programs(d, c->s2, Z, U, V);
    if (rc == SF_OK) rc = upload_program(c->zbc, Z);
    if (rc == SF_OK) rc = upload_program(c->ubc, U);
    if (rc == SF_OK) rc = upload_program(c->vbc, V);
    if (rc == SF_OK) rc = build_pred_maps(c, Z, U, V);
    if (rc == SF_OK) {
        if (cudaMalloc(&c->dev_err, sizeof(int)) != cudaSuccess ||
            cudaMemset(c->dev_err, 0, sizeof(int)) != cudaSuccess)
            rc = fail(SF_ENOMEM, "cudaMalloc error word");
    }
    if (rc != SF_OK) {
        free_ctx(c);
        return rc;
    }
    *out = c;
    return SF_OK;
}

int sf_ctx_destroy(sf_ctx *ctx) {
    free_ctx(ctx);
    return SF_OK;
}

// ---- 2D ---------------------------------------------------------------------------------
int sf_zeta_rhs(sf_ctx *c, const void *zeta, const void *ubar, const void *vbar, double *DU,
                double *DV, double *Zt, int is_predictor, double cff1, void *rzeta,
                sf_stream s) {
    if (!is_predictor && (!DU || !DV || !Zt)) return fail(SF_EINVAL, "accumulators required");
    return dispatch(c, "sf_zeta_rhs", [&](auto *t) {
        using R = std::remove_pointer_t<decltype(t)>;
        return sf::Ops<R>::zeta_rhs(c, (const R *)zeta, (const R *)ubar, (const R *)vbar,
                                    (R *)rzeta, is_predictor ? 0 : 1, cff1, Zt, DU, DV, nullptr,
                                    nullptr, 0.0, S(s));
    });
}

int sf_zeta_pred(sf_ctx *c, double Dt, const void *z0, void *z2, const void *rz1, sf_stream s) {
    return dispatch(c, "sf_zeta_pred", [&](auto *t) {
        using R = std::remove_pointer_t<decltype(t)>;
        return sf::Ops<R>::zeta_pred(c, Dt, (const R *)z0, (R *)z2, (const R *)rz1, S(s));
    });
}

int sf_momentum_rhs(sf_ctx *c, void *ru, void *rv, const void *za, const void *zb, double g,
                    double weight, sf_stream s) {
    return dispatch(c, "sf_momentum_rhs", [&](auto *t) {
        using R = std::remove_pointer_t<decltype(t)>;
        return sf::Ops<R>::momentum(c, (R *)ru, (R *)rv, (const R *)za, (const R *)zb, g, weight,
                                    1, 0, 0.0, nullptr, nullptr, nullptr, nullptr, nullptr,
                                    nullptr, S(s));
    });
}

int sf_momentum_pred(sf_ctx *c, double Dt, const void *u_t1, void *u_t2, const void *v_t1,
                     void *v_t2, const void *rhsu, const void *rhsv, const void *z1,
                     const void *z2, sf_stream s) {
    return dispatch(c, "sf_momentum_pred", [&](auto *t) {
        using R = std::remove_pointer_t<decltype(t)>;
        return sf::Ops<R>::momentum(c, (R *)rhsu, (R *)rhsv, nullptr, nullptr, 0.0, 0.0, 0, 1, Dt,
                                    (const R *)u_t1, (R *)u_t2, (const R *)v_t1, (R *)v_t2,
                                    (const R *)z1, (const R *)z2, S(s));
    });
}

int sf_am3(sf_ctx *c, double Dt, void *v, const void *r0, const void *r1, const void *r2,
           sf_stream s) {
    return dispatch(c, "sf_am3", [&](auto *t) {
        using R = std::remove_pointer_t<decltype(t)>;
        return sf::Ops<R>::am3(c, Dt, (R *)v, (const R *)r0, (const R *)r1, (const R *)r2, S(s));
    });
}

int sf_zetabc(sf_ctx *c, void *zeta, sf_stream s) {
    return dispatch(c, "sf_zetabc", [&](auto *t) {
        using R = std::remove_pointer_t<decltype(t)>;
        sf::BcProgram none;
        return sf::Ops<R>::bc_apply(c, c->zbc, (R *)zeta, none, nullptr, 0.0, S(s));
    });
}

int sf_barotropic_velocity_bc(sf_ctx *c, void *ubar, void *vbar, double time2D, sf_stream s) {
    const double val = .05 * std::sin(time2D * kBcOmega);
    return dispatch(c, "sf_barotropic_velocity_bc", [&](auto *t) {
        using R = std::remove_pointer_t<decltype(t)>;
        return sf::Ops<R>::bc_apply(c, c->ubc, (R *)ubar, c->vbc, (R *)vbar, val, S(s));
    });
}

int sf_step2d_predictor(sf_ctx *c, const sf_state2d *st, double dtfast, double time2D,
                        int first_step, sf_stream s) {
    if (!st) return fail(SF_EINVAL, "null state");
    const double val = .05 * std::sin(time2D * kBcOmega);
    return dispatch(c, "sf_step2d_predictor", [&](auto *t) -> cudaError_t {
        using R = std::remove_pointer_t<decltype(t)>;
        using O = sf::Ops<R>;
        R *z0 = (R *)st->zeta[0], *z1 = (R *)st->zeta[1], *z2 = (R *)st->zeta[2];
        cudaError_t e;
        if (!first_step && c->nmem == 1 && c->pred_ok && c->use_fused) {
            // the leapfrog branch as one fused launch (identical results, see substep())
            return O::pred2d(c, z0, z1, z2, (R *)st->ubar[1], (R *)st->vbar[1], (R *)st->ubar[2],
                             (R *)st->vbar[2], (R *)st->rzeta[1], (R *)st->rubar[1],
                             (R *)st->rvbar[1], dtfast, 2.0 / 5.0, val, nullptr, S(s));
        }
        if (first_step) {
            e = O::zeta_rhs(c, z1, (R *)st->ubar[1], (R *)st->vbar[1], (R *)st->rzeta[1], 0, 0.0,
                            nullptr, nullptr, nullptr, nullptr, nullptr, 0.0, S(s));
            if (e == cudaSuccess) e = O::zeta_euler(c, dtfast, z1, z2, (R *)st->rzeta[1], S(s));
        } else {
            e = O::zeta_rhs(c, z1, (R *)st->ubar[1], (R *)st->vbar[1], (R *)st->rzeta[1], 2, 0.0,
                            nullptr, nullptr, nullptr, z0, z2, dtfast, S(s));
        }
        sf::BcProgram none;
        if (e == cudaSuccess) e = O::bc_apply(c, c->zbc, z2, none, nullptr, 0.0, S(s));
        const double w = first_step ? 0.5 : 2.0 / 5.0;
        if (e == cudaSuccess)
            e = O::momentum(c, (R *)st->rubar[1], (R *)st->rvbar[1], z2, z0, 10.0, w, 1, 1, dtfast,
                            (R *)st->ubar[1], (R *)st->ubar[2], (R *)st->vbar[1], (R *)st->vbar[2],
                            z1, z2, S(s));
        if (e == cudaSuccess)
            e = O::bc_apply(c, c->ubc, (R *)st->ubar[2], c->vbc, (R *)st->vbar[2], val, S(s));
        return e;
    });
}

int sf_step2d_corrector(sf_ctx *c, const sf_state2d *st, double dtfast, double time2D,
                        double cff1, sf_stream s) {
    if (!st) return fail(SF_EINVAL, "null state");
    const double val = .05 * std::sin(time2D * kBcOmega);
    return dispatch(c, "sf_step2d_corrector", [&](auto *t) -> cudaError_t {
        using R = std::remove_pointer_t<decltype(t)>;
        using O = sf::Ops<R>;
        R *z2 = (R *)st->zeta[2];
        cudaError_t e = O::zeta_rhs(c, z2, (R *)st->ubar[2], (R *)st->vbar[2], (R *)st->rzeta[1],
                                    1, cff1, st->Zt_avg1, st->DU_avg1, st->DV_avg1, nullptr,
                                    nullptr, 0.0, S(s));
        // AdamsMoultonCorr3rd on zeta (step2d.py:109) and on ubar_t1 through the mis-bound
        // AdamsMoultonCorr3rd2 (step2d.py:120-123); independent of zetabc and of the
        // momentum RHS, so both run in one pass here.
        if (e == cudaSuccess)
            e = O::corr_point(c, dtfast, z2, (R *)st->rzeta[0], (R *)st->rzeta[1],
                              (R *)st->rzeta[2], (R *)st->ubar[1], (R *)st->vbar[1],
                              (R *)st->rubar[0], (R *)st->rubar[1], nullptr, S(s));
        sf::BcProgram none;
        if (e == cudaSuccess) e = O::bc_apply(c, c->zbc, z2, none, nullptr, 0.0, S(s));
        if (e == cudaSuccess)
            e = O::momentum(c, (R *)st->rubar[2], (R *)st->rvbar[2], z2, (R *)st->zeta[1], 10.0,
                            2.0 / 5.0, 1, 0, 0.0, nullptr, nullptr, nullptr, nullptr, nullptr,
                            nullptr, S(s));
        if (e == cudaSuccess)
            e = O::bc_apply(c, c->ubc, (R *)st->ubar[2], c->vbc, (R *)st->vbar[2], val, S(s));
        return e;
    });
}

}  // extern "C"

namespace {
template <typename R>
// vb_zero: vbar_t1 is all +0, as in every substep of a loop after its first (the previous
// substep's corrector zeroed the slot, main3d.py:189); the single-grid kernels then take the
// zeros without loading them (the same operands).
cudaError_t substep(const sf_ctx *c, const sf_state2d *st, double dtfast, double time2D,
                    double cff1, int last, cudaStream_t s, const double *dval = nullptr,
                    int vb_zero = 0) {
    using O = sf::Ops<R>;
    const bool vz = vb_zero && c->nmem == 1;
    const double val = .05 * std::sin(time2D * kBcOmega);
    R *z0 = (R *)st->zeta[0], *z1 = (R *)st->zeta[1], *z2 = (R *)st->zeta[2];
    sf::BcProgram none;
    // predictor (step2d.py:23-81): computeZetaRHS + computeZetaPred, zetabc,
    // computeMomentumRHSPred + computeMomentumPred, barotropicVelocityBC
    cudaError_t e = cudaSuccess;
    if (c->nmem == 1 && c->pred_ok && c->use_fused) {
        e = O::pred2d(c, z0, z1, z2, (R *)st->ubar[1], (R *)st->vbar[1], (R *)st->ubar[2],
                      (R *)st->vbar[2], (R *)st->rzeta[1], (R *)st->rubar[1], (R *)st->rvbar[1],
                      dtfast, 2.0 / 5.0, val, dval, s, vz ? 1 : 0);
    } else {
        e = O::zeta_rhs(c, z1, (R *)st->ubar[1], (R *)st->vbar[1], (R *)st->rzeta[1], 2, 0.0,
                        nullptr, nullptr, nullptr, z0, z2, dtfast, s);
        if (e == cudaSuccess) e = O::bc_apply(c, c->zbc, z2, none, nullptr, 0.0, s);
        if (e == cudaSuccess)
            e = O::momentum(c, (R *)st->rubar[1], (R *)st->rvbar[1], z2, z0, 10.0, 2.0 / 5.0, 1,
                            1, dtfast, (R *)st->ubar[1], (R *)st->ubar[2], (R *)st->vbar[1],
                            (R *)st->vbar[2], z1, z2, s);
        if (e == cudaSuccess)
            e = O::bc_apply(c, c->ubc, (R *)st->ubar[2], c->vbc, (R *)st->vbar[2], val, s, dval);
    }
    // corrector (step2d.py:84-128) and vbar_t2[:] = 0 (main3d.py:189)
    if (e == cudaSuccess)
        e = O::zeta_rhs(c, z2, (R *)st->ubar[2], (R *)st->vbar[2], (R *)st->rzeta[1], 1, cff1,
                        st->Zt_avg1, st->DU_avg1, st->DV_avg1, nullptr, nullptr, 0.0, s);
    const R *vb1 = vz ? nullptr : (const R *)st->vbar[1];
    if (e == cudaSuccess && last)   // barotropicVelocityBC of the corrector is idempotent
        e = O::corr_point(c, dtfast, z2, (R *)st->rzeta[0], (R *)st->rzeta[1], (R *)st->rzeta[2],
                          (R *)st->ubar[1], vb1, (R *)st->rubar[0], (R *)st->rubar[1],
                          nullptr, s);
    else if (e == cudaSuccess)
        e = O::corr_point(c, dtfast, z2, (R *)st->rzeta[0], (R *)st->rzeta[1], (R *)st->rzeta[2],
                          (R *)st->ubar[1], vb1, (R *)st->rubar[0], (R *)st->rubar[1],
                          (R *)st->vbar[2], s);
    if (e == cudaSuccess) e = O::bc_apply(c, c->zbc, z2, none, nullptr, 0.0, s);
    if (e == cudaSuccess && last) {
        e = O::momentum(c, (R *)st->rubar[2], (R *)st->rvbar[2], z2, z1, 10.0, 2.0 / 5.0, 1, 0, 0.0,
                        nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, s);
        if (e == cudaSuccess)
            e = cudaMemsetAsync(st->vbar[2], 0, (size_t)c->s2 * sizeof(R), s);
    }
    return e;
}
}  // namespace

extern "C" {

int sf_barotropic_substep(sf_ctx *c, const sf_state2d *st, double dtfast, double time2D,
                          double cff1, int last, sf_stream s) {
    if (!st) return fail(SF_EINVAL, "null state");
    return dispatch(c, "sf_barotropic_substep", [&](auto *t) {
        using R = std::remove_pointer_t<decltype(t)>;
        return substep<R>(c, st, dtfast, time2D, cff1, last, S(s));
    });
}

}  // extern "C"

namespace {
// The clamped boundary values of the substeps of one loop, passed by value to a one-block
// kernel that writes them to the context's device array before the captured loop replays.
struct BcVals {
    double v[256];
};
__global__ void k_set_bcvals(BcVals vals, int n, double *dst) {
    for (int k = threadIdx.x; k < n; k += blockDim.x) dst[k] = vals.v[k];
}

void rotate(sf_state2d *st) {   // T_OCEAN.cycleTimes2D
    void **arrs[6] = {st->zeta, st->ubar, st->vbar, st->rzeta, st->rubar, st->rvbar};
    for (void **a : arrs) {
        void *t0 = a[0];
        a[0] = a[1];
        a[1] = a[2];
        a[2] = t0;
    }
}

bool graph_matches(const sf_loop_graph &g, const sf_state2d *st, int nsub, const double *w,
                   double dtfast) {
    if (!g.exec || g.nsub != nsub || g.dtfast != dtfast) return false;
    void *const *arrs[6] = {st->zeta, st->ubar, st->vbar, st->rzeta, st->rubar, st->rvbar};
    for (int a = 0; a < 6; ++a)
        for (int k = 0; k < 3; ++k)
            if (g.slots[3 * a + k] != arrs[a][k]) return false;
    if (g.acc[0] != st->Zt_avg1 || g.acc[1] != st->DU_avg1 || g.acc[2] != st->DV_avg1) return false;
    for (int k = 0; k < nsub; ++k)
        if (g.w[k] != w[k]) return false;
    return true;
}

// The loop's launches in order on stream s; with `dval` the clamped boundary values are read
// from dval[iif-1] on the device instead of being passed by value.
int loop_body(sf_ctx *c, sf_state2d *st, int nsub, const double *weight1, double dtfast,
              double t2, cudaStream_t s, const double *dval) {
    const size_t n2 = (size_t)c->s2 * sizeof(double);
    cudaError_t e = cudaMemsetAsync(st->Zt_avg1, 0, n2, s);
    if (e == cudaSuccess) e = cudaMemsetAsync(st->DU_avg1, 0, n2, s);
    if (e == cudaSuccess) e = cudaMemsetAsync(st->DV_avg1, 0, n2, s);
    if (e != cudaSuccess) return cuda_fail(e, "sf_barotropic_loop");
    for (int iif = 1; iif <= nsub; ++iif) {
        t2 += dtfast;
        rotate(st);
        const double *dv = dval ? dval + (iif - 1) : nullptr;
        e = c->prec == SF_FP64
                ? substep<double>(c, st, dtfast, t2, weight1[iif - 1], iif == nsub, s, dv, iif > 1)
                : substep<float>(c, st, dtfast, t2, weight1[iif - 1], iif == nsub, s, dv, iif > 1);
        if (e != cudaSuccess) return cuda_fail(e, "sf_barotropic_loop");
    }
    return SF_OK;
}
}  // namespace

extern "C" {

int sf_ctx_set_graphs(sf_ctx *c, int enable) {
    if (!c) return fail(SF_EINVAL, "null context");
    c->use_graphs = enable ? 1 : 0;
    return SF_OK;
}

int sf_ctx_set_fused(sf_ctx *c, int enable) {
    if (!c) return fail(SF_EINVAL, "null context");
    if (c->use_fused != (enable ? 1 : 0)) {
        for (auto &g : c->graphs) {   // captured loops hold the other form
            if (g.exec) cudaGraphExecDestroy(g.exec);
            g.exec = nullptr;
        }
    }
    c->use_fused = enable ? 1 : 0;
    return SF_OK;
}

int sf_ctx_set_bulk(sf_ctx *c, int enable) {
    if (!c) return fail(SF_EINVAL, "null context");
    c->use_bulk = enable ? 1 : 0;
    return SF_OK;
}

int sf_ctx_tune(sf_ctx *c, int knob, int value) {
    if (!c) return fail(SF_EINVAL, "null context");
    switch (knob) {
    case SF_TUNE_MO_CHUNK:
        if (value != 0 && value != 4 && value != 5 && value != 8)
            return fail(SF_EINVAL, "chunk is 0, 4, 5 or 8");
        c->mo_chunk = value;
        return SF_OK;
    case SF_TUNE_PRED_PAIR:
        if (value < 0 || value > 2) return fail(SF_EINVAL, "pair is 0, 1 or 2");
        if (c->pred_pair != value)
            for (auto &g : c->graphs) {   // captured loops hold the other kernel
                if (g.exec) cudaGraphExecDestroy(g.exec);
                g.exec = nullptr;
            }
        c->pred_pair = value;
        return SF_OK;
    case SF_TUNE_S3_VEC:
        if (value != 0 && value != 1) return fail(SF_EINVAL, "vec is 0 or 1");
        c->s3_vec = value;
        return SF_OK;
    case SF_TUNE_RHS_MARCH:
        if (value < 0 || value > 3) return fail(SF_EINVAL, "march is 0, 1, 2 or 3");
        c->rhs_march = value;
        return SF_OK;
    case SF_TUNE_RHS_CHUNKS:
        if (value != 0 && value != 1) return fail(SF_EINVAL, "chunks is 0 or 1");
        c->rhs_chunks = value;
        return SF_OK;
    default:
        return fail(SF_EINVAL, "unknown tuning knob");
    }
}

int sf_ctx_fused_available(const sf_ctx *c) { return c && c->nmem == 1 && c->pred_ok ? 1 : 0; }

int sf_ctx_set_pdl(sf_ctx *c, int enable) {
    if (!c) return fail(SF_EINVAL, "null context");
    if (c->use_pdl != (enable ? 1 : 0)) {
        for (auto &g : c->graphs) {   // captured loops hold the old launch attribute
            if (g.exec) cudaGraphExecDestroy(g.exec);
            g.exec = nullptr;
        }
    }
    c->use_pdl = enable ? 1 : 0;
    return SF_OK;
}

int sf_barotropic_loop(sf_ctx *c, sf_state2d *st, int nsub, const double *weight1, double dtfast,
                       double *time2D, sf_stream s) {
    if (!st || !weight1 || !time2D || nsub < 1) return fail(SF_EINVAL, "bad argument");
    if (!c) return fail(SF_EINVAL, "null context");
    if (c->use_graphs && nsub <= 256) {
        // Replay a captured loop: the same launches with the same arguments; only the clamped
        // boundary values (a function of time2D) change, and they are read on the device.
        sf_loop_graph *g = nullptr;
        for (auto &cand : c->graphs)
            if (graph_matches(cand, st, nsub, weight1, dtfast)) g = &cand;
        cudaError_t e = cudaSuccess;
        if (!g) {
            if (!c->cap) {
                e = cudaStreamCreateWithFlags(&c->cap, cudaStreamNonBlocking);
                if (e != cudaSuccess) return cuda_fail(e, "cudaStreamCreate");
            }
            if (!c->d_bcval) {
                e = cudaMalloc(&c->d_bcval, 256 * sizeof(double));
                if (e != cudaSuccess) return fail(SF_ENOMEM, "cudaMalloc bcval");
            }
            g = &c->graphs[c->graph_next];
            c->graph_next = (c->graph_next + 1) % 3;
            if (g->exec) {
                cudaGraphExecDestroy(g->exec);
                g->exec = nullptr;
            }
            sf_state2d tmp = *st;
            e = cudaStreamBeginCapture(c->cap, cudaStreamCaptureModeThreadLocal);
            if (e != cudaSuccess) return cuda_fail(e, "cudaStreamBeginCapture");
            const int rc = loop_body(c, &tmp, nsub, weight1, dtfast, 0.0, c->cap, c->d_bcval);
            cudaGraph_t graph = nullptr;
            e = cudaStreamEndCapture(c->cap, &graph);
            if (rc != SF_OK) {
                if (graph) cudaGraphDestroy(graph);
                return rc;
            }
            if (e != cudaSuccess) return cuda_fail(e, "cudaStreamEndCapture");
            e = cudaGraphInstantiate(&g->exec, graph, 0);
            cudaGraphDestroy(graph);
            if (e != cudaSuccess) {
                g->exec = nullptr;
                return cuda_fail(e, "cudaGraphInstantiate");
            }
            g->nsub = nsub;
            g->dtfast = dtfast;
            void *const *arrs[6] = {st->zeta, st->ubar, st->vbar, st->rzeta, st->rubar, st->rvbar};
            for (int a = 0; a < 6; ++a)
                for (int k = 0; k < 3; ++k) g->slots[3 * a + k] = arrs[a][k];
            g->acc[0] = st->Zt_avg1;
            g->acc[1] = st->DU_avg1;
            g->acc[2] = st->DV_avg1;
            for (int k = 0; k < nsub; ++k) g->w[k] = weight1[k];
        }
        BcVals vals;
        double t2 = *time2D;
        for (int iif = 1; iif <= nsub; ++iif) {
            t2 += dtfast;                              // CompTimes.next2DTimeStep
            vals.v[iif - 1] = .05 * std::sin(t2 * kBcOmega);
            rotate(st);
        }
        k_set_bcvals<<<1, 256, 0, S(s)>>>(vals, nsub, c->d_bcval);
        e = cudaGetLastError();
        if (e == cudaSuccess) e = cudaGraphLaunch(g->exec, S(s));
        if (e != cudaSuccess) return cuda_fail(e, "sf_barotropic_loop (graph)");
        *time2D = t2;
        return SF_OK;
    }
    const size_t n2 = (size_t)c->s2 * sizeof(double);
    cudaError_t e = cudaMemsetAsync(st->Zt_avg1, 0, n2, S(s));
    if (e == cudaSuccess) e = cudaMemsetAsync(st->DU_avg1, 0, n2, S(s));
    if (e == cudaSuccess) e = cudaMemsetAsync(st->DV_avg1, 0, n2, S(s));
    if (e != cudaSuccess) return cuda_fail(e, "sf_barotropic_loop");
    double t2 = *time2D;
    for (int iif = 1; iif <= nsub; ++iif) {
        t2 += dtfast;                                  // CompTimes.next2DTimeStep
        void **arrs[6] = {st->zeta, st->ubar, st->vbar, st->rzeta, st->rubar, st->rvbar};
        for (void **a : arrs) {                        // T_OCEAN.cycleTimes2D
            void *t0 = a[0];
            a[0] = a[1];
            a[1] = a[2];
            a[2] = t0;
        }
        const int rc = sf_barotropic_substep(c, st, dtfast, t2, weight1[iif - 1], iif == nsub, s);
        if (rc != SF_OK) return rc;
    }
    *time2D = t2;
    return SF_OK;
}

// ---- ROMS-form barotropic step (sf_roms.cuh) ----------------------------------------------
}  // extern "C"

namespace {
// One phase (0 predictor, 1 corrector) of the ROMS-form substep on the slots of st:
// [0] = n-1, [1] = n, [2] = the predicted n+1*.
template <typename R>
cudaError_t roms_phase(const sf_ctx *c, const sf_state2d *st, double *DU2, double *DV2,
                       const void *sustr, const void *svstr, double rdrag2, double dtfast,
                       int phase, int first, int acc, double c1, double c2, int step,
                       cudaStream_t s) {
    sf::RomsArgs<R> a;
    a.zb = (const R *)st->zeta[0];
    a.zn = (const R *)st->zeta[1];
    a.zp = (const R *)st->zeta[2];
    a.ub = (const R *)st->ubar[0];
    a.un = (const R *)st->ubar[1];
    a.up = (const R *)st->ubar[2];
    a.vb = (const R *)st->vbar[0];
    a.vn = (const R *)st->vbar[1];
    a.vp = (const R *)st->vbar[2];
    const int out = phase == 0 ? 2 : 0;
    a.zout = (R *)st->zeta[out];
    a.uout = (R *)st->ubar[out];
    a.vout = (R *)st->vbar[out];
    const int kstp = phase == 0 ? (first ? 1 : 0) : 1;
    a.zkstp = (const R *)st->zeta[kstp];
    a.ukstp = (const R *)st->ubar[kstp];
    a.vkstp = (const R *)st->vbar[kstp];
    const int krhs = phase == 0 ? 1 : 2;
    a.zrhs = (const R *)st->zeta[krhs];
    a.urhs = (const R *)st->ubar[krhs];
    a.vrhs = (const R *)st->vbar[krhs];
    a.rz_n = (R *)st->rzeta[1];
    a.ru_n = (R *)st->rubar[1];
    a.rv_n = (R *)st->rvbar[1];
    a.rz_b = (const R *)st->rzeta[0];
    a.ru_b = (const R *)st->rubar[0];
    a.rv_b = (const R *)st->rvbar[0];
    a.sustr = (const R *)sustr;
    a.svstr = (const R *)svstr;
    a.Zt = st->Zt_avg1;
    a.DU1 = st->DU_avg1;
    a.DV1 = st->DV_avg1;
    a.DU2 = DU2;
    a.DV2 = DV2;
    a.rdrag2 = rdrag2;
    a.dtfast = dtfast;
    a.c1 = c1;
    a.c2 = c2;
    a.phase = phase;
    a.first = first;
    a.acc = acc;
    a.step = step;
    return sf::Ops<R>::roms_phase(c, a, s);
}

void roms_swap(sf_state2d *st) {   // n+1 (written over n-1) becomes n, n becomes n-1
    void **arrs[6] = {st->zeta, st->ubar, st->vbar, st->rzeta, st->rubar, st->rvbar};
    for (void **a : arrs) {
        void *t = a[0];
        a[0] = a[1];
        a[1] = t;
    }
}

int roms_check(const sf_ctx *c, const sf_state2d *st, const void *sustr, const void *svstr) {
    if (!c) return fail(SF_EINVAL, "null context");
    if (!st || !sustr || !svstr) return fail(SF_EINVAL, "null state or stress");
    for (void *const *a : {st->zeta, st->ubar, st->vbar})
        for (int k = 0; k < 3; ++k)
            if (!a[k]) return fail(SF_EINVAL, "null 2D slot");
    for (void *const *a : {st->rzeta, st->rubar, st->rvbar})
        for (int k = 0; k < 2; ++k)
            if (!a[k]) return fail(SF_EINVAL, "null tendency slot");
    return SF_OK;
}
}  // namespace

extern "C" {

int sf_roms_barotropic_loop(sf_ctx *c, sf_state2d *st, double *DU_avg2, double *DV_avg2,
                            const void *sustr, const void *svstr, double rdrag2, int nfast,
                            const double *W1, const double *W2, double dtfast, sf_stream s) {
    int rc = roms_check(c, st, sustr, svstr);
    if (rc) return rc;
    if (!DU_avg2 || !DV_avg2 || !st->Zt_avg1 || !st->DU_avg1 || !st->DV_avg1 || !W1 || !W2)
        return fail(SF_EINVAL, "null accumulator or weights");
    if (nfast < 1 || nfast > 254) return fail(SF_EINVAL, "nfast must be in [1, 254]");
    for (int iif = 1; iif <= nfast + 1; ++iif) {
        // fast-time averages (step2d_LF_AM3.h.py:778-846), ROMS-indexed weights
        const int acc = iif == 1 ? 2 : 1;
        const double pc1 = iif == 1 ? 0.0 : W1[iif - 1];
        const double pc2 = iif == 1 ? (-1.0 / 12.0) * W2[2]
                                    : (8.0 / 12.0) * W2[iif] - (1.0 / 12.0) * W2[iif + 1];
        const double cc2 = iif == 1 ? W2[1] : (5.0 / 12.0) * W2[iif];
        const int step = iif <= nfast, first = iif == 1;
        cudaError_t e = c->prec == SF_FP64
            ? roms_phase<double>(c, st, DU_avg2, DV_avg2, sustr, svstr, rdrag2, dtfast, 0, first,
                                 acc, pc1, pc2, step, S(s))
            : roms_phase<float>(c, st, DU_avg2, DV_avg2, sustr, svstr, rdrag2, dtfast, 0, first,
                                acc, pc1, pc2, step, S(s));
        if (e == cudaSuccess && step)
            e = c->prec == SF_FP64
                ? roms_phase<double>(c, st, DU_avg2, DV_avg2, sustr, svstr, rdrag2, dtfast, 1,
                                     first, 1, 0.0, cc2, 1, S(s))
                : roms_phase<float>(c, st, DU_avg2, DV_avg2, sustr, svstr, rdrag2, dtfast, 1,
                                    first, 1, 0.0, cc2, 1, S(s));
        if (e != cudaSuccess) return cuda_fail(e, "sf_roms_barotropic_loop");
        if (step) roms_swap(st);
    }
    return SF_OK;
}

int sf_roms_step2d(sf_ctx *c, sf_state2d *st, const void *sustr, const void *svstr,
                   double rdrag2, double dtfast, int first, sf_stream s) {
    int rc = roms_check(c, st, sustr, svstr);
    if (rc) return rc;
    cudaError_t e = cudaSuccess;
    for (int phase = 0; phase < 2 && e == cudaSuccess; ++phase)
        e = c->prec == SF_FP64
            ? roms_phase<double>(c, st, nullptr, nullptr, sustr, svstr, rdrag2, dtfast, phase,
                                 first ? 1 : 0, 0, 0.0, 0.0, 1, S(s))
            : roms_phase<float>(c, st, nullptr, nullptr, sustr, svstr, rdrag2, dtfast, phase,
                                first ? 1 : 0, 0, 0.0, 0.0, 1, S(s));
    if (e != cudaSuccess) return cuda_fail(e, "sf_roms_step2d");
    roms_swap(st);
    return SF_OK;
}

static double ab3_cff(int iic, int ntfirst) {   // step3D_uv.kernels.cpp:663-666
    if (iic == ntfirst) return 1.0;
    if (iic == ntfirst + 1) return 3.0 / 2.0;
    return 23.0 / 12.0;
}

int sf_roms_stress3d(sf_ctx *c, const void *u, const void *v, void *ru, void *rv,
                     const void *sustr, const void *svstr, double rdrag2, sf_stream s) {
    if (!u || !v || !ru || !rv || !sustr || !svstr) return fail(SF_EINVAL, "null argument");
    return dispatch(c, "sf_roms_stress3d", [&](auto *t) {
        using R = std::remove_pointer_t<decltype(t)>;
        return sf::Ops<R>::roms_stress3d(c, (const R *)u, (const R *)v, (R *)ru, (R *)rv,
                                         (const R *)sustr, (const R *)svstr, rdrag2, S(s));
    });
}

int sf_roms_rhs3d(sf_ctx *c, const void *u, const void *v, const void *Huon, const void *Hvom,
                  const void *Hz, void *ru, void *rv, sf_stream s) {
    if (!u || !v || !Huon || !Hvom || !Hz || !ru || !rv) return fail(SF_EINVAL, "null argument");
    return dispatch(c, "sf_roms_rhs3d", [&](auto *t) {
        using R = std::remove_pointer_t<decltype(t)>;
        return sf::Ops<R>::roms_rhs3d(c, (const R *)u, (const R *)v, (const R *)Huon,
                                      (const R *)Hvom, (const R *)Hz, (R *)ru, (R *)rv, S(s));
    });
}

int sf_roms_step3d_uv(sf_ctx *c, void *u, void *v, const void *ru0, const void *ru1,
                      const void *ru2, const void *rv0, const void *rv1, const void *rv2,
                      void *ubar_n, void *vbar_n, void *ubar_s, void *vbar_s, const void *Hz,
                      const void *Akv, const void *z_r, const void *W, const double *DU,
                      const double *DV, int iic, int ntfirst, double lambda, double Dt,
                      sf_stream s) {
    if (!u || !v || !ru0 || !ru1 || !ru2 || !rv0 || !rv1 || !rv2 || !ubar_n || !vbar_n ||
        !ubar_s || !vbar_s || !Hz || !Akv || !z_r || !W || !DU || !DV)
        return fail(SF_EINVAL, "null argument");
    if (iic < ntfirst) return fail(SF_EINVAL, "sf_roms_step3d_uv: iic < ntfirst");
    if (c && (c->nmem > 1 ? c->maxN : c->N) > sf::kRomsMaxN)
        return fail(SF_EINVAL, "sf_roms_step3d_uv: N > 64");
    // Adams-Bashforth weights of ru(n), ru(n-1), ru(n-2): forward Euler, AB2, then AB3
    static const double kAB[3][3] = {{1.0, 0.0, 0.0}, {1.5, -0.5, 0.0},
                                     {23.0 / 12.0, -16.0 / 12.0, 5.0 / 12.0}};
    const double *coef = kAB[iic - ntfirst < 2 ? iic - ntfirst : 2];
    return dispatch(c, "sf_roms_step3d_uv", [&](auto *t) {
        using R = std::remove_pointer_t<decltype(t)>;
        const R *ru[3] = {(const R *)ru0, (const R *)ru1, (const R *)ru2};
        const R *rv[3] = {(const R *)rv0, (const R *)rv1, (const R *)rv2};
        return sf::Ops<R>::roms_step3d(c, (R *)u, (R *)v, ru, rv, coef, (R *)ubar_n, (R *)vbar_n,
                                       (R *)ubar_s, (R *)vbar_s, (const R *)Hz, (const R *)Akv,
                                       (const R *)z_r, (const R *)W, DU, DV, Dt, lambda * Dt,
                                       S(s));
    });
}

int sf_roms_closed_walls(sf_ctx *c, void *u, void *v, sf_stream s) {
    if (!u || !v) return fail(SF_EINVAL, "null argument");
    return dispatch(c, "sf_roms_closed_walls", [&](auto *t) {
        using R = std::remove_pointer_t<decltype(t)>;
        return sf::Ops<R>::roms_walls3d(c, (R *)u, (R *)v, S(s));
    });
}

// ---- 3D ---------------------------------------------------------------------------------
int sf_rhs3d(sf_ctx *c, const void *u, const void *v, const void *Huon, const void *Hvom,
             const void *W, const void *Hz, void *ru, void *rv, sf_stream s) {
    return dispatch(c, "sf_rhs3d", [&](auto *t) {
        using R = std::remove_pointer_t<decltype(t)>;
        return sf::Ops<R>::rhs3d(c, (const R *)u, (const R *)v, (const R *)Huon, (const R *)Hvom,
                                 (const R *)W, (const R *)Hz, (R *)ru, (R *)rv, S(s));
    });
}

int sf_set_maxflux(sf_ctx *c, const void *u, const void *v, void *Huon, void *Hvom, const void *Hz,
                   sf_stream s) {
    return dispatch(c, "sf_set_maxflux", [&](auto *t) {
        using R = std::remove_pointer_t<decltype(t)>;
        return sf::Ops<R>::maxflux_omega(c, (const R *)u, (const R *)v, (R *)Huon, (R *)Hvom,
                                         (const R *)Hz, nullptr, nullptr, 1, 0, nullptr, nullptr,
                                         nullptr, S(s));
    });
}

int sf_omega(sf_ctx *c, void *W, const void *Huon, const void *Hvom, const void *z_w,
             sf_stream s) {
    return dispatch(c, "sf_omega", [&](auto *t) {
        using R = std::remove_pointer_t<decltype(t)>;
        return sf::Ops<R>::maxflux_omega(c, nullptr, nullptr, (R *)Huon, (R *)Hvom, nullptr,
                                         (R *)W, (const R *)z_w, 0, 1, nullptr, nullptr, nullptr,
                                         S(s));
    });
}

int sf_maxflux_omega(sf_ctx *c, const void *u, const void *v, void *Huon, void *Hvom,
                     const void *Hz, void *W, const void *z_w, void *zeta_t1, void *zeta_t2,
                     const double *Zt, sf_stream s) {
    if ((zeta_t1 || zeta_t2 || Zt) && !(zeta_t1 && zeta_t2 && Zt))
        return fail(SF_EINVAL, "set_zeta needs zeta_t1, zeta_t2 and Zt_avg1");
    return dispatch(c, "sf_maxflux_omega", [&](auto *t) {
        using R = std::remove_pointer_t<decltype(t)>;
        return sf::Ops<R>::maxflux_omega(c, (const R *)u, (const R *)v, (R *)Huon, (R *)Hvom,
                                         (const R *)Hz, (R *)W, (const R *)z_w, 1, 1,
                                         (R *)zeta_t1, (R *)zeta_t2, Zt, S(s));
    });
}

int sf_set_zeta(sf_ctx *c, void *z1, void *z2, const double *Zt, sf_stream s) {
    return dispatch(c, "sf_set_zeta", [&](auto *t) {
        using R = std::remove_pointer_t<decltype(t)>;
        return sf::Ops<R>::set_zeta(c, (R *)z1, (R *)z2, Zt, S(s));
    });
}

int sf_set_depth(sf_ctx *c, const double *Zt, void *z_w, void *z_r, void *Hz, sf_stream s) {
    return dispatch(c, "sf_set_depth", [&](auto *t) {
        using R = std::remove_pointer_t<decltype(t)>;
        return sf::Ops<R>::set_depth(c, Zt, (R *)z_w, (R *)z_r, (R *)Hz, S(s));
    });
}

}  // extern "C"

// ---- state check (non-finite / blow-up detection) --------------------------------------------
namespace {
constexpr int kCheckBlocks = 4 * 148;
constexpr int kCheckFields = 5;   // zeta, ubar, vbar, u, v
const char *const kCheckNames[kCheckFields] = {"zeta", "ubar", "vbar", "u", "v"};

struct CheckArgs {
    const void *f[kCheckFields];
    long n[kCheckFields];
    double bound[kCheckFields];   // |value| above the bound counts as a blow-up
};

// One grid-stride pass over each field; a value that is NaN, infinite or above its bound
// records key = field << 56 | flat index with atomicMin, so the smallest field and index win.
template <typename R>
__global__ void __launch_bounds__(256) k_check_state(CheckArgs a, unsigned long long *key) {
    const long stride = (long)gridDim.x * blockDim.x;
    for (int f = 0; f < kCheckFields; ++f) {
        const R *x = static_cast<const R *>(a.f[f]);
        if (!x) continue;
        const R bound = (R)a.bound[f];
        unsigned long long best = ~0ULL;
        for (long p = (long)blockIdx.x * blockDim.x + threadIdx.x; p < a.n[f]; p += stride) {
            const R v = __ldg(x + p);
            if (!(fabs(v) <= bound)) {   // NaN compares false
                best = ((unsigned long long)f << 56) | (unsigned long long)p;
                break;
            }
        }
        if (best != ~0ULL) atomicMin(key, best);
    }
}
}  // namespace

extern "C" {

int sf_check_state(sf_ctx *c, const void *zeta, const void *ubar, const void *vbar,
                   const void *u, const void *v, double surface_bound, double velocity_bound,
                   sf_stream s) {
    if (!c) return fail(SF_EINVAL, "null context");
    if (c->nmem != 1) return fail(SF_EUNSUPPORTED, "sf_check_state: single-grid contexts only");
    if (!(surface_bound > 0.0) || !(velocity_bound > 0.0))
        return fail(SF_EINVAL, "sf_check_state: bounds must be positive");
    cudaError_t e;
    if (!c->check_dev) {
        e = cudaMalloc(&c->check_dev, sizeof(unsigned long long));
        if (e != cudaSuccess) return fail(SF_ENOMEM, "sf_check_state: device flag");
        e = cudaMallocHost(&c->check_host, sizeof(unsigned long long));
        if (e != cudaSuccess) return fail(SF_ENOMEM, "sf_check_state: host flag");
    }
    const long n3 = (long)(c->N + 1) * c->s2;
    CheckArgs a{{zeta, ubar, vbar, u, v}, {c->s2, c->s2, c->s2, n3, n3},
                {surface_bound, velocity_bound, velocity_bound, velocity_bound, velocity_bound}};
    SF_TRY_CUDA(cudaMemsetAsync(c->check_dev, 0xFF, sizeof(unsigned long long), S(s)),
                "sf_check_state");
    if (c->prec == SF_FP64)
        k_check_state<double><<<kCheckBlocks, 256, 0, S(s)>>>(a, c->check_dev);
    else
        k_check_state<float><<<kCheckBlocks, 256, 0, S(s)>>>(a, c->check_dev);
    SF_TRY_CUDA(cudaGetLastError(), "sf_check_state");
    SF_TRY_CUDA(cudaMemcpyAsync(c->check_host, c->check_dev, sizeof(unsigned long long),
                                cudaMemcpyDeviceToHost, S(s)), "sf_check_state");
    SF_TRY_CUDA(cudaStreamSynchronize(S(s)), "sf_check_state");
    if (c->dev_err) {
        int werr = 0;
        SF_TRY_CUDA(cudaMemcpy(&werr, c->dev_err, sizeof(int), cudaMemcpyDeviceToHost),
                    "sf_check_state");
        if (werr) {
            SF_TRY_CUDA(cudaMemset(c->dev_err, 0, sizeof(int)), "sf_check_state");
            return fail(SF_ETIMEOUT, "a kernel's bounded wait for its staged data gave up "
                                     "(the results of the step are not valid)");
        }
    }
    const unsigned long long key = *c->check_host;
    if (key == ~0ULL) return SF_OK;
    const int f = (int)(key >> 56);
    const long p = (long)(key & ((1ULL << 56) - 1));
    const long lev = f >= 3 ? p / c->s2 : 0, q = p % c->s2;
    char msg[200];
    std::snprintf(msg, sizeof msg,
                  "non-finite or out-of-bound %s at flat index %ld (level %ld, j %ld, i %ld)",
                  kCheckNames[f < kCheckFields ? f : 0], p, lev, q / c->I, q % c->I);
    return fail(SF_ENONFINITE, msg);
}

int sf_step3d_uv(sf_ctx *c, void *u, void *v, const void *ru, const void *rv, void *ubar_t1,
                 void *vbar_t1, void *ubar_t2, void *vbar_t2, const void *Hz, const void *Akv,
                 const void *z_r, const double *DU, const double *DV, const void *tmpU,
                 const void *tmpV, int iic, int ntfirst, double lambda, double Dt, sf_stream s) {
    const double cff = ab3_cff(iic, ntfirst);
    return dispatch(c, "sf_step3d_uv", [&](auto *t) {
        using R = std::remove_pointer_t<decltype(t)>;
        return sf::Ops<R>::step3d_uv(c, (R *)u, (R *)v, (const R *)ru, (const R *)rv, (R *)ubar_t1,
                                     (R *)vbar_t1, (R *)ubar_t2, (R *)vbar_t2, (const R *)Hz,
                                     (const R *)Akv, (const R *)z_r, DU, DV, (const R *)tmpU,
                                     (const R *)tmpV, cff, lambda, Dt, 0, 0.0, S(s));
    });
}

int sf_step3d_uv_bc(sf_ctx *c, void *u, void *v, const void *ru, const void *rv, void *ubar_t1,
                    void *vbar_t1, void *ubar_t2, void *vbar_t2, const void *Hz, const void *Akv,
                    const void *z_r, const double *DU, const double *DV, int iic, int ntfirst,
                    double lambda, double Dt, double time, sf_stream s) {
    const double cff = ab3_cff(iic, ntfirst);
    const double val = 0.05 * std::sin(time * kBcOmega);
    return dispatch(c, "sf_step3d_uv_bc", [&](auto *t) {
        using R = std::remove_pointer_t<decltype(t)>;
        return sf::Ops<R>::step3d_uv(c, (R *)u, (R *)v, (const R *)ru, (const R *)rv, (R *)ubar_t1,
                                     (R *)vbar_t1, (R *)ubar_t2, (R *)vbar_t2, (const R *)Hz,
                                     (const R *)Akv, (const R *)z_r, DU, DV, nullptr, nullptr,
                                     cff, lambda, Dt, 1, val, S(s));
    });
}

int sf_lateral_uv_bc(sf_ctx *c, double time, void *u, void *v, sf_stream s) {
    const double val = 0.05 * std::sin(time * kBcOmega);
    return dispatch(c, "sf_lateral_uv_bc", [&](auto *t) {
        using R = std::remove_pointer_t<decltype(t)>;
        return sf::Ops<R>::lateral_uv_bc(c, (R *)u, (R *)v, val, S(s));
    });
}

int sf_gls_corrector(sf_ctx *c, const sf_gls_params *P, double dt, const void *u, const void *v,
                     const void *z_r, const void *Hz, const void *bvf, const void *sustr,
                     const void *svstr, void *tke, void *gls, void *Akv, void *Akt, void *Akk,
                     void *Akp, void *Lscale, sf_stream s) {
    return sf_gls_corrector_cols(c, P, dt, u, v, z_r, Hz, bvf, sustr, svstr, tke, gls, Akv, Akt,
                                 Akk, Akp, Lscale, nullptr, s);
}

namespace {
int gls_checks(const sf_gls_params *P) {
    if (!P) return fail(SF_EINVAL, "null GLS parameters");
    if (P->n == 0.0) return fail(SF_EINVAL, "GLS exponent n must be non-zero");
    if (P->p == 0.0 && P->m == 1.0 && P->n == 1.0)
        return fail(SF_EUNSUPPORTED, "Mellor-Yamada 2.5 (p=0, m=1, n=1) needs the wall function, "
                                     "which is not built");
    return SF_OK;
}
}  // namespace

int sf_gls_corrector_list(sf_ctx *c, const sf_gls_params *P, double dt, const void *u,
                          const void *v, const void *z_r, const void *Hz, const void *bvf,
                          const void *sustr, const void *svstr, void *tke, void *gls, void *Akv,
                          void *Akt, void *Akk, void *Akp, void *Lscale, const int *list,
                          const int *count, sf_stream s) {
    if (!list || !count) return fail(SF_EINVAL, "null column list");
    if (const int rc = gls_checks(P)) return rc;
    return dispatch(c, "sf_gls_corrector_list", [&](auto *t) {
        using R = std::remove_pointer_t<decltype(t)>;
        return sf::Ops<R>::gls_corrector(c, *P, dt, (const R *)u, (const R *)v, (const R *)z_r,
                                         (const R *)Hz, (const R *)bvf, (const R *)sustr,
                                         (const R *)svstr, (R *)tke, (R *)gls, (R *)Akv, (R *)Akt,
                                         (R *)Akk, (R *)Akp, (R *)Lscale, nullptr, nullptr,
                                         nullptr, list, count, S(s));
    });
}

int sf_gls_corrector_cols(sf_ctx *c, const sf_gls_params *P, double dt, const void *u,
                          const void *v, const void *z_r, const void *Hz, const void *bvf,
                          const void *sustr, const void *svstr, void *tke, void *gls, void *Akv,
                          void *Akt, void *Akk, void *Akp, void *Lscale, const uint8_t *columns,
                          sf_stream s) {
    if (const int rc = gls_checks(P)) return rc;
    return dispatch(c, "sf_gls_corrector", [&](auto *t) {
        using R = std::remove_pointer_t<decltype(t)>;
        return sf::Ops<R>::gls_corrector(c, *P, dt, (const R *)u, (const R *)v, (const R *)z_r,
                                         (const R *)Hz, (const R *)bvf, (const R *)sustr,
                                         (const R *)svstr, (R *)tke, (R *)gls, (R *)Akv, (R *)Akt,
                                         (R *)Akk, (R *)Akp, (R *)Lscale, nullptr, nullptr,
                                         columns, nullptr, nullptr, S(s));
    });
}

int sf_gls_corrector_nnew(sf_ctx *c, const sf_gls_params *P, double dt, const void *u,
                          const void *v, const void *z_r, const void *Hz, const void *bvf,
                          const void *sustr, const void *svstr, const void *tke_nnew,
                          const void *gls_nnew, void *tke, void *gls, void *Akv, void *Akt,
                          void *Akk, void *Akp, void *Lscale, sf_stream s) {
    if (const int rc = gls_checks(P)) return rc;
    if (!tke_nnew || !gls_nnew) return fail(SF_EINVAL, "null tke_nnew/gls_nnew");
    if (tke_nnew == tke || gls_nnew == gls || tke_nnew == gls || gls_nnew == tke)
        return fail(SF_EINVAL, "tke_nnew/gls_nnew must not alias tke/gls (the old level is read "
                               "after the new one is formed)");
    return dispatch(c, "sf_gls_corrector_nnew", [&](auto *t) {
        using R = std::remove_pointer_t<decltype(t)>;
        return sf::Ops<R>::gls_corrector(c, *P, dt, (const R *)u, (const R *)v, (const R *)z_r,
                                         (const R *)Hz, (const R *)bvf, (const R *)sustr,
                                         (const R *)svstr, (R *)tke, (R *)gls, (R *)Akv, (R *)Akt,
                                         (R *)Akk, (R *)Akp, (R *)Lscale, (const R *)tke_nnew,
                                         (const R *)gls_nnew, nullptr, nullptr, nullptr, S(s));
    });
}

int sf_gls_advect(sf_ctx *c, const sf_gls_params *P, double dt, double gadv, const void *Huon,
                  const void *Hvom, const void *W, const void *tke_aux, const void *gls_aux,
                  void *tke_nnew, void *gls_nnew, sf_stream s) {
    if (!P) return fail(SF_EINVAL, "null GLS parameters");
    if (c && c->N < 3) return fail(SF_EUNSUPPORTED, "GLS advection needs N >= 3 levels");
    if (tke_aux == tke_nnew || gls_aux == gls_nnew || tke_aux == gls_nnew || gls_aux == tke_nnew)
        return fail(SF_EINVAL, "the auxiliary and new levels must be distinct arrays");
    return dispatch(c, "sf_gls_advect", [&](auto *t) {
        using R = std::remove_pointer_t<decltype(t)>;
        return sf::Ops<R>::gls_advect(c, dt, gadv, P->Kmin, P->Pmin, (const R *)Huon,
                                      (const R *)Hvom, (const R *)W, (const R *)tke_aux,
                                      (const R *)gls_aux, (R *)tke_nnew, (R *)gls_nnew, S(s));
    });
}

int sf_gls_predictor(sf_ctx *c, double dt, int first_step, const void *Huon, const void *Hvom,
                     const void *W, const void *Hz, const void *tke_nstp, const void *tke_indx,
                     void *tke_aux, void *tke_nnew, const void *gls_nstp, const void *gls_indx,
                     void *gls_aux, void *gls_nnew, void *Hz_half, sf_stream s) {
    if (c && c->N < 3) return fail(SF_EUNSUPPORTED, "the GLS predictor needs N >= 3 levels");
    constexpr double kGamma = 1.0 / 6.0;   // AM3 weight of the half-step interpolation
    sf::GlsPre pc;
    if (first_step) {
        pc.c1 = 1.0;
        pc.c2 = 0.0;
        pc.c3 = 0.5 * dt;
        tke_indx = tke_nstp;
        gls_indx = gls_nstp;
    } else {
        pc.c1 = 0.5 + kGamma;
        pc.c2 = 0.5 - kGamma;
        pc.c3 = (1.0 - kGamma) * dt;
    }
    return dispatch(c, "sf_gls_predictor", [&](auto *t) {
        using R = std::remove_pointer_t<decltype(t)>;
        return sf::Ops<R>::gls_prestep(c, pc, (const R *)Huon, (const R *)Hvom,
                                         (const R *)W, (const R *)Hz, (const R *)tke_nstp,
                                         (const R *)tke_indx, (R *)tke_aux, (R *)tke_nnew,
                                         (const R *)gls_nstp, (const R *)gls_indx, (R *)gls_aux,
                                         (R *)gls_nnew, (R *)Hz_half, S(s));
    });
}

int sf_obc_volcons(sf_ctx *c, const void *zeta, void *ubar, void *vbar, int edges, int correct,
                   double *out, sf_stream s) {
    if (!out) return fail(SF_EINVAL, "null output");
    if (edges < 0 || edges > 15) return fail(SF_EINVAL, "edges is a mask of W=1, E=2, S=4, N=8");
    return dispatch(c, "sf_obc_volcons", [&](auto *t) {
        using R = std::remove_pointer_t<decltype(t)>;
        return sf::Ops<R>::obc_volcons(c, (const R *)zeta, (R *)ubar, (R *)vbar, edges, correct,
                                       out, S(s));
    });
}

int sf_analytic_bvf(sf_ctx *c, const void *z_w, double dT, double zscale, double alpha, double g,
                    void *bvf, sf_stream s) {
    if (!(zscale > 0.0)) return fail(SF_EINVAL, "zscale must be positive");
    return dispatch(c, "sf_analytic_bvf", [&](auto *t) {
        using R = std::remove_pointer_t<decltype(t)>;
        return sf::Ops<R>::analytic_bvf(c, (const R *)z_w, dT, zscale, g * alpha, (R *)bvf, S(s));
    });
}

}  // extern "C"
