// Host runtime of libmbgpu.so: the C ABI of include/mumblebee_gpu.h.
//
// Problems are kept host-side in the reference's block form.  A solver or a batch runs the
// symbolic analysis (symbkkt, src/IPM/src/kkt/kkt.jl:23-53, with the ordering restated in
// mb_symbolic.hpp), packs every instance into a handful of device arenas (a few large copies, no
// per-array transfers) and launches the batched solver kernel of mb_solver.cu.  Nothing numeric
// runs on the host: equilibration, BᵀB, factorization and the iteration are all on the device.
#include <cuda_runtime.h>
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <atomic>
#include <chrono>
#include <cstdlib>
#include <mutex>
#include <unordered_map>
#include <map>
#include <memory>
#include <string>
#include <thread>
#include <vector>

#include "../../include/mumblebee_gpu.h"
#include "mb_internal.h"
#include "mb_symbolic.hpp"

extern "C" int mb_launch_batch(const mb::DevInst* d_inst, int ninst, int mode, const mb::Settings* set,
                               int* d_counter, int grid, int fp32, cudaStream_t stream);
extern "C" int mb_launch_coop(const mb::DevInst* d_inst, int mode, const mb::Settings* set, mb::CoopCtl* d_ctl,
                              int grid, cudaStream_t stream);
extern "C" int mb_coop_grid(int device, int nsm);
extern "C" int mb_launch_twomv(const mb::TwoMv* a, cudaStream_t st);
// the tensor-core build of the solver kernels (mb_solver_tc.cu): same arguments
extern "C" int mb_launch_batch_tc(const mb::DevInst* d_inst, int ninst, int mode, const mb::Settings* set,
                                  int* d_counter, int grid, int fp32, cudaStream_t stream);
extern "C" int mb_launch_coop_tc(const mb::DevInst* d_inst, int mode, const mb::Settings* set, mb::CoopCtl* d_ctl,
                                 int grid, cudaStream_t stream);
extern "C" int mb_coop_grid_tc(int device, int nsm);

// Which build of the solver kernels a launch uses.  The tensor-core build (FP32 update tiles on
// tcgen05) runs one CTA per SM, the default build two, which the batched path needs to hide its
// latency; so with settings.fp32_tiles left to the runtime (0) the tensor cores serve only a lone
// grid-cooperative instance with an FP32 factor, where the large fronts' update tiles dominate.
// 1 always takes the FFMA tiles, 2 always the tensor cores (when an FP32 factor runs at all).
static bool use_tc_build(const mb_settings& s, bool coop) {
    if (s.precision == MB_PREC_FP64 || s.fp32_tiles == 1) return false;
    return s.fp32_tiles == 2 || coop;
}
static int launch_coop(const mb_settings& s, const mb::DevInst* d_inst, int mode, const mb::Settings* ds,
                       mb::CoopCtl* d_ctl, int device, int nsm, cudaStream_t st) {
    return use_tc_build(s, true) ? mb_launch_coop_tc(d_inst, mode, ds, d_ctl, mb_coop_grid_tc(device, nsm), st)
                                 : mb_launch_coop(d_inst, mode, ds, d_ctl, mb_coop_grid(device, nsm), st);
}
static int launch_batch(const mb_settings& s, const mb::DevInst* d_inst, int ninst, int mode, const mb::Settings* ds,
                        int* d_counter, int grid, cudaStream_t st) {
    const int fp32 = s.precision == MB_PREC_FP32;
    return use_tc_build(s, false) ? mb_launch_batch_tc(d_inst, ninst, mode, ds, d_counter, grid, fp32, st)
                                  : mb_launch_batch(d_inst, ninst, mode, ds, d_counter, grid, fp32, st);
}

using mbh::i64;

// Device and pinned-host blocks freed by a batch are kept on the context and handed to the next
// batch that fits (a block at most twice the request), so repeated batch solves pay neither
// cudaMalloc nor the device-wide synchronisation of cudaFree.  A block returns to the cache only
// after its batch's results were read back; a failed cudaMalloc empties the cache and retries.
struct BlockCache {
    std::mutex mu;
    std::multimap<size_t, void*> freeb;          // size -> block
    std::unordered_map<void*, size_t> size;      // every block this cache handed out or holds
    size_t held = 0;
    static constexpr size_t LIMIT = (size_t)64 << 30;
};

struct mb_ctx {
    int device = 0;
    int nsm = 148;
    cudaStream_t stream = nullptr;
    std::string err;
    BlockCache dev, host;
};

static cudaError_t cache_alloc(mb_ctx* ctx, BlockCache& c, bool dev, void** p, size_t bytes) {
    bytes = std::max<size_t>(bytes, 256);
    {
        std::lock_guard<std::mutex> g(c.mu);
        auto it = c.freeb.lower_bound(bytes);
        if (it != c.freeb.end() && it->first <= 2 * bytes) {
            *p = it->second; c.held -= it->first; c.freeb.erase(it);
            return cudaSuccess;
        }
    }
    cudaError_t e = dev ? cudaMalloc(p, bytes) : cudaMallocHost(p, bytes);
    if (e != cudaSuccess) {   // give the cached blocks back to the driver and retry once
        cudaGetLastError();
        std::lock_guard<std::mutex> g(c.mu);
        for (auto& kv : c.freeb) { if (dev) cudaFree(kv.second); else cudaFreeHost(kv.second); c.size.erase(kv.second); }
        c.freeb.clear(); c.held = 0;
        e = dev ? cudaMalloc(p, bytes) : cudaMallocHost(p, bytes);
    }
    if (e == cudaSuccess) { std::lock_guard<std::mutex> g(c.mu); c.size[*p] = bytes; }
    (void)ctx;
    return e;
}
static void cache_free(BlockCache& c, bool dev, void* p) {
    if (!p) return;
    std::lock_guard<std::mutex> g(c.mu);
    auto it = c.size.find(p);
    if (it == c.size.end()) { if (dev) cudaFree(p); else cudaFreeHost(p); return; }
    if (c.held + it->second <= BlockCache::LIMIT) { c.freeb.insert({it->second, p}); c.held += it->second; return; }
    c.size.erase(it);
    if (dev) cudaFree(p); else cudaFreeHost(p);
}
static void cache_clear(BlockCache& c, bool dev) {
    std::lock_guard<std::mutex> g(c.mu);
    for (auto& kv : c.freeb) { if (dev) cudaFree(kv.second); else cudaFreeHost(kv.second); }
    c.freeb.clear(); c.size.clear(); c.held = 0;
}

struct mb_problem {
    mb_ctx* ctx = nullptr;
    mbh::BSM Q, B;
    std::vector<double> f, g;
    double mu = 0;
    std::vector<int32_t> kind;
    std::vector<double> param;
    std::vector<i64> P1, P2;   // 0-based user row / column of each problem row / column
};

static int fail(mb_ctx* ctx, int code, const std::string& msg) {
    if (ctx) ctx->err = msg;
    return code;
}
#define CUDA_TRY(ctx, call)                                                                         \
    do {                                                                                            \
        cudaError_t e_ = (call);                                                                    \
        if (e_ != cudaSuccess) return fail(ctx, MB_E_CUDA, std::string(#call ": ") + cudaGetErrorString(e_)); \
    } while (0)

// ---------------------------------------------------------------------------------------------
// symbolic: the vertex order (minimum degree + etree postorder) and the fronts
// ---------------------------------------------------------------------------------------------
struct Sym {
    std::vector<i64> vperm;    // problem vertex of each solver vertex
    mbh::Fronts fr;
};

static Sym do_symbolic_(const mb_problem* P);

// The symbolic analysis depends only on the sparsity structure: the block-column layout and arc
// pattern of B and Q and the vertex weights.  Batches and request streams repeat structures
// (portfolio instances of the same size, re-solved models), so analyses are kept in a bounded
// cache keyed by that structure; a hit is checked against the full key, never the hash alone.
struct SymKey {
    std::vector<i64> data;
    uint64_t hash = 0;
    bool operator==(const SymKey& o) const { return hash == o.hash && data == o.data; }
};
struct SymKeyHash { size_t operator()(const SymKey& k) const { return (size_t)k.hash; } };

static SymKey sym_key(const mb_problem* P) {
    SymKey k;
    const mbh::BSM &B = P->B, &Q = P->Q;
    auto add = [&](const std::vector<i64>& v) { k.data.push_back((i64)v.size()); k.data.insert(k.data.end(), v.begin(), v.end()); };
    k.data.push_back(B.nvtx); k.data.push_back(B.nout);
    add(B.xcol); add(B.xrow); add(B.xsrc); add(B.tgt); add(Q.xsrc); add(Q.tgt);
    uint64_t h = 1469598103934665603ull;   // FNV-1a over the 64-bit words
    for (i64 x : k.data) { h ^= (uint64_t)x; h *= 1099511628211ull; }
    k.hash = h;
    return k;
}

static std::mutex g_sym_mu;
static std::unordered_map<SymKey, std::shared_ptr<const Sym>, SymKeyHash> g_sym_cache;
constexpr size_t SYM_CACHE_MAX = 4096;

static Sym do_symbolic(const mb_problem* P) {
    SymKey key = sym_key(P);
    {
        std::lock_guard<std::mutex> lk(g_sym_mu);
        auto it = g_sym_cache.find(key);
        if (it != g_sym_cache.end()) return *it->second;
    }
    auto S = std::make_shared<const Sym>(do_symbolic_(P));
    std::lock_guard<std::mutex> lk(g_sym_mu);
    if (g_sym_cache.size() >= SYM_CACHE_MAX) g_sym_cache.clear();
    g_sym_cache.emplace(std::move(key), S);
    return *S;
}

static Sym do_symbolic_(const mb_problem* P) {
    Sym S;
    const mbh::BSM& B = P->B;
    i64 nv = B.nvtx;
    auto adj = mbh::vertex_graph(B, P->Q);
    std::vector<i64> w(nv);
    for (i64 v = 0; v < nv; ++v) w[v] = B.ncols(v);
    std::vector<i64> order = mbh::minimum_degree(adj, w);
    std::vector<i64> inv(nv);
    for (i64 k = 0; k < nv; ++k) inv[order[k]] = k;
    std::vector<std::vector<i64>> adj2(nv);
    std::vector<i64> w2(nv);
    for (i64 k = 0; k < nv; ++k) {
        i64 v = order[k];
        w2[k] = w[v];
        for (i64 u : adj[v]) adj2[k].push_back(inv[u]);
    }
    S.fr = mbh::analyze(adj2, w2);
    S.vperm.resize(nv);
    for (i64 k = 0; k < nv; ++k) S.vperm[k] = order[S.fr.postperm[k]];
    return S;
}

// ---------------------------------------------------------------------------------------------
// packing instances into device arenas
// ---------------------------------------------------------------------------------------------
// vector storage whose resize leaves new elements uninitialised (arenas are filled by copies)
template <class T>
struct NoInitAlloc : std::allocator<T> {
    using value_type = T;
    NoInitAlloc() = default;
    template <class U> NoInitAlloc(const NoInitAlloc<U>&) {}
    template <class U> struct rebind { using other = NoInitAlloc<U>; };
    template <class U> void construct(U* p) { ::new (static_cast<void*>(p)) U; }
    template <class U, class... Args> void construct(U* p, Args&&... args) { ::new (static_cast<void*>(p)) U(std::forward<Args>(args)...); }
};

template <class T>
struct Arena {
    std::vector<T, NoInitAlloc<T>> h;
    size_t n = 0;                 // for device-only arenas (no host image)
    bool host = true;
    static size_t al(size_t x) { return (x + 31) / 32 * 32; }
    size_t put(const T* p, size_t k) {
        size_t o = al(h.size());
        h.resize(o + k);
        if (k) std::memcpy(h.data() + o, p, k * sizeof(T));
        return o;
    }
    size_t put(const std::vector<T>& v) { return put(v.data(), v.size()); }
    size_t take(size_t k) {        // reserve without data
        if (host) { size_t o = al(h.size()); h.resize(o + k, T(0)); return o; }
        size_t o = al(n); n = o + k; return o;
    }
    size_t size() const { return host ? h.size() : n; }
};

static std::vector<int32_t> to32(const std::vector<i64>& v) { return std::vector<int32_t>(v.begin(), v.end()); }

// offsets of one instance's arrays in the arenas
struct InstPlan {
    i64 n, m, nvtx, nfront, nu;
    int has_p0, has_d0, has_y0;
    double mut;
    int wsize;
    i64 fsize;
    double fflops;            // algorithmic flops of one factorization
    i64 Bnnz, Qnnz, nqoff;
    i64 nBlongr, nBlongc, nhlong;
    // i32
    size_t xcol, colvtx, cfront, Brptr, Bcidx, Bcptr, Bridx, Bcpos, Qrptr, Qcidx, Qcptr, Qridx, Qcpos, hdld, qoffk;
    size_t Blongr, Blongc, hlong, hflag;
    size_t sbrp, sbrow, sbloc, fchp, fch;   // stable factor: B rows per front, their front positions, children
    size_t kind, fres0, fnres, fnsep, fparent, fsepp, fsep, frel;
    // i64
    size_t hdoff, hdpos, qoffpos, cxblk, fptr, qd0off;
    // double in
    size_t Bval, Qval, Qd, f, g, kpar, p, d, y;
    // work
    size_t wBval, wQval, wQd, Hd, Finit, pscl, yscl, vn, vm, vv, work, uhist, cghist, cache, cache2, wf, wg, wp, wd, wy, swork;
    // factor (bytes)
    size_t F;
    // out
    size_t po, dout, yo, scal, hist;
    // status words
    size_t status;
    // host-side mapping for results
    std::vector<i64> colmap;   // user column of each solver column
    std::vector<i64> rowmap;   // user row of each solver row
};

struct Packed {
    Arena<int32_t> i32;
    Arena<i64> i64a;
    Arena<double> din;
    Arena<double> work;       // device-only
    Arena<double> out;        // device-only (copied back through pinned staging)
    Arena<int32_t> ost;       // device-only status words (copied back)
    size_t fbytes = 0;        // factor arena, bytes
    std::vector<InstPlan> plans;
    Packed() { work.host = false; out.host = false; ost.host = false; }
    size_t device_bytes() const {
        return i32.size() * 4 + i64a.size() * 8 + din.size() * 8 + work.size() * 8 + out.size() * 8 +
               ost.size() * 4 + fbytes;
    }
};

// cachesize / workspacesize / degree  (soc.jl:116-134, tdc.jl:122-143, pos.jl:21-31, noc.jl:20-28,
// sdp.jl:41-70: an SDP block of svec length n has order d = triroot(n), cache R | S | s = 2d² + d
// plus the scaling point W (d², for the structured H x), workspace max(3d², 2d² + 2d))
static int64_t triroot(i64 n) {
    int64_t t = 1 + 8 * n, r = (int64_t)std::sqrt((double)t);
    while (r * r > t) --r;
    while ((r + 1) * (r + 1) <= t) ++r;
    return (r - 1) / 2;
}
static int64_t cone_cachesize(int k, i64 n) {
    if (k == MB_CONE_SDP) { int64_t d = triroot(n); return 3 * d * d + d; }
    return k == MB_CONE_SOC ? 5 + n : ((k == MB_CONE_EXP || k == MB_CONE_POW) ? 19 : 0);
}
static int64_t cone_workspacesize(int k, i64 n) {
    if (k == MB_CONE_SDP) { int64_t d = triroot(n); return std::max<int64_t>(3 * d * d, 2 * d * d + 2 * d); }
    return k == MB_CONE_SOC ? 2 * n : 0;
}
static int64_t cone_degree(int k, i64 n) {
    if (k == MB_CONE_SDP) return triroot(n);
    return k == MB_CONE_POS ? n : (k == MB_CONE_SOC ? 2 : ((k == MB_CONE_EXP || k == MB_CONE_POW) ? 3 : 0));
}

// Build one instance into its own (local) Packed: symbkkt (kkt/kkt.jl:23-53) with the host ordering,
// the device index structures, the front placement of H and every arena offset.  Thread-safe: the
// problem is only read.
static int plan_instance(const mb_problem* P, const mb_settings& set, const double* p0, const double* d0,
                         const double* y0, Packed& pk, std::string& err) {
    Sym sym = do_symbolic(P);
    const auto& vp = sym.vperm;
    // with the identity order, selectvtxs is a copy, and the double transpose of halfselectvtxs
    // returns Q itself when each column's arcs are already in ascending target order: skip them
    bool ident = true;
    for (size_t k = 0; k < vp.size() && ident; ++k) ident = vp[k] == (i64)k;
    bool qsorted = ident;
    for (i64 v = 0; v < P->Q.nvtx && qsorted; ++v)
        for (i64 e = P->Q.xsrc[v] + 1; e < P->Q.xsrc[v + 1] && qsorted; ++e) qsorted = P->Q.tgt[e - 1] < P->Q.tgt[e];
    mbh::BSM Bp, Qp;
    if (!ident) Bp = mbh::selectvtxs(P->B, vp);
    if (!qsorted) Qp = mbh::blockdiag(P->Q) ? mbh::select_blockdiag(P->Q, vp)
                                            : mbh::halfselectvtxs(mbh::halfselectvtxs(P->Q, vp), vp);
    const mbh::BSM& B = ident ? P->B : Bp;
    const mbh::BSM& Q = qsorted ? P->Q : Qp;
    const mbh::Fronts& fr = sym.fr;
    InstPlan ip;
    const i64 n = B.ncol, m = B.nrow, nv = B.nvtx;
    ip.n = n; ip.m = m; ip.nvtx = nv; ip.nfront = fr.nfront;
    ip.mut = P->mu;
    for (i64 v = 0; v < nv; ++v) {
        int k = P->kind[vp[v]];
        if (k == MB_CONE_SDP && triroot(B.ncols(v)) * (triroot(B.ncols(v)) + 1) / 2 != B.ncols(v)) {
            err = "a semidefinite cone's dimension must be d(d+1)/2"; return MB_E_ARG;
        }
        if ((k == MB_CONE_EXP || k == MB_CONE_POW) && B.ncols(v) != 3) { err = "exponential/power cones have dimension 3"; return MB_E_ARG; }
        if (k == MB_CONE_POW && !(P->param[vp[v]] > 0 && P->param[vp[v]] < 1)) { err = "PowerCone needs 0 < α < 1"; return MB_E_ARG; }
    }
    // column map: solver column -> problem column -> user column
    std::vector<i64> cperm;
    cperm.reserve(n);
    for (i64 k = 0; k < nv; ++k) for (i64 j = P->B.xcol[vp[k]]; j < P->B.xcol[vp[k] + 1]; ++j) cperm.push_back(j);
    ip.colmap.resize(n); ip.rowmap.resize(m);
    for (i64 i = 0; i < n; ++i) ip.colmap[i] = P->P2[cperm[i]];
    for (i64 i = 0; i < m; ++i) ip.rowmap[i] = P->P1[i];
    std::vector<i64> colvtx(n), cfront(n);
    for (i64 v = 0; v < nv; ++v) for (i64 j = B.xcol[v]; j < B.xcol[v + 1]; ++j) { colvtx[j] = v; cfront[j] = fr.vfront[v]; }
    // scalar nonzeros: CSR + CSC (CSC entries carry their CSR position).  With `skipdiag`, the
    // entries inside the diagonal blocks are left out (they live in the dense Qd blocks).  Each
    // stored block is read once, contiguously; its nonzeros, gathered arc by arc in the vertex's
    // arc order, are counting-sorted (stably) by column, so within a column the entries come arc by
    // arc and each block's rows in order: the order a column-by-column scan of the arcs gives.
    auto scalar = [&](const mbh::BSM& A, bool skipdiag, std::vector<i64>& rptr, std::vector<i64>& cidx,
                      std::vector<double>& val, std::vector<i64>& cptr, std::vector<i64>& ridx, std::vector<i64>& cpos) {
        std::vector<i64> tr, tc; std::vector<double> tv;   // nonzeros in arc order
        rptr.assign(A.nrow + 1, 0); cptr.assign(A.ncol + 1, 0);
        for (i64 v = 0; v < A.nvtx; ++v) {
            const i64 nc = A.ncols(v), c0 = A.xcol[v];
            for (i64 e = A.xsrc[v]; e < A.xsrc[v + 1]; ++e) {
                const i64 u = A.tgt[e];
                if (skipdiag && u == v) continue;
                const i64 nr = A.nrows(u), r0 = A.xrow[u];
                const double* blk = A.val.data() + A.xblk[e];
                for (i64 jl = 0; jl < nc; ++jl)
                    for (i64 il = 0; il < nr; ++il)
                        if (blk[jl * nr + il] != 0) {
                            tr.push_back(r0 + il); tc.push_back(c0 + jl); tv.push_back(blk[jl * nr + il]);
                            rptr[r0 + il + 1]++; cptr[c0 + jl + 1]++;
                        }
            }
        }
        for (i64 i = 0; i < A.nrow; ++i) rptr[i + 1] += rptr[i];
        for (i64 j = 0; j < A.ncol; ++j) cptr[j + 1] += cptr[j];
        const i64 nnz = (i64)tr.size();
        std::vector<double> cv(nnz);
        ridx.assign(nnz, 0);
        std::vector<i64> pc(cptr.begin(), cptr.end() - 1);
        for (i64 t = 0; t < nnz; ++t) { const i64 k = pc[tc[t]]++; ridx[k] = tr[t]; cv[k] = tv[t]; }
        cidx.assign(nnz, 0); val.assign(nnz, 0); cpos.assign(nnz, 0);
        std::vector<i64> rc(rptr.begin(), rptr.end() - 1);
        for (i64 j = 0; j < A.ncol; ++j)   // CSR by a stable counting sort of the CSC entries
            for (i64 k = cptr[j]; k < cptr[j + 1]; ++k) {
                const i64 q = rc[ridx[k]]++;
                cidx[q] = j; val[q] = cv[k]; cpos[k] = q;
            }
    };
    std::vector<i64> Brptr, Bcidx, Bcptr, Bridx, Bcpos, Qrptr, Qcidx, Qcptr, Qridx, Qcpos;
    std::vector<double> Bval, Qval;
    scalar(B, false, Brptr, Bcidx, Bval, Bcptr, Bridx, Bcpos);
    scalar(Q, true, Qrptr, Qcidx, Qval, Qcptr, Qridx, Qcpos);
    ip.Bnnz = (i64)Bval.size(); ip.Qnnz = (i64)Qval.size();
    // front row position of scalar row s in front f
    auto rowpos = [&](i64 f, i64 srow) -> i64 {
        i64 r0 = fr.res0[f], nres = fr.nres[f];
        if (srow >= r0 && srow < r0 + nres) return srow - r0;
        auto it = std::lower_bound(fr.sep[f].begin(), fr.sep[f].end(), srow);
        if (it == fr.sep[f].end() || *it != srow) return -1;
        return nres + (i64)(it - fr.sep[f].begin());
    };
    // dense diagonal blocks of Q and their place in F; every non-free cone needs one (cone.jl:146-174)
    // Only the nonzero blocks are stored (Qd, one after another; qd0off[v] = -1 for a zero or absent
    // block): the device zero-fills the rest of its working copy, so an instance whose large cone
    // blocks carry no Q uploads none of them.
    std::vector<i64> hdoff(nv + 1, 0), hdpos(nv, 0), hdld(nv, 0), qd0off(nv, -1);
    for (i64 v = 0; v < nv; ++v) hdoff[v + 1] = hdoff[v] + B.ncols(v) * B.ncols(v);
    std::vector<double> Qd;
    for (i64 v = 0; v < nv; ++v) {
        bool found = false;
        for (i64 e = Q.xsrc[v]; e < Q.xsrc[v + 1]; ++e)
            if (Q.tgt[e] == v) {
                found = true;
                const auto b0 = Q.val.begin() + Q.xblk[e], b1 = Q.val.begin() + Q.xblk[e + 1];
                if (std::any_of(b0, b1, [](double x) { return x != 0.0; })) {
                    qd0off[v] = (i64)Qd.size();
                    Qd.insert(Qd.end(), b0, b1);
                }
            }
        if (!found && P->kind[vp[v]] != MB_CONE_FREE) { err = "Q lacks the diagonal block of a cone vertex"; return MB_E_ARG; }
        i64 f = fr.vfront[v], ld = mb::front_ld(fr.nres[f] + (i64)fr.sep[f].size());
        hdpos[v] = fr.fptr[f] + (B.xcol[v] - fr.res0[f]) * (ld + 1);
        hdld[v] = ld;
    }
    // off-diagonal-block nonzeros of Q in the lower triangle and their F offsets
    std::vector<i64> qoffk, qoffpos;
    for (i64 i = 0; i < n; ++i)
        for (i64 k = Qrptr[i]; k < Qrptr[i + 1]; ++k) {
            i64 j = Qcidx[k];
            if (i < j) continue;
            i64 f = cfront[j], ld = mb::front_ld(fr.nres[f] + (i64)fr.sep[f].size());
            i64 rp = rowpos(f, i);
            if (rp < 0) { err = "internal: Q entry outside the front structure"; return MB_E_ARG; }
            qoffk.push_back(k);
            qoffpos.push_back(fr.fptr[f] + rp + (j - fr.res0[f]) * ld);
        }
    ip.nqoff = (i64)qoffk.size();
    // rows and columns with more than LONG_ROW terms in the sparse products: a warp each on the device.
    // A row of the H (or Q) product has its vertex block's nc terms, or one when the block is applied in
    // structured form (an SOC or SDP vertex whose Q block is zero), plus its off-diagonal-block Q terms.
    auto longlist = [](const std::vector<i64>& ptr) {
        std::vector<i64> L;
        for (size_t i = 0; i + 1 < ptr.size(); ++i) if (ptr[i + 1] - ptr[i] > mb::LONG_ROW) L.push_back((i64)i);
        return L;
    };
    std::vector<i64> Blongr = longlist(Brptr), Blongc = longlist(Bcptr), hlong, hflag(n, 0);
    for (i64 v = 0; v < nv; ++v) {
        const i64 nc = B.ncols(v);
        const int kv = P->kind[vp[v]];
        const bool qzero = qd0off[v] < 0;
        const bool structured = (kv == MB_CONE_SOC || kv == MB_CONE_SDP) && qzero;
        const i64 blk = structured ? 1 : nc;
        for (i64 i = B.xcol[v]; i < B.xcol[v + 1]; ++i) {
            if (blk + (Qrptr[i + 1] - Qrptr[i]) > mb::LONG_ROW) { hflag[i] |= 1; hlong.push_back(i); }
            if (qzero) hflag[i] |= 2;   // the vertex's Q block is zero: equilibration skips it
        }
    }
    ip.nBlongr = (i64)Blongr.size(); ip.nBlongc = (i64)Blongc.size(); ip.nhlong = (i64)hlong.size();
    // fronts
    std::vector<i64> fnsep(fr.nfront), fsepp(fr.nfront + 1, 0), fsep, frel;
    for (i64 f = 0; f < fr.nfront; ++f) {
        fnsep[f] = (i64)fr.sep[f].size();
        fsepp[f + 1] = fsepp[f] + fnsep[f];
        fsep.insert(fsep.end(), fr.sep[f].begin(), fr.sep[f].end());
        if (fr.parent[f] >= 0) frel.insert(frel.end(), fr.rel[f].begin(), fr.rel[f].end());
        else frel.insert(frel.end(), fr.sep[f].size(), 0);
    }
    // StableUzawaSolver (kkt/uzawa.jl:32-67,117-163): each nonempty row of B goes to the front of its
    // first column (its columns are a clique of BᵀB, so they all lie in that front's rows), with the
    // front position of each entry; the children of each front; the QR scratch, the largest
    // (rows x columns) front of the stacked system [√δ Uᵀ; B rows; children's triangles]
    std::vector<i64> sbrp(fr.nfront + 1, 0), sbrow, sbloc, fchp(fr.nfront + 1, 0), fch;
    i64 sworksz = 0;
    if (set.stable) {
        if (ip.nqoff > 0) { err = "stable=true needs Q without off-diagonal blocks (uzawa.jl:136 copies H into its block diagonal)"; return MB_E_UNSUPPORTED; }
        std::vector<i64> rf(m, -1);
        sbloc.assign(ip.Bnnz, 0);
        for (i64 i = 0; i < m; ++i) {
            if (Brptr[i + 1] == Brptr[i]) continue;
            const i64 f = cfront[Bcidx[Brptr[i]]];
            rf[i] = f;
            sbrp[f + 1]++;
            for (i64 k = Brptr[i]; k < Brptr[i + 1]; ++k) {
                sbloc[k] = rowpos(f, Bcidx[k]);
                if (sbloc[k] < 0) { err = "internal: a row of B outside its front"; return MB_E_ARG; }
            }
        }
        for (i64 f = 0; f < fr.nfront; ++f) sbrp[f + 1] += sbrp[f];
        sbrow.assign(sbrp[fr.nfront], 0);
        std::vector<i64> pos(sbrp.begin(), sbrp.end() - 1);
        for (i64 i = 0; i < m; ++i) if (rf[i] >= 0) sbrow[pos[rf[i]]++] = i;
        for (i64 f = 0; f < fr.nfront; ++f) if (fr.parent[f] >= 0) fchp[fr.parent[f] + 1]++;
        for (i64 f = 0; f < fr.nfront; ++f) fchp[f + 1] += fchp[f];
        fch.assign(fchp[fr.nfront], 0);
        std::vector<i64> cp(fchp.begin(), fchp.end() - 1);
        for (i64 f = 0; f < fr.nfront; ++f) if (fr.parent[f] >= 0) fch[cp[fr.parent[f]]++] = f;
        for (i64 f = 0; f < fr.nfront; ++f) {
            i64 rows = fr.nres[f] + (sbrp[f + 1] - sbrp[f]);
            for (i64 k = fchp[f]; k < fchp[f + 1]; ++k) rows += fnsep[fch[k]];
            sworksz = std::max(sworksz, rows * (fr.nres[f] + fnsep[f]));
        }
    }
    std::vector<i64> kind(nv), cx(nv + 1, 0);
    std::vector<double> kpar(nv);
    i64 wmax = 1;
    ip.nu = 0;
    for (i64 v = 0; v < nv; ++v) {
        kind[v] = P->kind[vp[v]]; kpar[v] = P->param[vp[v]];
        cx[v + 1] = cx[v] + cone_cachesize((int)kind[v], B.ncols(v));
        wmax = std::max<i64>(wmax, cone_workspacesize((int)kind[v], B.ncols(v)));
        ip.nu += cone_degree((int)kind[v], B.ncols(v));
    }
    ip.wsize = (int)wmax;
    ip.fflops = 0;
    for (i64 f = 0; f < fr.nfront; ++f) {
        double r = (double)fr.nres[f], sp = (double)fr.sep[f].size();
        ip.fflops += r * r * r / 3 + r * r * sp + r * sp * sp;
    }
    // i32 arena
    ip.xcol = pk.i32.put(to32(B.xcol)); ip.colvtx = pk.i32.put(to32(colvtx)); ip.cfront = pk.i32.put(to32(cfront));
    ip.Brptr = pk.i32.put(to32(Brptr)); ip.Bcidx = pk.i32.put(to32(Bcidx)); ip.Bcptr = pk.i32.put(to32(Bcptr));
    ip.Bridx = pk.i32.put(to32(Bridx)); ip.Bcpos = pk.i32.put(to32(Bcpos));
    ip.Qrptr = pk.i32.put(to32(Qrptr)); ip.Qcidx = pk.i32.put(to32(Qcidx)); ip.Qcptr = pk.i32.put(to32(Qcptr));
    ip.Qridx = pk.i32.put(to32(Qridx)); ip.Qcpos = pk.i32.put(to32(Qcpos));
    ip.hdld = pk.i32.put(to32(hdld)); ip.qoffk = pk.i32.put(to32(qoffk)); ip.kind = pk.i32.put(to32(kind));
    ip.fres0 = pk.i32.put(to32(fr.res0)); ip.fnres = pk.i32.put(to32(fr.nres)); ip.fnsep = pk.i32.put(to32(fnsep));
    ip.fparent = pk.i32.put(to32(fr.parent)); ip.fsepp = pk.i32.put(to32(fsepp)); ip.fsep = pk.i32.put(to32(fsep));
    ip.frel = pk.i32.put(to32(frel));
    ip.Blongr = pk.i32.put(to32(Blongr)); ip.Blongc = pk.i32.put(to32(Blongc));
    ip.hlong = pk.i32.put(to32(hlong)); ip.hflag = pk.i32.put(to32(hflag));
    ip.sbrp = pk.i32.put(to32(sbrp)); ip.sbrow = pk.i32.put(to32(sbrow)); ip.sbloc = pk.i32.put(to32(sbloc));
    ip.fchp = pk.i32.put(to32(fchp)); ip.fch = pk.i32.put(to32(fch));
    // i64 arena
    ip.hdoff = pk.i64a.put(hdoff); ip.hdpos = pk.i64a.put(hdpos); ip.qoffpos = pk.i64a.put(qoffpos);
    ip.qd0off = pk.i64a.put(qd0off);
    ip.cxblk = pk.i64a.put(cx); ip.fptr = pk.i64a.put(fr.fptr);
    // values
    std::vector<double> f(n), g(P->g);
    for (i64 i = 0; i < n; ++i) f[i] = P->f[cperm[i]];
    ip.Bval = pk.din.put(Bval); ip.Qval = pk.din.put(Qval); ip.Qd = pk.din.put(Qd);
    ip.f = pk.din.put(f); ip.g = pk.din.put(g); ip.kpar = pk.din.put(kpar);
    std::vector<double> pv(n, 0.0), dv(n, 0.0), yv(m, 0.0);
    ip.has_p0 = p0 != nullptr; ip.has_d0 = d0 != nullptr; ip.has_y0 = y0 != nullptr;
    for (i64 i = 0; i < n; ++i) { if (p0) pv[i] = p0[ip.colmap[i]]; if (d0) dv[i] = d0[ip.colmap[i]]; }
    if (y0) for (i64 i = 0; i < m; ++i) yv[i] = y0[ip.rowmap[i]];
    ip.p = pk.din.put(pv); ip.d = pk.din.put(dv); ip.y = pk.din.put(yv);
    // workspace
    ip.fsize = fr.fsize;
    ip.wBval = pk.work.take(Bval.size()); ip.wQval = pk.work.take(Qval.size()); ip.wQd = pk.work.take(hdoff[nv]);
    ip.Hd = pk.work.take(hdoff[nv]); ip.Finit = pk.work.take(fr.fsize);
    ip.pscl = pk.work.take(n); ip.yscl = pk.work.take(m);
    ip.vn = pk.work.take((size_t)(mb::NVEC_N + 2) * n); ip.vm = pk.work.take((size_t)(mb::NVEC_M + 1) * m);
    ip.vv = pk.work.take((size_t)mb::NVEC_V * nv); ip.work = pk.work.take((size_t)(mb::CTA_THREADS / 32) * wmax);
    ip.uhist = pk.work.take(set.refine_max_iter + 2); ip.cghist = pk.work.take(set.newton_max_iter + 1);
    ip.cache = pk.work.take(std::max<i64>(cx[nv], 1)); ip.cache2 = pk.work.take(std::max<i64>(cx[nv], 1));
    ip.wf = pk.work.take(n); ip.wg = pk.work.take(m); ip.wp = pk.work.take(n); ip.wd = pk.work.take(n); ip.wy = pk.work.take(m);
    ip.swork = pk.work.take(sworksz);
    size_t esz = set.precision == MB_PREC_FP32 ? 4 : 8;   // mixed needs room for the FP64 factor
    ip.F = (pk.fbytes + 255) / 256 * 256;
    pk.fbytes = ip.F + fr.fsize * esz;
    ip.po = pk.out.take(n); ip.dout = pk.out.take(n); ip.yo = pk.out.take(m);
    ip.scal = pk.out.take(mb::NSCAL); ip.hist = pk.out.take((size_t)(set.max_iter + 1) * mb::ROW_DOUBLES);
    ip.status = pk.ost.take(mb::NSTAT);
    pk.plans.push_back(std::move(ip));
    return MB_OK;
}

// append a single-instance Packed to the batch, shifting its offsets
static void merge(Packed& dst, Packed& src) {
    InstPlan ip = std::move(src.plans[0]);
    auto cat = [](auto& D, auto& S) -> size_t {
        size_t base = D.al(D.size());
        if (D.host) { D.h.resize(base); D.h.insert(D.h.end(), S.h.begin(), S.h.end()); }
        else D.n = base + S.size();
        return base;
    };
    size_t b32 = cat(dst.i32, src.i32), b64 = cat(dst.i64a, src.i64a), bin = cat(dst.din, src.din);
    size_t bw = cat(dst.work, src.work), bo = cat(dst.out, src.out), bs = cat(dst.ost, src.ost);
    for (size_t* f : {&ip.xcol, &ip.colvtx, &ip.cfront, &ip.Brptr, &ip.Bcidx, &ip.Bcptr, &ip.Bridx, &ip.Bcpos,
                      &ip.Qrptr, &ip.Qcidx, &ip.Qcptr, &ip.Qridx, &ip.Qcpos, &ip.hdld, &ip.qoffk, &ip.kind,
                      &ip.fres0, &ip.fnres, &ip.fnsep, &ip.fparent, &ip.fsepp, &ip.fsep, &ip.frel,
                      &ip.Blongr, &ip.Blongc, &ip.hlong, &ip.hflag, &ip.sbrp, &ip.sbrow, &ip.sbloc, &ip.fchp, &ip.fch}) *f += b32;
    for (size_t* f : {&ip.hdoff, &ip.hdpos, &ip.qoffpos, &ip.cxblk, &ip.fptr, &ip.qd0off}) *f += b64;
    for (size_t* f : {&ip.Bval, &ip.Qval, &ip.Qd, &ip.f, &ip.g, &ip.kpar, &ip.p, &ip.d, &ip.y}) *f += bin;
    for (size_t* f : {&ip.wBval, &ip.wQval, &ip.wQd, &ip.Hd, &ip.Finit, &ip.pscl, &ip.yscl, &ip.vn, &ip.vm, &ip.vv,
                      &ip.work, &ip.uhist, &ip.cghist, &ip.cache, &ip.cache2, &ip.wf, &ip.wg, &ip.wp, &ip.wd, &ip.wy, &ip.swork}) *f += bw;
    for (size_t* f : {&ip.po, &ip.dout, &ip.yo, &ip.scal, &ip.hist}) *f += bo;
    ip.status += bs;
    size_t fb = (dst.fbytes + 255) / 256 * 256;
    ip.F += fb;
    dst.fbytes = fb + src.fbytes;
    dst.plans.push_back(std::move(ip));
}

namespace {
mb::DevInst static_devinst(const InstPlan& p, int32_t* i32, i64* q64, double* dn, double* wk, double* ot,
                           int32_t* ost, char* F);
}  // namespace

// Work-queue order of a batch: the persistent grid takes instances in DevInst-array order, so the
// array is uploaded largest estimated cost first (LPT: the long solves start early and the short
// ones fill the tail).  Cost = one factorization's flops + 16 x the factor's entries (the
// triangular solves, assembly and matvecs that scale with its size).  Each DevInst carries its own
// output pointers, so the order changes nothing a caller reads back.
static void order_by_cost(std::vector<mb::DevInst>& hi, const std::vector<InstPlan>& plans) {
    if (hi.size() < 2) return;
    std::vector<size_t> idx(hi.size());
    for (size_t k = 0; k < idx.size(); ++k) idx[k] = k;
    auto cost = [&](size_t k) { return plans[k].fflops + 16.0 * (double)plans[k].fsize; };
    std::stable_sort(idx.begin(), idx.end(), [&](size_t a, size_t b) { return cost(a) > cost(b); });
    std::vector<mb::DevInst> out(hi.size());
    for (size_t j = 0; j < idx.size(); ++j) out[j] = hi[idx[j]];
    hi.swap(out);
}

struct mb_batch {
    mb_ctx* ctx = nullptr;
    mb_settings set{};
    std::vector<mb_problem*> probs;
    Packed pk;
    int32_t* d_i32 = nullptr;
    int32_t* d_ost = nullptr;
    i64* d_i64 = nullptr;
    double* d_din = nullptr;
    double* d_work = nullptr;
    double* d_out = nullptr;
    void* d_F = nullptr;
    mb::DevInst* d_inst = nullptr;
    int* d_counter = nullptr;
    mb::CoopCtl* d_coop = nullptr;   // grid-cooperative mode control block (one large instance)
    int32_t* h_i32 = nullptr;   // pinned mirrors of the status words
    double* h_out = nullptr;    // pinned output staging
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    int64_t launches = 0;
    cudaStream_t own = nullptr;   // the batch's own stream (chunks of a split mb_batch_solve), else ctx's
    cudaStream_t stream() const { return own ? own : ctx->stream; }
    ~mb_batch() {
        if (ctx) {
            cudaStreamSynchronize(stream());   // nothing of this batch may still use a block it returns
            for (void* p : {(void*)d_i32, (void*)d_i64, (void*)d_din, (void*)d_work, (void*)d_out, d_F, (void*)d_inst,
                            (void*)d_counter, (void*)d_ost})
                cache_free(ctx->dev, true, p);
            cache_free(ctx->host, false, h_i32);
            cache_free(ctx->host, false, h_out);
        }
        cudaFree(d_coop);
        if (e0) cudaEventDestroy(e0);
        if (e1) cudaEventDestroy(e1);
        if (own) cudaStreamDestroy(own);
    }
};

static int upload(mb_batch* b) {
    mb_ctx* ctx = b->ctx;
    Packed& pk = b->pk;
    cudaStream_t st = b->stream();
    auto dalloc = [&](void** p, size_t bytes) { return cache_alloc(ctx, ctx->dev, true, p, bytes); };
    auto halloc = [&](void** p, size_t bytes) { return cache_alloc(ctx, ctx->host, false, p, bytes); };
    auto alloc_copy = [&](auto*& dptr, auto& arena) -> int {
        using T = typename std::remove_reference<decltype(arena.h)>::type::value_type;
        size_t bytes = std::max<size_t>(arena.size(), 1) * sizeof(T);
        CUDA_TRY(ctx, dalloc((void**)&dptr, bytes));
        if (arena.host && arena.size()) CUDA_TRY(ctx, cudaMemcpyAsync(dptr, arena.h.data(), arena.size() * sizeof(T), cudaMemcpyHostToDevice, st));
        return MB_OK;
    };
    int rc;
    if ((rc = alloc_copy(b->d_i32, pk.i32))) return rc;
    if ((rc = alloc_copy(b->d_i64, pk.i64a))) return rc;
    if ((rc = alloc_copy(b->d_din, pk.din))) return rc;
    CUDA_TRY(ctx, dalloc((void**)&b->d_work, std::max<size_t>(pk.work.size(), 1) * sizeof(double)));
    CUDA_TRY(ctx, dalloc((void**)&b->d_out, std::max<size_t>(pk.out.size(), 1) * sizeof(double)));
    CUDA_TRY(ctx, dalloc(&b->d_F, std::max<size_t>(pk.fbytes, 256)));
    CUDA_TRY(ctx, dalloc((void**)&b->d_counter, sizeof(int)));
    CUDA_TRY(ctx, halloc((void**)&b->h_out, std::max<size_t>(pk.out.size(), 1) * sizeof(double)));
    const size_t ost_bytes = std::max<size_t>(pk.ost.size(), 1) * sizeof(int32_t);
    CUDA_TRY(ctx, dalloc((void**)&b->d_ost, ost_bytes));
    CUDA_TRY(ctx, halloc((void**)&b->h_i32, ost_bytes));
    // status words zeroed by a copy from the zeroed pinned mirror, not a memset: a memset runs as a
    // kernel, which waits for SMs that a running chunk's persistent grid holds, and the pageable
    // copies queued after it would then hold up the host, and the planning of the next chunk, too
    std::memset(b->h_i32, 0, ost_bytes);
    CUDA_TRY(ctx, cudaMemcpyAsync(b->d_ost, b->h_i32, ost_bytes, cudaMemcpyHostToDevice, st));
    std::vector<mb::DevInst> hi(pk.plans.size());
    for (size_t k = 0; k < pk.plans.size(); ++k)
        hi[k] = static_devinst(pk.plans[k], b->d_i32, b->d_i64, b->d_din, b->d_work, b->d_out, b->d_ost, (char*)b->d_F);
    order_by_cost(hi, pk.plans);
    CUDA_TRY(ctx, dalloc((void**)&b->d_inst, hi.size() * sizeof(mb::DevInst)));
    CUDA_TRY(ctx, cudaMemcpyAsync(b->d_inst, hi.data(), hi.size() * sizeof(mb::DevInst), cudaMemcpyHostToDevice, st));
    CUDA_TRY(ctx, cudaEventCreate(&b->e0));
    CUDA_TRY(ctx, cudaEventCreate(&b->e1));
    CUDA_TRY(ctx, cudaStreamSynchronize(st));
    return MB_OK;
}

static double host_time() {
    return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch()).count();
}
static bool trace_on() {   // MB_TRACE=1 prints the host phases of batch preparation to stderr
    static const bool on = [] { const char* e = std::getenv("MB_TRACE"); return e && e[0] == '1'; }();
    return on;
}

// Concatenate single-instance plans into the batch arenas: offsets first (the layout merge()
// builds), one allocation per arena, then the instances copied in parallel.
static void merge_all(Packed& dst, std::vector<Packed>& src, int nth) {
    const size_t n = src.size();
    std::vector<size_t> b32(n), b64(n), bin(n), bw(n), bo(n), bs(n), bf(n);
    size_t t32 = dst.i32.size(), t64 = dst.i64a.size(), tin = dst.din.size(), tw = dst.work.size(),
           to = dst.out.size(), ts = dst.ost.size(), tf = dst.fbytes;
    auto al = [](size_t x) { return (x + 31) / 32 * 32; };
    for (size_t k = 0; k < n; ++k) {
        b32[k] = al(t32); t32 = b32[k] + src[k].i32.size();
        b64[k] = al(t64); t64 = b64[k] + src[k].i64a.size();
        bin[k] = al(tin); tin = bin[k] + src[k].din.size();
        bw[k] = al(tw); tw = bw[k] + src[k].work.size();
        bo[k] = al(to); to = bo[k] + src[k].out.size();
        bs[k] = al(ts); ts = bs[k] + src[k].ost.size();
        bf[k] = (tf + 255) / 256 * 256; tf = bf[k] + src[k].fbytes;
    }
    dst.i32.h.resize(t32); dst.i64a.h.resize(t64); dst.din.h.resize(tin);
    dst.work.n = tw; dst.out.n = to; dst.ost.n = ts; dst.fbytes = tf;
    const size_t p0 = dst.plans.size();
    dst.plans.resize(p0 + n);
    std::atomic<size_t> next{0};
    auto worker = [&]() {
        for (;;) {
            const size_t k = next.fetch_add(1);
            if (k >= n) break;
            Packed& s = src[k];
            if (s.i32.size()) std::memcpy(dst.i32.h.data() + b32[k], s.i32.h.data(), s.i32.size() * sizeof(int32_t));
            if (s.i64a.size()) std::memcpy(dst.i64a.h.data() + b64[k], s.i64a.h.data(), s.i64a.size() * sizeof(i64));
            if (s.din.size()) std::memcpy(dst.din.h.data() + bin[k], s.din.h.data(), s.din.size() * sizeof(double));
            InstPlan ip = std::move(s.plans[0]);
            for (size_t* f : {&ip.xcol, &ip.colvtx, &ip.cfront, &ip.Brptr, &ip.Bcidx, &ip.Bcptr, &ip.Bridx, &ip.Bcpos,
                              &ip.Qrptr, &ip.Qcidx, &ip.Qcptr, &ip.Qridx, &ip.Qcpos, &ip.hdld, &ip.qoffk, &ip.kind,
                              &ip.fres0, &ip.fnres, &ip.fnsep, &ip.fparent, &ip.fsepp, &ip.fsep, &ip.frel,
                      &ip.Blongr, &ip.Blongc, &ip.hlong, &ip.hflag, &ip.sbrp, &ip.sbrow, &ip.sbloc, &ip.fchp, &ip.fch}) *f += b32[k];
            for (size_t* f : {&ip.hdoff, &ip.hdpos, &ip.qoffpos, &ip.cxblk, &ip.fptr, &ip.qd0off}) *f += b64[k];
            for (size_t* f : {&ip.Bval, &ip.Qval, &ip.Qd, &ip.f, &ip.g, &ip.kpar, &ip.p, &ip.d, &ip.y}) *f += bin[k];
            for (size_t* f : {&ip.wBval, &ip.wQval, &ip.wQd, &ip.Hd, &ip.Finit, &ip.pscl, &ip.yscl, &ip.vn, &ip.vm, &ip.vv,
                              &ip.work, &ip.uhist, &ip.cghist, &ip.cache, &ip.cache2, &ip.wf, &ip.wg, &ip.wp, &ip.wd, &ip.wy, &ip.swork}) *f += bw[k];
            for (size_t* f : {&ip.po, &ip.dout, &ip.yo, &ip.scal, &ip.hist}) *f += bo[k];
            ip.status += bs[k];
            ip.F += bf[k];
            dst.plans[p0 + k] = std::move(ip);
            s = Packed();   // release this instance's staging early
        }
    };
    std::vector<std::thread> th;
    for (int t = 1; t < std::max(1, nth); ++t) th.emplace_back(worker);
    worker();
    for (auto& t : th) t.join();
}

static int make_batch(mb_ctx* ctx, mb_problem* const* probs, int32_t nprob, const mb_settings* set,
                      const double* p0, const double* d0, const double* y0, mb_batch** out, bool own_stream = false) {
    if (!ctx || !out || nprob < 0 || (nprob > 0 && !probs)) return fail(ctx, MB_E_ARG, "bad arguments");
    mb_settings s;
    if (set) s = *set; else mb_settings_default(&s);
    if (s.stable && s.precision != MB_PREC_FP64)
        return fail(ctx, MB_E_UNSUPPORTED, "stable=true (StableUzawaSolver) factors in FP64: precision must be 0");
    if (s.max_iter < 0 || s.refine_max_iter < 0 || s.newton_max_iter < 0) return fail(ctx, MB_E_ARG, "negative iteration limit");
    if (s.precision < 0 || s.precision > 2) return fail(ctx, MB_E_ARG, "precision must be 0 (FP64), 1 (FP32) or 2 (mixed)");
    auto b = std::make_unique<mb_batch>();
    b->ctx = ctx; b->set = s;
    const double t_start = host_time();
    CUDA_TRY(ctx, cudaSetDevice(ctx->device));
    if (own_stream) CUDA_TRY(ctx, cudaStreamCreateWithFlags(&b->own, cudaStreamNonBlocking));
    for (int32_t k = 0; k < nprob; ++k) if (!probs[k]) return fail(ctx, MB_E_ARG, "null problem");
    std::vector<Packed> local(nprob);
    std::vector<int> rcs(nprob, 0);
    std::vector<std::string> errs(nprob);
    std::atomic<int32_t> next{0};
    auto worker = [&]() {
        for (;;) {
            int32_t k = next.fetch_add(1);
            if (k >= nprob) break;
            rcs[k] = plan_instance(probs[k], s, p0, d0, y0, local[k], errs[k]);
        }
    };
    int nth = (int)std::min<unsigned>(std::max(1u, std::thread::hardware_concurrency()), (unsigned)std::max(1, nprob));
    std::vector<std::thread> th;
    for (int t = 1; t < nth; ++t) th.emplace_back(worker);
    worker();
    for (auto& t : th) t.join();
    for (int32_t k = 0; k < nprob; ++k) if (rcs[k]) return fail(ctx, rcs[k], errs[k]);
    const double t_plan = host_time();
    merge_all(b->pk, local, nth);
    for (int32_t k = 0; k < nprob; ++k) b->probs.push_back(probs[k]);
    const double t_merge = host_time();
    int rc = upload(b.get());
    if (rc) return rc;
    if (trace_on())
        fprintf(stderr, "mb_batch: %d instances, plan %.1f ms, merge %.1f ms, upload %.1f ms (%d threads)\n", nprob,
                1e3 * (t_plan - t_start), 1e3 * (t_merge - t_plan), 1e3 * (host_time() - t_merge), nth);
    *out = b.release();
    return MB_OK;
}

static int run_batch(mb_batch* b, int mode, int32_t grid, float* ms) {
    mb_ctx* ctx = b->ctx;
    int ninst = (int)b->pk.plans.size();
    if (ninst == 0) { if (ms) *ms = 0; return MB_OK; }
    int g = grid > 0 ? grid : ctx->nsm * mb::CTA_PER_SM;
    g = std::min(g, ninst);
    mb::Settings s;
    static_assert(sizeof(mb::Settings) == sizeof(mb_settings), "settings layout");
    std::memcpy(&s, &b->set, sizeof(s));
    CUDA_TRY(ctx, cudaSetDevice(ctx->device));
    // a lone large instance runs on the whole GPU (grid-cooperative mode)
    const bool coop = ninst == 1 && !b->set.stable && (b->set.large == 1 || (b->set.large == 0 && b->pk.plans[0].fflops >= MB_LARGE_FLOPS));
    if (coop && !b->d_coop) CUDA_TRY(ctx, cudaMalloc((void**)&b->d_coop, sizeof(mb::CoopCtl)));
    cudaStream_t st = b->stream();
    CUDA_TRY(ctx, cudaEventRecord(b->e0, st));
    if (!coop && use_tc_build(b->set, false)) g = std::min({grid > 0 ? grid : ctx->nsm, ctx->nsm, ninst});   // one CTA per SM
    int rc = coop ? launch_coop(b->set, b->d_inst, mode, &s, b->d_coop, ctx->device, ctx->nsm, st)
                  : launch_batch(b->set, b->d_inst, ninst, mode, &s, b->d_counter, g, st);
    if (rc) return fail(ctx, MB_E_CUDA, std::string("launch failed: ") + cudaGetErrorString(cudaGetLastError()));
    b->launches++;
    CUDA_TRY(ctx, cudaEventRecord(b->e1, st));
    if (!ms && b->own) return MB_OK;   // a chunk of a split solve: the caller waits on the stream
    CUDA_TRY(ctx, cudaEventSynchronize(b->e1));
    if (ms) CUDA_TRY(ctx, cudaEventElapsedTime(ms, b->e0, b->e1));
    return MB_OK;
}

static const char* COOP_TIMEOUT_MSG =
    "a grid-barrier wait of the grid-cooperative mode ran past settings.coop_wait; the solve was abandoned";
static const char* TC_TIMEOUT_MSG =
    "a tensor-core completion wait of the FP32 factor ran out; the solve was abandoned";
// status word 7 of an instance: 1 a grid-barrier wait ran out, 2 a tensor-core completion wait did
static const char* timeout_msg(int32_t w) { return w == 2 ? TC_TIMEOUT_MSG : COOP_TIMEOUT_MSG; }

static int fetch_batch(mb_batch* b) {
    mb_ctx* ctx = b->ctx;
    cudaStream_t st = b->stream();
    CUDA_TRY(ctx, cudaMemcpyAsync(b->h_out, b->d_out, std::max<size_t>(b->pk.out.size(), 1) * sizeof(double), cudaMemcpyDeviceToHost, st));
    CUDA_TRY(ctx, cudaMemcpyAsync(b->h_i32, b->d_ost, std::max<size_t>(b->pk.ost.size(), 1) * sizeof(int32_t), cudaMemcpyDeviceToHost, st));
    CUDA_TRY(ctx, cudaStreamSynchronize(st));
    for (const InstPlan& ip : b->pk.plans)
        if (b->h_i32[ip.status + 7]) return fail(ctx, MB_E_TIMEOUT, timeout_msg(b->h_i32[ip.status + 7]));
    return MB_OK;
}

static void unpack_one(const mb_batch* b, size_t k, double* p, double* d, double* y, mb_result* r) {
    const InstPlan& ip = b->pk.plans[k];
    const double* o = b->h_out;
    if (p) for (i64 i = 0; i < ip.n; ++i) p[ip.colmap[i]] = o[ip.po + i];
    if (d) for (i64 i = 0; i < ip.n; ++i) d[ip.colmap[i]] = o[ip.dout + i];
    if (y) for (i64 i = 0; i < ip.m; ++i) y[ip.rowmap[i]] = o[ip.yo + i];
    if (r) {
        const int32_t* st = b->h_i32 + ip.status;
        r->status = st[0]; r->niter = st[1]; r->nfactor_retry = st[2]; r->nfactor = st[3];
        r->nfp32 = st[4]; r->nfallback = st[5];
        r->factor_flops = ip.fflops;
        const double* sc = o + ip.scal;
        r->mu = sc[0]; r->pres = sc[1]; r->dres = sc[2]; r->pobj = sc[3]; r->dobj = sc[4];
        int ns = 0;
        const double* h = o + ip.hist;
        int nr = std::min<int>(st[1], b->set.max_iter + 1);
        for (int i = 0; i < nr; ++i) {
            const double* row = h + (size_t)i * mb::ROW_DOUBLES;
            ns += (int)(row[5] + row[6] + row[8] + row[9]);
        }
        r->nsolve = ns;
    }
}

// ---------------------------------------------------------------------------------------------
// C ABI
// ---------------------------------------------------------------------------------------------
struct mb_solver {
    mb_problem* prob = nullptr;
    std::unique_ptr<mb_batch> b;
    bool done = false;
    int32_t status = MB_CONTINUE;
    double* d_sx = nullptr;   // sensitivity exchange (DevInst::sx), from the first frule / rrule
    ~mb_solver() { if (d_sx && b && b->ctx) cache_free(b->ctx->dev, true, d_sx); }
};

extern "C" {

int mb_version(int32_t* major, int32_t* minor) {
    if (major) *major = 0;
    if (minor) *minor = 1;
    return MB_OK;
}

void mb_settings_default(mb_settings* s) {
    if (!s) return;
    std::memset(s, 0, sizeof(*s));
    s->verbose = 0; s->max_iter = 100; s->scale_max_iter = 10; s->refine_max_iter = 10; s->newton_max_iter = 100;
    s->stable = 0; s->precision = MB_PREC_FP64; s->large = 0; s->coop_wait = 60.0;
    s->step_frac = 0.99; s->feas_tol = 1e-8; s->gap_tol = 1e-8; s->near_factor = 1000.0; s->stall_tol = 1e-3;
    s->refine_stall_tol = 0.5; s->aug_tol = 1e-7; s->infeas_abs = 1e-8; s->infeas_rel = 1e-8;
}

int mb_ctx_create(int32_t device, mb_ctx** out) {
    if (!out) return MB_E_ARG;
    auto c = std::make_unique<mb_ctx>();
    c->device = device;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || device < 0 || device >= ndev) return MB_E_CUDA;
    if (cudaSetDevice(device) != cudaSuccess) return MB_E_CUDA;
    cudaDeviceProp prop;
    if (cudaGetDeviceProperties(&prop, device) != cudaSuccess) return MB_E_CUDA;
    c->nsm = prop.multiProcessorCount;
    if (cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking) != cudaSuccess) return MB_E_CUDA;
    *out = c.release();
    return MB_OK;
}

int mb_ctx_destroy(mb_ctx* ctx) {
    if (!ctx) return MB_E_ARG;
    cudaSetDevice(ctx->device);
    cudaDeviceSynchronize();
    cache_clear(ctx->dev, true);
    cache_clear(ctx->host, false);
    if (ctx->stream) cudaStreamDestroy(ctx->stream);
    delete ctx;
    return MB_OK;
}

int mb_last_error(mb_ctx* ctx, char* buf, int64_t size) {
    if (!ctx || !buf || size <= 0) return MB_E_ARG;
    std::snprintf(buf, (size_t)size, "%s", ctx->err.c_str());
    return MB_OK;
}

static int read_bsm(mb_ctx* ctx, const mb_bsm* A, mbh::BSM& R, const char* name) {
    if (!A || A->nout < 0 || A->nvtx < 0 || A->narc < 0 || A->ncol < 0 || A->nrow < 0 || A->nbnz < 0)
        return fail(ctx, MB_E_ARG, std::string(name) + ": bad sizes");
    if (!A->xsrc || !A->xcol || !A->xrow || !A->xblk || (A->narc && !A->tgt) || (A->nbnz && !A->val))
        return fail(ctx, MB_E_ARG, std::string(name) + ": null array");
    R.nout = A->nout; R.nvtx = A->nvtx; R.narc = A->narc; R.ncol = A->ncol; R.nrow = A->nrow; R.nbnz = A->nbnz;
    R.xsrc.resize(R.nvtx + 1); R.xcol.resize(R.nvtx + 1); R.xrow.resize(R.nout + 1); R.xblk.resize(R.narc + 1);
    R.tgt.resize(R.narc); R.val.assign(A->val, A->val + R.nbnz);
    for (i64 i = 0; i <= R.nvtx; ++i) { R.xsrc[i] = A->xsrc[i] - 1; R.xcol[i] = A->xcol[i] - 1; }
    for (i64 i = 0; i <= R.nout; ++i) R.xrow[i] = A->xrow[i] - 1;
    for (i64 i = 0; i <= R.narc; ++i) R.xblk[i] = A->xblk[i] - 1;
    for (i64 i = 0; i < R.narc; ++i) R.tgt[i] = A->tgt[i] - 1;
    // validate (block_sparse_matrix.jl:658-716)
    if (R.xsrc[0] != 0 || R.xcol[0] != 0 || R.xrow[0] != 0 || R.xblk[0] != 0 || R.xsrc[R.nvtx] != R.narc ||
        R.xcol[R.nvtx] != R.ncol || R.xrow[R.nout] != R.nrow || R.xblk[R.narc] != R.nbnz)
        return fail(ctx, MB_E_ARG, std::string(name) + ": inconsistent index arrays");
    for (i64 v = 0; v < R.nvtx; ++v) {
        if (R.xsrc[v] > R.xsrc[v + 1] || R.xcol[v] > R.xcol[v + 1]) return fail(ctx, MB_E_ARG, std::string(name) + ": xsrc/xcol not monotone");
        i64 prev = -1;
        for (i64 e = R.xsrc[v]; e < R.xsrc[v + 1]; ++e) {
            i64 u = R.tgt[e];
            if (!(prev < u && u < R.nout)) return fail(ctx, MB_E_ARG, std::string(name) + ": arcs not sorted or target out of range");
            prev = u;
            if (R.xblk[e + 1] - R.xblk[e] != R.nrows(u) * R.ncols(v)) return fail(ctx, MB_E_ARG, std::string(name) + ": block size mismatch");
        }
    }
    for (i64 u = 0; u < R.nout; ++u) if (R.xrow[u] > R.xrow[u + 1]) return fail(ctx, MB_E_ARG, std::string(name) + ": xrow not monotone");
    return MB_OK;
}

// ---- compensated products: extmul! / twomul! (BlockSparseArrays/src/comp/comp.jl:280-311) ------
// A BlockSparseMatrix resident on the device as two scalar views of ALL its stored block entries
// (explicit zeros too, as the reference's block loops visit them): the CSR with each row's
// columns ascending (the order twogemv_impl! adds into an entry of A b) and the CSC with each
// column's rows ascending plus block marks (the order, and the register pairs, of Aᵀ b).
struct mb_matrix {
    mb_ctx* ctx = nullptr;
    i64 nrow = 0, ncol = 0, nnz = 0;
    int64_t* rptr = nullptr; int32_t* cidx = nullptr; double* rval = nullptr;
    int64_t* cptr = nullptr; int32_t* ridx = nullptr; double* cval = nullptr; unsigned char* brk = nullptr;
    double* vec = nullptr;   // b | c | cc | s | cs, max(nrow, ncol) each
    ~mb_matrix() {
        for (void* p : {(void*)rptr, (void*)cidx, (void*)rval, (void*)cptr, (void*)ridx, (void*)cval, (void*)brk, (void*)vec})
            if (p) cudaFree(p);
    }
};

int mb_matrix_create(mb_ctx* ctx, const mb_bsm* A, mb_matrix** out) {
    if (!ctx || !A || !out) return fail(ctx, MB_E_ARG, "bad arguments");
    mbh::BSM R;
    if (int rc = read_bsm(ctx, A, R, "A")) return rc;
    if (R.nbnz > INT64_C(0x7fffffff) || R.nrow > INT64_C(0x7fffffff) || R.ncol > INT64_C(0x7fffffff))
        return fail(ctx, MB_E_ARG, "A: more than 2^31 - 1 rows, columns or stored entries");
    const i64 nr = R.nrow, nc = R.ncol, nz = R.nbnz;
    std::vector<int64_t> rptr(nr + 1, 0), cptr(nc + 1, 0);
    for (i64 v = 0; v < R.nvtx; ++v)
        for (i64 e = R.xsrc[v]; e < R.xsrc[v + 1]; ++e) {
            const i64 u = R.tgt[e];
            for (i64 i = R.xrow[u]; i < R.xrow[u + 1]; ++i) rptr[i + 1] += R.ncols(v);
            for (i64 j = R.xcol[v]; j < R.xcol[v + 1]; ++j) cptr[j + 1] += R.nrows(u);
        }
    for (i64 i = 0; i < nr; ++i) rptr[i + 1] += rptr[i];
    for (i64 j = 0; j < nc; ++j) cptr[j + 1] += cptr[j];
    std::vector<int32_t> cidx(nz), ridx(nz);
    std::vector<double> rval(nz), cval(nz);
    std::vector<unsigned char> brk(nz, 0);
    std::vector<int64_t> rpos(rptr.begin(), rptr.end() - 1), cpos(cptr.begin(), cptr.end() - 1);
    // vertices, arcs and columns ascending: each row receives its entries in ascending column order,
    // each column its blocks in ascending target order
    for (i64 v = 0; v < R.nvtx; ++v)
        for (i64 e = R.xsrc[v]; e < R.xsrc[v + 1]; ++e) {
            const i64 u = R.tgt[e], r0 = R.xrow[u], nru = R.nrows(u), ncv = R.ncols(v);
            const double* blk = R.val.data() + R.xblk[e];
            for (i64 jl = 0; jl < ncv; ++jl) {
                const i64 j = R.xcol[v] + jl;
                for (i64 il = 0; il < nru; ++il) {
                    const double a = blk[il + jl * nru];
                    const i64 q = rpos[r0 + il]++;
                    cidx[q] = (int32_t)j; rval[q] = a;
                    const i64 t = cpos[j]++;
                    ridx[t] = (int32_t)(r0 + il); cval[t] = a;
                    if (il == 0) brk[t] = (nru == 1 && ncv == 1) ? 2 : 1;
                }
            }
        }
    auto m = std::make_unique<mb_matrix>();
    m->ctx = ctx; m->nrow = nr; m->ncol = nc; m->nnz = nz;
    CUDA_TRY(ctx, cudaSetDevice(ctx->device));
    auto up = [&](auto*& d, const auto& h) -> cudaError_t {
        const size_t bytes = std::max<size_t>(h.size(), 1) * sizeof(h[0]);
        cudaError_t e = cudaMalloc((void**)&d, bytes);
        if (e == cudaSuccess && !h.empty()) e = cudaMemcpyAsync(d, h.data(), h.size() * sizeof(h[0]), cudaMemcpyHostToDevice, ctx->stream);
        return e;
    };
    CUDA_TRY(ctx, up(m->rptr, rptr)); CUDA_TRY(ctx, up(m->cidx, cidx)); CUDA_TRY(ctx, up(m->rval, rval));
    CUDA_TRY(ctx, up(m->cptr, cptr)); CUDA_TRY(ctx, up(m->ridx, ridx)); CUDA_TRY(ctx, up(m->cval, cval));
    CUDA_TRY(ctx, up(m->brk, brk));
    CUDA_TRY(ctx, cudaMalloc((void**)&m->vec, 5 * (size_t)std::max<i64>(std::max(nr, nc), 1) * sizeof(double)));
    CUDA_TRY(ctx, cudaStreamSynchronize(ctx->stream));
    *out = m.release();
    return MB_OK;
}

int mb_matrix_destroy(mb_matrix* A) {
    if (!A) return MB_E_ARG;
    cudaSetDevice(A->ctx->device);
    delete A;
    return MB_OK;
}

// c ← α op(A) b + β c through host buffers: b and (β ≠ 0) c in, c (and cc, s, cs) out
static int twomv(mb_matrix* A, int32_t trans, const double* b, double alpha, double beta, double* c, double* cc,
                 double* s, double* cs) {
    if (!A) return MB_E_ARG;
    mb_ctx* ctx = A->ctx;
    const i64 nin = trans ? A->nrow : A->ncol, nout = trans ? A->ncol : A->nrow;
    if ((nin > 0 && !b) || (nout > 0 && !c) || (s == nullptr) != (cs == nullptr))
        return fail(ctx, MB_E_ARG, "null vector (b and c are required; s and cs go together)");
    CUDA_TRY(ctx, cudaSetDevice(ctx->device));
    const size_t w = (size_t)std::max<i64>(std::max(A->nrow, A->ncol), 1);
    double* db = A->vec; double* dc = db + w; double* dcc = dc + w; double* ds = dcc + w; double* dcs = ds + w;
    cudaStream_t st = ctx->stream;
    if (nin > 0) CUDA_TRY(ctx, cudaMemcpyAsync(db, b, nin * sizeof(double), cudaMemcpyHostToDevice, st));
    if (beta != 0.0 && nout > 0) CUDA_TRY(ctx, cudaMemcpyAsync(dc, c, nout * sizeof(double), cudaMemcpyHostToDevice, st));
    mb::TwoMv a{};
    a.nout = nout; a.trans = trans ? 1 : 0;
    a.acls = alpha == 1.0 ? 1 : (alpha == -1.0 ? 2 : 0);
    a.bcls = beta == 0.0 ? 0 : (beta == 1.0 ? 1 : (beta == -1.0 ? 2 : 3));
    a.ptr = trans ? A->cptr : A->rptr; a.idx = trans ? A->ridx : A->cidx; a.val = trans ? A->cval : A->rval;
    a.brk = A->brk; a.b = db; a.alpha = alpha; a.beta = beta;
    a.c = dc; a.cc = cc ? dcc : nullptr; a.s = s ? ds : nullptr; a.cs = s ? dcs : nullptr;
    CUDA_TRY(ctx, (cudaError_t)mb_launch_twomv(&a, st));
    if (nout > 0) {
        CUDA_TRY(ctx, cudaMemcpyAsync(c, dc, nout * sizeof(double), cudaMemcpyDeviceToHost, st));
        if (cc) CUDA_TRY(ctx, cudaMemcpyAsync(cc, dcc, nout * sizeof(double), cudaMemcpyDeviceToHost, st));
        if (s) {
            CUDA_TRY(ctx, cudaMemcpyAsync(s, ds, nout * sizeof(double), cudaMemcpyDeviceToHost, st));
            CUDA_TRY(ctx, cudaMemcpyAsync(cs, dcs, nout * sizeof(double), cudaMemcpyDeviceToHost, st));
        }
    }
    CUDA_TRY(ctx, cudaStreamSynchronize(st));
    return MB_OK;
}

int mb_extmul(mb_matrix* A, int32_t trans, const double* b, double alpha, double beta, double* c, double* s,
              double* cs) {
    return twomv(A, trans, b, alpha, beta, c, nullptr, s, cs);
}

int mb_twomul(mb_matrix* A, int32_t trans, const double* b, double alpha, double beta, double* c, double* cc,
              double* s, double* cs) {
    if (!cc && A) return fail(A->ctx, MB_E_ARG, "cc is required");
    return twomv(A, trans, b, alpha, beta, c, cc, s, cs);
}

int mb_problem_create(mb_ctx* ctx, const mb_bsm* Q, const mb_bsm* B, const double* f, const double* g, double mu,
                      const int32_t* cone_kind, const double* cone_param, const int64_t* P1, const int64_t* P2,
                      mb_problem** out) {
    if (!out || !f || !g || !cone_kind) return fail(ctx, MB_E_ARG, "null argument");
    auto P = std::make_unique<mb_problem>();
    P->ctx = ctx;
    int rc;
    if ((rc = read_bsm(ctx, Q, P->Q, "Q"))) return rc;
    if ((rc = read_bsm(ctx, B, P->B, "B"))) return rc;
    // IPMProblem inner constructor asserts (problem.jl:32-38)
    if (P->Q.nvtx != P->B.nvtx || P->Q.nout != P->Q.nvtx || P->Q.ncol != P->B.ncol || P->Q.nrow != P->B.ncol)
        return fail(ctx, MB_E_ARG, "Q and B vertex/column layouts differ");
    for (i64 v = 0; v <= P->B.nvtx; ++v)
        if (P->Q.xcol[v] != P->B.xcol[v] || P->Q.xrow[v] != P->B.xcol[v]) return fail(ctx, MB_E_ARG, "ncols(B, v) != ncols(Q, v)");
    i64 n = P->B.ncol, m = P->B.nrow, nv = P->B.nvtx;
    P->f.assign(f, f + n); P->g.assign(g, g + m); P->mu = mu;
    P->kind.assign(cone_kind, cone_kind + nv);
    P->param.assign(nv, 0.0);
    if (cone_param) P->param.assign(cone_param, cone_param + nv);
    for (i64 v = 0; v < nv; ++v) if (P->kind[v] < 0 || P->kind[v] > 5) return fail(ctx, MB_E_ARG, "unknown cone kind");
    P->P1.resize(m); P->P2.resize(n);
    std::vector<char> seen;
    seen.assign(m, 0);
    for (i64 i = 0; i < m; ++i) {
        i64 t = P1 ? P1[i] - 1 : i;
        if (t < 0 || t >= m || seen[t]) return fail(ctx, MB_E_ARG, "P1 is not a permutation");
        seen[t] = 1; P->P1[i] = t;
    }
    seen.assign(n, 0);
    for (i64 i = 0; i < n; ++i) {
        i64 t = P2 ? P2[i] - 1 : i;
        if (t < 0 || t >= n || seen[t]) return fail(ctx, MB_E_ARG, "P2 is not a permutation");
        seen[t] = 1; P->P2[i] = t;
    }
    *out = P.release();
    return MB_OK;
}

static int read_csc(mb_ctx* ctx, const mb_csc* A, mbh::CSC& R, const char* name) {
    if (!A || A->m < 0 || A->n < 0 || !A->colptr) return fail(ctx, MB_E_ARG, std::string(name) + ": bad CSC");
    i64 nnz = A->colptr[A->n] - 1;
    if (nnz < 0 || (nnz && (!A->rowval || !A->nzval))) return fail(ctx, MB_E_ARG, std::string(name) + ": bad CSC arrays");
    R.m = A->m; R.n = A->n;
    R.colptr.resize(A->n + 1);
    for (i64 j = 0; j <= A->n; ++j) R.colptr[j] = A->colptr[j] - 1;
    R.rowval.resize(nnz); R.nzval.assign(A->nzval, A->nzval + nnz);
    for (i64 p = 0; p < nnz; ++p) {
        R.rowval[p] = A->rowval[p] - 1;
        if (R.rowval[p] < 0 || R.rowval[p] >= R.m) return fail(ctx, MB_E_ARG, std::string(name) + ": row index out of range");
    }
    for (i64 j = 0; j < A->n; ++j) if (R.colptr[j] > R.colptr[j + 1]) return fail(ctx, MB_E_ARG, std::string(name) + ": colptr not monotone");
    mbh::sort_csc(R);
    return MB_OK;
}

// IPMProblem(Q::SparseMatrixCSC, B::SparseMatrixCSC, f, g, μ, K, s; compress)  (problem.jl:84-127)
int mb_problem_create_csc(mb_ctx* ctx, const mb_csc* Qc, const mb_csc* Bc, const double* f, const double* g,
                          double mu, int64_t ncone, const int32_t* cone_kind, const int64_t* cone_size,
                          const double* cone_param, double compress, mb_problem** out) {
    if (!out || !f || !g || !cone_kind || !cone_size || ncone < 0) return fail(ctx, MB_E_ARG, "null argument");
    mbh::CSC Q, B;
    int rc;
    if ((rc = read_csc(ctx, Qc, Q, "Q"))) return rc;
    if ((rc = read_csc(ctx, Bc, B, "B"))) return rc;
    i64 m = B.m, n = B.n;
    i64 tot = 0;
    for (i64 k = 0; k < ncone; ++k) { if (cone_size[k] < 0) return fail(ctx, MB_E_ARG, "negative cone size"); tot += cone_size[k]; }
    if (Q.m != n || Q.n != n || tot != n) return fail(ctx, MB_E_ARG, "shape mismatch (problem.jl:102-108)");
    if (!(compress > 0 && compress <= 1)) return fail(ctx, MB_E_ARG, "compress must lie in (0, 1]");
    for (i64 k = 0; k < ncone; ++k) if (cone_kind[k] < 0 || cone_kind[k] > 5) return fail(ctx, MB_E_ARG, "unknown cone kind");
    Q = mbh::dropoffdz(Q);
    B = mbh::dropzeros(B);
    // colpartition (problem.jl:262-349)
    i64 ncolP = 0, ncolC = 0, nvR = 0;
    for (i64 k = 0; k < ncone; ++k) {
        if (cone_kind[k] == MB_CONE_POS) ncolP += cone_size[k];
        else if (cone_kind[k] == MB_CONE_FREE) ncolC += cone_size[k];
        else nvR++;
    }
    std::vector<i64> work(n);
    {
        i64 p = 0, c = 0, r = 0, j = 0;
        for (i64 k = 0; k < ncone; ++k)
            for (i64 t = 0; t < cone_size[k]; ++t, ++j) {
                if (cone_kind[k] == MB_CONE_POS) work[p++] = j;
                else if (cone_kind[k] == MB_CONE_FREE) work[ncolP + c++] = j;
                else work[ncolP + ncolC + r++] = j;
            }
    }
    // pattern of [Q; B] restricted to a column group, transposed: rows = the group's columns
    auto group_twins = [&](i64 off, i64 cnt, std::vector<i64>& xptr, std::vector<i64>& perm) -> i64 {
        mbh::CSC T;  // (cnt) x (n + m), column r lists the group columns with an entry in row r
        T.m = cnt; T.n = n + m;
        std::vector<std::vector<i64>> buckets(n + m);
        for (i64 t = 0; t < cnt; ++t) {
            i64 j = work[off + t];
            for (i64 p = Q.colptr[j]; p < Q.colptr[j + 1]; ++p) buckets[Q.rowval[p]].push_back(t);
            for (i64 p = B.colptr[j]; p < B.colptr[j + 1]; ++p) buckets[n + B.rowval[p]].push_back(t);
        }
        T.colptr.assign(n + m + 1, 0);
        for (i64 r = 0; r < n + m; ++r) { T.colptr[r + 1] = T.colptr[r] + (i64)buckets[r].size(); T.rowval.insert(T.rowval.end(), buckets[r].begin(), buckets[r].end()); }
        T.nzval.assign(T.rowval.size(), 1.0);
        return mbh::twins_rows(T, compress, xptr, perm);
    };
    std::vector<i64> xcP, pmP, xcC, pmC;
    i64 nvP = group_twins(0, ncolP, xcP, pmP);
    i64 nvC = group_twins(ncolP, ncolC, xcC, pmC);
    i64 nvtx = nvP + nvC + nvR;
    std::vector<i64> colperm(n), xcol(nvtx + 1);
    std::vector<int32_t> kind(nvtx);
    std::vector<double> param(nvtx, 0.0);
    for (i64 j = 0; j < ncolP; ++j) colperm[j] = work[pmP[j] - 1];
    for (i64 v = 0; v < nvP; ++v) { xcol[v] = xcP[v] - 1; kind[v] = MB_CONE_POS; }
    for (i64 j = 0; j < ncolC; ++j) colperm[ncolP + j] = work[ncolP + pmC[j] - 1];
    for (i64 v = 0; v < nvC; ++v) { xcol[nvP + v] = ncolP + xcC[v] - 1; kind[nvP + v] = MB_CONE_FREE; }
    for (i64 j = ncolP + ncolC; j < n; ++j) colperm[j] = work[j];
    {
        i64 r = 0, j = 0;
        for (i64 k = 0; k < ncone; ++k)
            if (cone_kind[k] != MB_CONE_POS && cone_kind[k] != MB_CONE_FREE) {
                xcol[nvP + nvC + r] = ncolP + ncolC + j;
                kind[nvP + nvC + r] = cone_kind[k];
                param[nvP + nvC + r] = cone_param ? cone_param[k] : 0.0;
                r++; j += cone_size[k];
            }
    }
    xcol[nvtx] = n;
    // colcompress (problem.jl:188-260): vertex pattern of B
    mbh::CSC Bc2; Bc2.m = m; Bc2.n = nvtx; Bc2.colptr.assign(nvtx + 1, 0);
    {
        std::vector<i64> mark(m, -1), rows;
        for (i64 v = 0; v < nvtx; ++v) {
            rows.clear();
            for (i64 j = xcol[v]; j < xcol[v + 1]; ++j) {
                i64 k = colperm[j];
                for (i64 p = B.colptr[k]; p < B.colptr[k + 1]; ++p) if (mark[B.rowval[p]] != v) { mark[B.rowval[p]] = v; rows.push_back(B.rowval[p]); }
            }
            std::sort(rows.begin(), rows.end());
            Bc2.rowval.insert(Bc2.rowval.end(), rows.begin(), rows.end());
            Bc2.colptr[v + 1] = (i64)Bc2.rowval.size();
        }
        Bc2.nzval.assign(Bc2.rowval.size(), 1.0);
    }
    std::vector<i64> xrow1, rowperm1;
    i64 nout = mbh::twins_rows(Bc2, compress, xrow1, rowperm1);
    std::vector<i64> rowperm(m), xrow(nout + 1);
    for (i64 i = 0; i < m; ++i) rowperm[i] = rowperm1[i] - 1;
    for (i64 u = 0; u <= nout; ++u) xrow[u] = xrow1[u] - 1;
    mbh::CSC Bp = mbh::permute(B, rowperm, colperm);
    mbh::CSC Qp = mbh::permute(Q, colperm, colperm);
    auto P = std::make_unique<mb_problem>();
    P->ctx = ctx;
    P->B = mbh::compress2(Bp, nvtx, nout, xcol, xrow);
    P->Q = mbh::compress2(Qp, nvtx, nvtx, xcol, xcol);
    P->f.resize(n); P->g.resize(m);
    for (i64 j = 0; j < n; ++j) P->f[j] = f[colperm[j]];
    for (i64 i = 0; i < m; ++i) P->g[i] = g[rowperm[i]];
    P->mu = mu; P->kind = kind; P->param = param;
    P->P1 = rowperm; P->P2 = colperm;
    *out = P.release();
    return MB_OK;
}

int mb_problem_info(const mb_problem* P, int64_t* info8) {
    if (!P || !info8) return MB_E_ARG;
    info8[0] = P->B.ncol; info8[1] = P->B.nrow; info8[2] = P->B.nvtx; info8[3] = P->B.nout;
    info8[4] = P->B.narc; info8[5] = P->B.nbnz; info8[6] = P->Q.narc; info8[7] = P->Q.nbnz;
    return MB_OK;
}

int mb_problem_export(const mb_problem* P, int64_t* Bxsrc, int64_t* Bxcol, int64_t* Bxrow, int64_t* Bxblk,
                      int64_t* Btgt, double* Bval, int64_t* Qxsrc, int64_t* Qxblk, int64_t* Qtgt, double* Qval,
                      double* f, double* g, int32_t* kind, double* param, int64_t* P1, int64_t* P2) {
    if (!P) return MB_E_ARG;
    auto cp1 = [](int64_t* dst, const std::vector<i64>& src) { if (dst) for (size_t i = 0; i < src.size(); ++i) dst[i] = src[i] + 1; };
    auto cpd = [](double* dst, const std::vector<double>& src) { if (dst) std::memcpy(dst, src.data(), src.size() * sizeof(double)); };
    cp1(Bxsrc, P->B.xsrc); cp1(Bxcol, P->B.xcol); cp1(Bxrow, P->B.xrow); cp1(Bxblk, P->B.xblk); cp1(Btgt, P->B.tgt);
    cpd(Bval, P->B.val);
    cp1(Qxsrc, P->Q.xsrc); cp1(Qxblk, P->Q.xblk); cp1(Qtgt, P->Q.tgt); cpd(Qval, P->Q.val);
    cpd(f, P->f); cpd(g, P->g); cpd(param, P->param);
    if (kind) std::memcpy(kind, P->kind.data(), P->kind.size() * sizeof(int32_t));
    cp1(P1, P->P1); cp1(P2, P->P2);
    return MB_OK;
}

int mb_problem_destroy(mb_problem* P) {
    if (!P) return MB_E_ARG;
    delete P;
    return MB_OK;
}

int mb_problem_symbolic(const mb_problem* Pc, int64_t* vperm, int64_t* nfront, int64_t* res0, int64_t* nres,
                        int64_t* nsep, int64_t* parent, int64_t cap) {
    if (!Pc) return MB_E_ARG;
    Sym S = do_symbolic(Pc);
    if (vperm) for (size_t k = 0; k < S.vperm.size(); ++k) vperm[k] = S.vperm[k];
    if (nfront) *nfront = S.fr.nfront;
    for (i64 f = 0; f < S.fr.nfront && f < cap; ++f) {
        if (res0) res0[f] = S.fr.res0[f];
        if (nres) nres[f] = S.fr.nres[f];
        if (nsep) nsep[f] = (i64)S.fr.sep[f].size();
        if (parent) parent[f] = S.fr.parent[f];
    }
    return MB_OK;
}

int mb_problem_footprint(mb_problem* prob, const mb_settings* settings, int64_t* bytes) {
    if (!prob || !bytes) return MB_E_ARG;
    mb_settings s;
    if (settings) s = *settings; else mb_settings_default(&s);
    Packed pk;
    std::string err;
    int rc = plan_instance(prob, s, nullptr, nullptr, nullptr, pk, err);
    if (rc) return fail(prob->ctx, rc, err);
    *bytes = (int64_t)pk.device_bytes();
    return MB_OK;
}

int mb_solver_create(mb_problem* prob, const mb_settings* settings, const double* p0, const double* d0,
                     const double* y0, mb_solver** out) {
    if (!prob || !out || !prob->ctx) return MB_E_ARG;
    mb_batch* b = nullptr;
    mb_problem* arr[1] = {prob};
    int rc = make_batch(prob->ctx, arr, 1, settings, p0, d0, y0, &b);
    if (rc) return rc;
    auto s = std::make_unique<mb_solver>();
    s->prob = prob;
    s->b.reset(b);
    rc = run_batch(b, mb::MODE_INIT, 1, nullptr);
    if (rc) return rc;
    *out = s.release();
    return MB_OK;
}

int mb_solver_step(mb_solver* s, int32_t* status) {
    if (!s) return MB_E_ARG;
    if (s->done) return fail(s->prob->ctx, MB_E_STATE, "solver already finished");
    int rc = run_batch(s->b.get(), mb::MODE_STEP, 1, nullptr);
    if (rc) return rc;
    int32_t st = 0;
    CUDA_TRY(s->prob->ctx, cudaMemcpy(&st, s->b->d_ost + s->b->pk.plans[0].status, sizeof(int32_t), cudaMemcpyDeviceToHost));
    s->status = st;
    if (st != MB_CONTINUE) s->done = true;
    if (status) *status = st;
    return MB_OK;
}

int mb_solver_solve(mb_solver* s, int32_t* status) {
    if (!s) return MB_E_ARG;
    int32_t st = s->status;
    while (!s->done) {
        int rc = mb_solver_step(s, &st);
        if (rc) return rc;
    }
    if (status) *status = s->status;
    return MB_OK;
}

int mb_solver_result(mb_solver* s, double* p, double* d, double* y, mb_result* res) {
    if (!s) return MB_E_ARG;
    int rc = run_batch(s->b.get(), mb::MODE_RESULT, 1, nullptr);
    if (rc) return rc;
    rc = fetch_batch(s->b.get());
    if (rc) return rc;
    unpack_one(s->b.get(), 0, p, d, y, res);
    return MB_OK;
}

// reinit!(s; p0, d0, y0, f, g) (solver/ipm.jl:371-429): the solver restarts from the cone identity
// (or the given p0/d0/y0, completed by shadows) with an empty history, optionally on a new f and/or
// g (user order, the problem's lengths); the equilibration, Q, B and BᵀB of init stay.
int mb_solver_reinit(mb_solver* s, const double* p0, const double* d0, const double* y0, const double* f,
                     const double* g) {
    if (!s) return MB_E_ARG;
    mb_batch* b = s->b.get();
    mb_ctx* ctx = b->ctx;
    InstPlan& ip = b->pk.plans[0];
    const i64 n = ip.n, m = ip.m;
    std::vector<double> v(std::max<i64>(std::max<i64>(n, m), 1));
    auto put = [&](size_t off, const double* src, i64 len, const std::vector<i64>& map) -> int {
        for (i64 i = 0; i < len; ++i) v[i] = src ? src[map[i]] : 0.0;
        if (len) CUDA_TRY(ctx, cudaMemcpy(b->d_din + off, v.data(), len * sizeof(double), cudaMemcpyHostToDevice));
        return MB_OK;
    };
    int rc;
    if (f && (rc = put(ip.f, f, n, ip.colmap))) return rc;
    if (g && (rc = put(ip.g, g, m, ip.rowmap))) return rc;
    if ((rc = put(ip.p, p0, n, ip.colmap)) || (rc = put(ip.d, d0, n, ip.colmap)) || (rc = put(ip.y, y0, m, ip.rowmap)))
        return rc;
    ip.has_p0 = p0 != nullptr; ip.has_d0 = d0 != nullptr; ip.has_y0 = y0 != nullptr;
    mb::DevInst I = static_devinst(ip, b->d_i32, b->d_i64, b->d_din, b->d_work, b->d_out, b->d_ost, (char*)b->d_F);
    I.reinit_fg = (f ? 1 : 0) | (g ? 2 : 0);
    I.sx = s->d_sx;
    CUDA_TRY(ctx, cudaMemcpy(b->d_inst, &I, sizeof(I), cudaMemcpyHostToDevice));
    rc = run_batch(b, mb::MODE_REINIT, 1, nullptr);
    if (rc) return rc;
    s->done = false;
    s->status = MB_CONTINUE;
    return MB_OK;
}

// frule! / rrule! (ipm/differential.jl): seeds (user order, NULL = 0) into the exchange buffer in
// solver order, one MODE_FRULE / MODE_RRULE launch, results back in user order
static int sens_run(mb_solver* s, int mode, const double* a, const double* bv, const double* c, double dmu,
                    double* oa, double* ob, double* oc, double* dmu_out) {
    mb_batch* b = s->b.get();
    mb_ctx* ctx = b->ctx;
    InstPlan& ip = b->pk.plans[0];
    const i64 n = ip.n, m = ip.m;
    const size_t len = (size_t)(4 * n + 2 * m + 3);
    if (!s->d_sx) {   // room for frule2!'s exchange too (8n + 5m + 3)
        CUDA_TRY(ctx, cache_alloc(ctx, ctx->dev, true, (void**)&s->d_sx, (size_t)(8 * n + 5 * m + 3) * sizeof(double)));
        mb::DevInst I = static_devinst(ip, b->d_i32, b->d_i64, b->d_din, b->d_work, b->d_out, b->d_ost, (char*)b->d_F);
        I.sx = s->d_sx;
        CUDA_TRY(ctx, cudaMemcpy(b->d_inst, &I, sizeof(I), cudaMemcpyHostToDevice));
    }
    if (mode < 0) return MB_OK;   // bind the buffer only
    std::vector<double> h(len, 0.0);
    for (i64 i = 0; i < n; ++i) {
        if (a) h[i] = a[ip.colmap[i]];
        if (c) h[n + m + i] = c[ip.colmap[i]];
    }
    if (bv) for (i64 i = 0; i < m; ++i) h[n + i] = bv[ip.rowmap[i]];
    h[4 * n + 2 * m] = dmu;
    CUDA_TRY(ctx, cudaMemcpy(s->d_sx, h.data(), len * sizeof(double), cudaMemcpyHostToDevice));
    int rc = run_batch(b, mode, 1, nullptr);
    if (rc) return rc;
    CUDA_TRY(ctx, cudaMemcpy(h.data(), s->d_sx, len * sizeof(double), cudaMemcpyDeviceToHost));
    if (h[4 * n + 2 * m + 2] != 1.0) return fail(ctx, MB_E_STATE, "the KKT factorization at the current iterate failed");
    const double* r = h.data() + 2 * n + m;
    for (i64 i = 0; i < n; ++i) {
        if (oa) oa[ip.colmap[i]] = r[i];
        if (oc) oc[ip.colmap[i]] = r[n + m + i];
    }
    if (ob) for (i64 i = 0; i < m; ++i) ob[ip.rowmap[i]] = r[n + i];
    if (dmu_out) *dmu_out = h[4 * n + 2 * m + 1];
    return MB_OK;
}

// frule2! (ipm/differential.jl:82-260): seeds f1 g1 f2 g2 at sx[0 .. 2n+2m), nine results after them,
// then [Δμ1, Δμ2, ok]
int mb_solver_frule2(mb_solver* s, const double* df1, const double* dg1, double dmu1, const double* df2,
                     const double* dg2, double dmu2, double* const* out) {
    if (!s) return MB_E_ARG;
    if (!s->d_sx) {   // allocate and bind the exchange buffer through a first-order call's path
        int rc = sens_run(s, -1, nullptr, nullptr, nullptr, 0.0, nullptr, nullptr, nullptr, nullptr);
        if (rc) return rc;
    }
    mb_batch* b = s->b.get();
    mb_ctx* ctx = b->ctx;
    InstPlan& ip = b->pk.plans[0];
    const i64 n = ip.n, m = ip.m;
    const size_t len = (size_t)(8 * n + 5 * m + 3);
    std::vector<double> h(len, 0.0);
    const double* fs[2] = {df1, df2};
    const double* gs[2] = {dg1, dg2};
    for (int k = 0; k < 2; ++k) {
        double* f = h.data() + (size_t)k * (n + m);
        double* g = f + n;
        if (fs[k]) for (i64 i = 0; i < n; ++i) f[i] = fs[k][ip.colmap[i]];
        if (gs[k]) for (i64 i = 0; i < m; ++i) g[i] = gs[k][ip.rowmap[i]];
    }
    double* ss = h.data() + len - 3;
    ss[0] = dmu1; ss[1] = dmu2;
    CUDA_TRY(ctx, cudaMemcpy(s->d_sx, h.data(), len * sizeof(double), cudaMemcpyHostToDevice));
    int rc = run_batch(b, mb::MODE_FRULE2, 1, nullptr);
    if (rc) return rc;
    CUDA_TRY(ctx, cudaMemcpy(h.data(), s->d_sx, len * sizeof(double), cudaMemcpyDeviceToHost));
    if (ss[2] != 1.0) return fail(ctx, MB_E_STATE, "the KKT factorization at the current iterate failed");
    const double* r = h.data() + 2 * (n + m);
    for (int k = 0; k < 9; ++k) {
        const bool row = k % 3 == 1;
        const i64 len_k = row ? m : n;
        if (out && out[k]) {
            if (row) for (i64 i = 0; i < m; ++i) out[k][ip.rowmap[i]] = r[i];
            else for (i64 i = 0; i < n; ++i) out[k][ip.colmap[i]] = r[i];
        }
        r += len_k;
    }
    return MB_OK;
}

int mb_solver_frule(mb_solver* s, const double* df, const double* dg, double dmu, double* dp, double* dy, double* dd) {
    if (!s) return MB_E_ARG;
    return sens_run(s, mb::MODE_FRULE, df, dg, nullptr, dmu, dp, dy, dd, nullptr);
}

int mb_solver_rrule(mb_solver* s, const double* dp, const double* dy, const double* dd, double* df, double* dg,
                    double* dmu) {
    if (!s) return MB_E_ARG;
    return sens_run(s, mb::MODE_RRULE, dp, dy, dd, 0.0, df, dg, nullptr, dmu);
}

// print_timers / the solver's TimerOutput: MB_NSECTIONS section clocks (SM cycles), then the numbers
// of triangular-solve sweeps and matvecs, as mb_batch_timers reports them for one instance
int mb_solver_timers(mb_solver* s, double* out, int64_t cap) {
    if (!s || !out) return MB_E_ARG;
    int rc = fetch_batch(s->b.get());
    if (rc) return rc;
    return mb_batch_timers(s->b.get(), out, cap);
}

int mb_solver_history(mb_solver* s, mb_history_row* rows, int32_t cap, int32_t* nrows) {
    if (!s) return MB_E_ARG;
    int rc = fetch_batch(s->b.get());
    if (rc) return rc;
    const InstPlan& ip = s->b->pk.plans[0];
    int32_t nr = std::min<int32_t>(s->b->h_i32[ip.status + 1], s->b->set.max_iter + 1);
    if (nrows) *nrows = nr;
    if (rows) for (int32_t i = 0; i < nr && i < cap; ++i)
        std::memcpy(&rows[i], s->b->h_out + ip.hist + (size_t)i * mb::ROW_DOUBLES, sizeof(mb_history_row));
    return MB_OK;
}

int mb_solver_destroy(mb_solver* s) {
    if (!s) return MB_E_ARG;
    delete s;
    return MB_OK;
}

int mb_batch_prepare(mb_ctx* ctx, mb_problem* const* probs, int32_t nprob, const mb_settings* settings, mb_batch** out) {
    return make_batch(ctx, probs, nprob, settings, nullptr, nullptr, nullptr, out);
}

int mb_batch_run(mb_batch* b, int32_t grid, float* ms) {
    if (!b) return MB_E_ARG;
    return run_batch(b, mb::MODE_SOLVE, grid, ms);
}

int mb_batch_fetch(mb_batch* b, double* const* p_out, double* const* d_out, double* const* y_out, mb_result* results) {
    if (!b) return MB_E_ARG;
    int rc = fetch_batch(b);
    if (rc) return rc;
    for (size_t k = 0; k < b->pk.plans.size(); ++k)
        unpack_one(b, k, p_out ? p_out[k] : nullptr, d_out ? d_out[k] : nullptr, y_out ? y_out[k] : nullptr,
                   results ? &results[k] : nullptr);
    return MB_OK;
}

int mb_batch_stats(mb_batch* b, int64_t* s) {
    if (!b || !s) return MB_E_ARG;
    s[0] = (int64_t)(b->pk.i32.size() * 4 + b->pk.i64a.size() * 8 + b->pk.din.size() * 8);
    s[1] = (int64_t)(b->pk.work.size() * 8);
    s[2] = (int64_t)b->pk.fbytes;
    s[3] = b->launches;
    s[4] = (int64_t)b->pk.plans.size();
    s[5] = (int64_t)(b->pk.out.size() * 8 + b->pk.ost.size() * 4);
    s[6] = 0; s[7] = 0;
    return MB_OK;
}

int mb_batch_timers(mb_batch* b, double* out, int64_t cap) {
    if (!b || !out) return MB_E_ARG;
    // per instance: NSEC section clocks, trsv sweeps, gemv calls (needs a prior mb_batch_fetch)
    static_assert(mb::NSEC == MB_NSECTIONS, "section count of the C header");
    const int W = mb::NSEC + 2;
    for (size_t k = 0; k < b->pk.plans.size() && (int64_t)((k + 1) * W) <= cap; ++k) {
        const double* sc = b->h_out + b->pk.plans[k].scal;
        for (int j = 0; j < mb::NSEC; ++j) out[k * W + j] = sc[mb::SCAL_SEC + j];
        out[k * W + mb::NSEC] = sc[mb::SCAL_NTRSV];
        out[k * W + mb::NSEC + 1] = sc[mb::SCAL_NGEMV];
    }
    return MB_OK;
}

int mb_batch_times(mb_batch* b, int64_t* out, int64_t cap) {
    if (!b || !out) return MB_E_ARG;
    for (size_t k = 0; k < b->pk.plans.size() && (int64_t)(2 * k + 2) <= cap; ++k) {
        const double* sc = b->h_out + b->pk.plans[k].scal;
        std::memcpy(&out[2 * k], &sc[mb::SCAL_T0], sizeof(int64_t));
        std::memcpy(&out[2 * k + 1], &sc[mb::SCAL_T1], sizeof(int64_t));
    }
    return MB_OK;
}

int mb_batch_destroy(mb_batch* b) {
    if (!b) return MB_E_ARG;
    delete b;
    return MB_OK;
}

// A large call is split into two or four chunks of decreasing estimated cost, each planned,
// uploaded and launched on its own stream: the host plans chunk c + 1 while the device runs chunk
// c, and the chunks' persistent grids fill each other's tails.  Nothing on a chunk's stream before
// its launch needs an SM (no memset kernels), so a running chunk never holds up the planning of the
// next.  Every instance is solved exactly as in a single launch.
int mb_batch_solve(mb_ctx* ctx, mb_problem* const* probs, int32_t nprob, const mb_settings* settings, int32_t grid,
                   double* const* p_out, double* const* d_out, double* const* y_out, mb_result* results) {
    const int nch = nprob >= 2048 ? 4 : (nprob >= 1024 ? 2 : 1);
    if (nch == 1 || grid > 0) {
        mb_batch* b = nullptr;
        int rc = make_batch(ctx, probs, nprob, settings, nullptr, nullptr, nullptr, &b);
        if (rc) return rc;
        std::unique_ptr<mb_batch> hold(b);
        rc = run_batch(b, mb::MODE_SOLVE, grid, nullptr);
        if (rc) return rc;
        return mb_batch_fetch(b, p_out, d_out, y_out, results);
    }
    if (!probs) return fail(ctx, MB_E_ARG, "bad arguments");
    std::vector<std::unique_ptr<mb_batch>> chunks(nch);
    // chunks in decreasing estimated cost (n³ of the problem's columns; only which chunk a problem
    // lands in depends on it): a small first chunk of the largest problems starts the device early,
    // the middle chunks carry the bulk while the host plans the next one, and a small last chunk of
    // the smallest problems fills the grid's tail and leaves little to read back at the end
    std::vector<int32_t> ord(nprob);
    for (int32_t k = 0; k < nprob; ++k) ord[k] = k;
    auto est = [&](int32_t k) { const double n = (double)probs[k]->B.ncol; return n * n * n; };
    std::stable_sort(ord.begin(), ord.end(), [&](int32_t a, int32_t b) { return est(a) > est(b); });
    std::vector<int32_t> cnt;
    if (nch == 2) cnt = {nprob / 8, nprob - nprob / 8};
    else {
        const int32_t c0 = nprob / 16, c3 = nprob / 8, c1 = (nprob - c0 - c3) / 2;
        cnt = {c0, c1, nprob - c0 - c3 - c1, c3};
    }
    std::vector<std::vector<int32_t>> idx(nch);
    for (int c = 0, k = 0; c < nch; ++c)
        for (int32_t j = 0; j < cnt[c]; ++j) idx[c].push_back(ord[k++]);
    const double t0 = host_time();
    for (int c = 0; c < nch; ++c) {
        std::vector<mb_problem*> sub(idx[c].size());
        for (size_t j = 0; j < sub.size(); ++j) sub[j] = probs[idx[c][j]];
        mb_batch* b = nullptr;
        int rc = make_batch(ctx, sub.data(), (int32_t)sub.size(), settings, nullptr, nullptr, nullptr, &b, true);
        if (rc) return rc;
        chunks[c].reset(b);
        if ((rc = run_batch(b, mb::MODE_SOLVE, 0, nullptr))) return rc;   // returns after the launch
        if (trace_on()) fprintf(stderr, "mb_batch_solve: chunk %d (%zu problems) launched at %.1f ms\n", c, sub.size(),
                                1e3 * (host_time() - t0));
    }
    for (int c = 0; c < nch; ++c) {
        const size_t nk = idx[c].size();
        std::vector<double*> pp(nk, nullptr), dd(nk, nullptr), yy(nk, nullptr);
        std::vector<mb_result> rr(results ? nk : 0);
        for (size_t j = 0; j < nk; ++j) {
            if (p_out) pp[j] = p_out[idx[c][j]];
            if (d_out) dd[j] = d_out[idx[c][j]];
            if (y_out) yy[j] = y_out[idx[c][j]];
        }
        int rc = mb_batch_fetch(chunks[c].get(), p_out ? pp.data() : nullptr, d_out ? dd.data() : nullptr,
                                y_out ? yy.data() : nullptr, results ? rr.data() : nullptr);
        if (rc) return rc;
        if (results) for (size_t j = 0; j < nk; ++j) results[idx[c][j]] = rr[j];
        if (trace_on()) {
            float a = 0, z = 0;
            cudaEventElapsedTime(&a, chunks[0]->e0, chunks[c]->e0);
            cudaEventElapsedTime(&z, chunks[0]->e0, chunks[c]->e1);
            fprintf(stderr, "mb_batch_solve: chunk %d fetched at %.1f ms; on the device from %.1f to %.1f ms after chunk 0's launch\n",
                    c, 1e3 * (host_time() - t0), a, z);
        }
    }
    return MB_OK;
}

}  // extern "C"

// ---------------------------------------------------------------------------------------------
// mb_batch_solve_static: the batched solve from the fixed device scratch of mb_solver.cu, for
// callers that may not allocate device memory during service (a process that reserved its HBM
// budget up front, or one whose other streams cannot absorb the device-wide synchronisation of
// cudaFree / a growing cudaMalloc).  No counterpart in the reference.  Same planning, DevInst
// layout and kernel as mb_batch_solve; only the placement of the device arrays differs, and no
// cudaMalloc, cudaMallocHost or cudaFree is called.  Calls that overlap on one device race on
// the scratch; the first call per device looks its address up and should precede stream capture.
// ---------------------------------------------------------------------------------------------
extern "C" int mb_static_scratch(int device, void** ptr, size_t* bytes);

namespace {

// byte offsets of the batch's arrays inside the scratch, each rounded up to 256 bytes
struct StaticLayout {
    size_t inst, counter, coop, ost, i32, i64a, din, work, out, F, total;
    StaticLayout(const Packed& pk) {
        size_t off = 0;
        auto region = [&](size_t bytes) { size_t o = off; off += (std::max<size_t>(bytes, 1) + 255) / 256 * 256; return o; };
        inst = region(pk.plans.size() * sizeof(mb::DevInst));
        counter = region(sizeof(int));
        coop = region(sizeof(mb::CoopCtl));
        ost = region(pk.ost.size() * sizeof(int32_t));
        i32 = region(pk.i32.size() * sizeof(int32_t));
        i64a = region(pk.i64a.size() * sizeof(i64));
        din = region(pk.din.size() * sizeof(double));
        work = region(pk.work.size() * sizeof(double));
        out = region(pk.out.size() * sizeof(double));
        F = region(pk.fbytes);
        total = off;
    }
};

// DevInst of plan p over arrays based at the given device pointers (the layout upload() builds)
mb::DevInst static_devinst(const InstPlan& p, int32_t* i32, i64* q64, double* dn, double* wk, double* ot,
                           int32_t* ost, char* F) {
    mb::DevInst I{};
    I.n = (int)p.n; I.m = (int)p.m; I.nvtx = (int)p.nvtx; I.nfront = (int)p.nfront; I.nu = (int)p.nu;
    I.has_p0 = p.has_p0; I.has_d0 = p.has_d0; I.has_y0 = p.has_y0; I.mut = p.mut;
    I.xcol = i32 + p.xcol; I.colvtx = i32 + p.colvtx; I.cfront = i32 + p.cfront;
    auto fillsp = [&](mb::DevSp& A, i64 nrow, i64 ncol, i64 nnz, size_t rptr, size_t cidx, size_t wval, size_t val0,
                      size_t cptr, size_t ridx, size_t cpos) {
        A.nrow = (int)nrow; A.ncol = (int)ncol; A.nnz = (int)nnz;
        A.rptr = i32 + rptr; A.cidx = i32 + cidx; A.val = wk + wval; A.val0 = dn + val0;
        A.cptr = i32 + cptr; A.ridx = i32 + ridx; A.cpos = i32 + cpos;
    };
    fillsp(I.B, p.m, p.n, p.Bnnz, p.Brptr, p.Bcidx, p.wBval, p.Bval, p.Bcptr, p.Bridx, p.Bcpos);
    fillsp(I.Q, p.n, p.n, p.Qnnz, p.Qrptr, p.Qcidx, p.wQval, p.Qval, p.Qcptr, p.Qridx, p.Qcpos);
    I.B.nlongr = (int)p.nBlongr; I.B.longr = i32 + p.Blongr; I.B.nlongc = (int)p.nBlongc; I.B.longc = i32 + p.Blongc;
    I.Q.nlongr = 0; I.Q.longr = nullptr; I.Q.nlongc = 0; I.Q.longc = nullptr;   // Q's rows go through hlong
    I.nhlong = (int)p.nhlong; I.hlong = i32 + p.hlong; I.hflag = i32 + p.hflag;
    I.hdoff = (const int64_t*)(q64 + p.hdoff); I.Qd = wk + p.wQd; I.Qd0 = dn + p.Qd; I.Hd = wk + p.Hd;
    I.qd0off = (const int64_t*)(q64 + p.qd0off);
    I.hdpos = (const int64_t*)(q64 + p.hdpos); I.hdld = i32 + p.hdld;
    I.nqoff = (int)p.nqoff; I.qoffk = i32 + p.qoffk; I.qoffpos = (const int64_t*)(q64 + p.qoffpos);
    I.kind = i32 + p.kind; I.kpar = dn + p.kpar; I.cxblk = (const int64_t*)(q64 + p.cxblk); I.cache = wk + p.cache;
    I.cache2 = wk + p.cache2;
    I.wsize = p.wsize;
    I.fres0 = i32 + p.fres0; I.fnres = i32 + p.fnres; I.fnsep = i32 + p.fnsep; I.fparent = i32 + p.fparent;
    I.fptr = (const int64_t*)(q64 + p.fptr); I.fsepp = i32 + p.fsepp; I.fsep = i32 + p.fsep; I.frel = i32 + p.frel;
    I.fsize = p.fsize;
    I.Finit = wk + p.Finit; I.F = F + p.F;
    I.sbrp = i32 + p.sbrp; I.sbrow = i32 + p.sbrow; I.sbloc = i32 + p.sbloc; I.fchp = i32 + p.fchp; I.fch = i32 + p.fch;
    I.swork = wk + p.swork;
    I.f0 = dn + p.f; I.g0 = dn + p.g; I.p0 = dn + p.p; I.d0 = dn + p.d; I.y0 = dn + p.y;
    I.f = wk + p.wf; I.g = wk + p.wg; I.pscl = wk + p.pscl; I.yscl = wk + p.yscl;
    I.p = wk + p.wp; I.d = wk + p.wd; I.y = wk + p.wy;
    I.vn = wk + p.vn; I.vm = wk + p.vm; I.vv = wk + p.vv; I.work = wk + p.work;
    I.po = ot + p.po; I.dout = ot + p.dout; I.yo = ot + p.yo;
    I.hist = ot + p.hist; I.uhist = wk + p.uhist; I.cghist = wk + p.cghist;
    I.status = ost + p.status; I.scal = ot + p.scal;
    return I;
}

// results of plan ip from host copies of the output and status arrays (what unpack_one reads)
void static_unpack(const InstPlan& ip, const double* o, const int32_t* st, int max_iter, double* p, double* d,
                   double* y, mb_result* r) {
    if (p) for (i64 i = 0; i < ip.n; ++i) p[ip.colmap[i]] = o[ip.po + i];
    if (d) for (i64 i = 0; i < ip.n; ++i) d[ip.colmap[i]] = o[ip.dout + i];
    if (y) for (i64 i = 0; i < ip.m; ++i) y[ip.rowmap[i]] = o[ip.yo + i];
    if (!r) return;
    st += ip.status;
    r->status = st[0]; r->niter = st[1]; r->nfactor_retry = st[2]; r->nfactor = st[3];
    r->nfp32 = st[4]; r->nfallback = st[5];
    r->factor_flops = ip.fflops;
    const double* sc = o + ip.scal;
    r->mu = sc[0]; r->pres = sc[1]; r->dres = sc[2]; r->pobj = sc[3]; r->dobj = sc[4];
    int ns = 0, nr = std::min<int>(st[1], max_iter + 1);
    for (int i = 0; i < nr; ++i) {
        const double* row = o + ip.hist + (size_t)i * mb::ROW_DOUBLES;
        ns += (int)(row[5] + row[6] + row[8] + row[9]);
    }
    r->nsolve = ns;
}

}  // namespace

extern "C" int mb_batch_solve_static(mb_ctx* ctx, mb_problem* const* probs, int32_t nprob, const mb_settings* settings,
                                     int32_t grid, double* const* p_out, double* const* d_out, double* const* y_out,
                                     mb_result* results) {
    if (!ctx || nprob < 0 || (nprob > 0 && !probs)) return fail(ctx, MB_E_ARG, "bad arguments");
    mb_settings s;
    if (settings) s = *settings; else mb_settings_default(&s);
    if (s.stable && s.precision != MB_PREC_FP64)
        return fail(ctx, MB_E_UNSUPPORTED, "stable=true (StableUzawaSolver) factors in FP64: precision must be 0");
    if (s.max_iter < 0 || s.refine_max_iter < 0 || s.newton_max_iter < 0) return fail(ctx, MB_E_ARG, "negative iteration limit");
    if (s.precision < 0 || s.precision > 2) return fail(ctx, MB_E_ARG, "precision must be 0 (FP64), 1 (FP32) or 2 (mixed)");
    for (int32_t k = 0; k < nprob; ++k) if (!probs[k]) return fail(ctx, MB_E_ARG, "null problem");
    if (nprob == 0) return MB_OK;
    // plan on the host, then check the fit before touching the device
    Packed pk;
    for (int32_t k = 0; k < nprob; ++k) {
        Packed one;
        std::string err;
        int rc = plan_instance(probs[k], s, nullptr, nullptr, nullptr, one, err);
        if (rc) return fail(ctx, rc, err);
        merge(pk, one);
    }
    const StaticLayout L(pk);
    if (L.total > (size_t)MB_STATIC_SCRATCH_BYTES)
        return fail(ctx, MB_E_NOMEM, "mb_batch_solve_static: the batch needs " + std::to_string(L.total) +
                                     " bytes of device scratch but the static scratch holds " +
                                     std::to_string((size_t)MB_STATIC_SCRATCH_BYTES) +
                                     " (MB_STATIC_SCRATCH_BYTES); solve fewer or smaller problems per call, or use mb_batch_solve");
    CUDA_TRY(ctx, cudaSetDevice(ctx->device));
    void* scratch = nullptr;
    size_t cap = 0;
    int e = mb_static_scratch(ctx->device, &scratch, &cap);
    if (e != 0) return fail(ctx, MB_E_CUDA, std::string("static scratch lookup: ") + cudaGetErrorString((cudaError_t)e));
    if (L.total > cap) return fail(ctx, MB_E_NOMEM, "mb_batch_solve_static: the static scratch is smaller than its declared size");
    char* base = (char*)scratch;
    int32_t* s_i32 = (int32_t*)(base + L.i32);
    i64* s_i64 = (i64*)(base + L.i64a);
    double* s_din = (double*)(base + L.din);
    double* s_work = (double*)(base + L.work);
    double* s_out = (double*)(base + L.out);
    int32_t* s_ost = (int32_t*)(base + L.ost);
    mb::DevInst* s_inst = (mb::DevInst*)(base + L.inst);
    int* s_counter = (int*)(base + L.counter);
    mb::CoopCtl* s_coop = (mb::CoopCtl*)(base + L.coop);
    std::vector<mb::DevInst> hi;
    hi.reserve(pk.plans.size());
    for (const InstPlan& p : pk.plans)
        hi.push_back(static_devinst(p, s_i32, s_i64, s_din, s_work, s_out, s_ost, base + L.F));
    order_by_cost(hi, pk.plans);
    cudaStream_t st = ctx->stream;
    if (pk.i32.size()) CUDA_TRY(ctx, cudaMemcpyAsync(s_i32, pk.i32.h.data(), pk.i32.size() * sizeof(int32_t), cudaMemcpyHostToDevice, st));
    if (pk.i64a.size()) CUDA_TRY(ctx, cudaMemcpyAsync(s_i64, pk.i64a.h.data(), pk.i64a.size() * sizeof(i64), cudaMemcpyHostToDevice, st));
    if (pk.din.size()) CUDA_TRY(ctx, cudaMemcpyAsync(s_din, pk.din.h.data(), pk.din.size() * sizeof(double), cudaMemcpyHostToDevice, st));
    CUDA_TRY(ctx, cudaMemcpyAsync(s_inst, hi.data(), hi.size() * sizeof(mb::DevInst), cudaMemcpyHostToDevice, st));
    // the status words start at zero (mb_batch_solve clears its fresh array the same way); the
    // work counter is cleared by mb_launch_batch
    CUDA_TRY(ctx, cudaMemsetAsync(s_ost, 0, std::max<size_t>(pk.ost.size(), 1) * sizeof(int32_t), st));
    int ninst = (int)pk.plans.size();
    int g = std::min(grid > 0 ? grid : ctx->nsm * mb::CTA_PER_SM, ninst);
    mb::Settings ds;
    std::memcpy(&ds, &s, sizeof(ds));
    // the same choice as mb_batch_solve: a lone large instance runs grid-cooperatively, its control
    // block in the scratch
    const bool coop = ninst == 1 && !s.stable && (s.large == 1 || (s.large == 0 && pk.plans[0].fflops >= MB_LARGE_FLOPS));
    const int lrc = coop ? launch_coop(s, s_inst, mb::MODE_SOLVE, &ds, s_coop, ctx->device, ctx->nsm, st)
                         : launch_batch(s, s_inst, ninst, mb::MODE_SOLVE, &ds, s_counter,
                                        use_tc_build(s, false) ? std::min(g, ctx->nsm) : g, st);
    if (lrc) return fail(ctx, MB_E_CUDA, std::string("launch failed: ") + cudaGetErrorString(cudaGetLastError()));
    std::vector<double> h_out(std::max<size_t>(pk.out.size(), 1));
    std::vector<int32_t> h_ost(std::max<size_t>(pk.ost.size(), 1));
    CUDA_TRY(ctx, cudaMemcpyAsync(h_out.data(), s_out, h_out.size() * sizeof(double), cudaMemcpyDeviceToHost, st));
    CUDA_TRY(ctx, cudaMemcpyAsync(h_ost.data(), s_ost, h_ost.size() * sizeof(int32_t), cudaMemcpyDeviceToHost, st));
    CUDA_TRY(ctx, cudaStreamSynchronize(st));
    for (const InstPlan& ip : pk.plans)
        if (h_ost[ip.status + 7]) return fail(ctx, MB_E_TIMEOUT, timeout_msg(h_ost[ip.status + 7]));
    for (size_t k = 0; k < pk.plans.size(); ++k)
        static_unpack(pk.plans[k], h_out.data(), h_ost.data(), s.max_iter, p_out ? p_out[k] : nullptr,
                      d_out ? d_out[k] : nullptr, y_out ? y_out[k] : nullptr, results ? &results[k] : nullptr);
    return MB_OK;
}

// ---------------------------------------------------------------------------------------------
// Serving loop: continuous batching of independent requests (no counterpart in the reference,
// which solves one problem per call).  One device arena and one descriptor ring are allocated at
// creation; requests are planned by a pool of host threads, admitted in arrival order while their
// footprint fits the arena and a ring slot is free, and launched in admission waves, each on an
// idle stream of a pool, so that new requests start on SMs as soon as earlier requests' CTAs
// retire while those keep running.  Each instance stamps its completion into mapped host memory;
// results are copied back as the stamps appear.  No kernel waits on the host or on another kernel.
// ---------------------------------------------------------------------------------------------
#include <chrono>
#include <condition_variable>
#include <deque>
#include <map>
#include <mutex>
#include <unordered_map>
#include <map>

extern "C" int mb_launch_wave(const mb::DevInst* d_inst, int ninst, const mb::Settings* set, int* d_counter, int grid,
                              unsigned long long* done, long long seq0, int cap, cudaStream_t stream);
extern "C" int mb_launch_wave_tc(const mb::DevInst* d_inst, int ninst, const mb::Settings* set, int* d_counter, int grid,
                                 unsigned long long* done, long long seq0, int cap, cudaStream_t stream);

namespace {

// first-fit allocator over [0, cap) in 256-byte granules, coalescing on release
struct RangeAlloc {
    std::map<size_t, size_t> fr;   // offset -> length
    size_t cap = 0, used = 0;
    void init(size_t c) { cap = c; fr.clear(); fr[0] = c; used = 0; }
    static size_t round(size_t n) { return (std::max<size_t>(n, 1) + 255) / 256 * 256; }
    bool alloc(size_t n, size_t& off) {
        n = round(n);
        for (auto it = fr.begin(); it != fr.end(); ++it)
            if (it->second >= n) {
                off = it->first;
                size_t rest = it->second - n;
                fr.erase(it);
                if (rest) fr[off + n] = rest;
                used += n;
                return true;
            }
        return false;
    }
    void release(size_t off, size_t n) {
        n = round(n);
        used -= n;
        auto it = fr.emplace(off, n).first;
        auto nx = std::next(it);
        if (nx != fr.end() && it->first + it->second == nx->first) { it->second += nx->second; fr.erase(nx); }
        if (it != fr.begin()) {
            auto pv = std::prev(it);
            if (pv->first + pv->second == it->first) { pv->second += it->second; fr.erase(it); }
        }
    }
};

double now_s() {
    using namespace std::chrono;
    return duration<double>(steady_clock::now().time_since_epoch()).count();
}

enum ReqState { RQ_QUEUED = 0, RQ_PLANNED = 1, RQ_RUNNING = 2, RQ_DONE = 3, RQ_FAILED = 4 };

struct Request {
    int64_t ticket = 0;
    mb_problem* prob = nullptr;
    int state = RQ_QUEUED;
    int rc = MB_OK;
    std::string err;
    Packed pk;
    size_t bytes = 0, off = 0;
    uint64_t seq = 0;
    double t_submit = 0, t_admit = 0, t_done = 0;
    std::vector<double> p, d, y;
    mb_result res{};
    int64_t dev_t0 = 0, dev_t1 = 0;
};

constexpr int SERVE_STREAMS = 64;

}  // namespace

struct mb_server {
    mb_ctx* ctx = nullptr;
    mb_settings set{};
    cudaStream_t cstream = nullptr;
    cudaStream_t ks[SERVE_STREAMS] = {};
    cudaEvent_t klast[SERVE_STREAMS] = {};   // last launch on each stream
    bool kused[SERVE_STREAMS] = {};
    cudaEvent_t evpub = nullptr;
    int rr = 0;
    int grid_max = 0;
    char* d_arena = nullptr;
    RangeAlloc arena;
    mb::DevInst* d_ring = nullptr;
    int* d_cnt = nullptr;                    // one work counter per stream
    unsigned long long* h_done = nullptr;    // mapped
    unsigned long long* dv_done = nullptr;   // its device alias
    int32_t* h_zero = nullptr;               // pinned zeros: a request's status words are cleared by a copy
    static constexpr size_t ZERO_WORDS = 256;
    int cap = 0;
    uint64_t next_seq = 0;
    std::map<uint64_t, Request*> inflight;   // by seq
    std::unordered_map<int64_t, std::unique_ptr<Request>> reqs;
    std::deque<Request*> queued, planned;
    int64_t next_ticket = 1;
    int64_t nlaunch = 0, ncomplete = 0, nfail = 0;
    double t0 = 0;
    std::mutex mu;
    std::condition_variable cv_plan, cv_done;
    bool quit = false;
    std::string fatal;
    std::vector<std::thread> planners;
    std::thread loop;

    ~mb_server() {
        {
            std::lock_guard<std::mutex> lk(mu);
            quit = true;
        }
        cv_plan.notify_all();
        for (auto& t : planners) if (t.joinable()) t.join();
        if (loop.joinable()) loop.join();
        for (int i = 0; i < SERVE_STREAMS; ++i) if (ks[i]) cudaStreamSynchronize(ks[i]);
        if (cstream) cudaStreamSynchronize(cstream);
        cudaFree(d_arena); cudaFree(d_ring); cudaFree(d_cnt);
        if (h_done) cudaFreeHost(h_done);
        if (h_zero) cudaFreeHost(h_zero);
        for (int i = 0; i < SERVE_STREAMS; ++i) {
            if (klast[i]) cudaEventDestroy(klast[i]);
            if (ks[i]) cudaStreamDestroy(ks[i]);
        }
        if (evpub) cudaEventDestroy(evpub);
        if (cstream) cudaStreamDestroy(cstream);
    }

    void plan_worker() {
        for (;;) {
            Request* r = nullptr;
            {
                std::unique_lock<std::mutex> lk(mu);
                cv_plan.wait(lk, [&] { return quit || !queued.empty(); });
                if (quit) return;
                r = queued.front();
                queued.pop_front();
            }
            std::string err;
            Packed pk;
            int rc = plan_instance(r->prob, set, nullptr, nullptr, nullptr, pk, err);
            size_t bytes = rc ? 0 : StaticLayout(pk).total;
            std::lock_guard<std::mutex> lk(mu);
            if (rc) { r->rc = rc; r->err = err; r->state = RQ_FAILED; r->t_done = now_s() - t0; ++nfail; cv_done.notify_all(); continue; }
            if (bytes > arena.cap) {
                r->rc = MB_E_NOMEM; r->err = "request footprint exceeds the server arena"; r->state = RQ_FAILED;
                r->t_done = now_s() - t0; ++nfail; cv_done.notify_all(); continue;
            }
            r->pk = std::move(pk);
            r->bytes = bytes;
            r->state = RQ_PLANNED;
            planned.push_back(r);
        }
    }

    // copy one planned request into the arena and its ring slot (caller holds mu)
    int stage(Request* r) {
        const StaticLayout L(r->pk);
        char* base = d_arena + r->off;
        int32_t* s_i32 = (int32_t*)(base + L.i32);
        i64* s_i64 = (i64*)(base + L.i64a);
        double* s_din = (double*)(base + L.din);
        int32_t* s_ost = (int32_t*)(base + L.ost);
        mb::DevInst I = static_devinst(r->pk.plans[0], s_i32, s_i64, s_din, (double*)(base + L.work),
                                       (double*)(base + L.out), s_ost, base + L.F);
        const Packed& pk = r->pk;
        cudaError_t e = cudaSuccess;
        if (pk.i32.size() && !e) e = cudaMemcpyAsync(s_i32, pk.i32.h.data(), pk.i32.size() * 4, cudaMemcpyHostToDevice, cstream);
        if (pk.i64a.size() && !e) e = cudaMemcpyAsync(s_i64, pk.i64a.h.data(), pk.i64a.size() * 8, cudaMemcpyHostToDevice, cstream);
        if (pk.din.size() && !e) e = cudaMemcpyAsync(s_din, pk.din.h.data(), pk.din.size() * 8, cudaMemcpyHostToDevice, cstream);
        // zeroed by a copy, not a memset: a memset runs as a kernel, which waits for SMs that running
        // waves hold, and the pageable copy of the ring slot below would then hold up admission
        const size_t ost_words = std::max<size_t>(pk.ost.size(), 1);
        if (!e) e = ost_words <= mb_server::ZERO_WORDS
                        ? cudaMemcpyAsync(s_ost, h_zero, ost_words * 4, cudaMemcpyHostToDevice, cstream)
                        : cudaMemsetAsync(s_ost, 0, ost_words * 4, cstream);
        r->seq = next_seq;
        if (!e) e = cudaMemcpyAsync(d_ring + r->seq % cap, &I, sizeof(I), cudaMemcpyHostToDevice, cstream);
        if (e) { fatal = std::string("serve staging: ") + cudaGetErrorString(e); return MB_E_CUDA; }
        ++next_seq;
        r->state = RQ_RUNNING;
        r->t_admit = now_s() - t0;
        inflight[r->seq] = r;
        return MB_OK;
    }

    // launch ring slots [s0, s1) on an idle stream after the staging copies (caller holds mu)
    void launch(uint64_t s0, uint64_t s1) {
        if (cudaEventRecord(evpub, cstream) != cudaSuccess) { fatal = "serve: event record failed"; return; }
        int k = -1;
        for (int t = 0; t < SERVE_STREAMS && k < 0; ++t) {
            int i = (rr + t) % SERVE_STREAMS;
            if (!kused[i] || cudaEventQuery(klast[i]) == cudaSuccess) k = i;
        }
        if (k < 0) k = rr % SERVE_STREAMS;   // every stream busy: queue behind the oldest choice
        rr = (k + 1) % SERVE_STREAMS;
        cudaStreamWaitEvent(ks[k], evpub, 0);
        mb::Settings ds;
        std::memcpy(&ds, &set, sizeof(ds));
        while (s0 < s1) {   // one launch per contiguous run of ring slots
            uint64_t end = std::min<uint64_t>(s1, (s0 / cap + 1) * (uint64_t)cap);
            int n = (int)(end - s0);
            int g = std::min(n, grid_max);
            const bool tcw = use_tc_build(set, false);
            if ((tcw ? mb_launch_wave_tc : mb_launch_wave)(d_ring + s0 % cap, n, &ds, d_cnt + k, tcw ? std::min(g, grid_max / mb::CTA_PER_SM) : g,
                                                           dv_done, (long long)s0, cap, ks[k])) {
                fatal = std::string("serve launch: ") + cudaGetErrorString(cudaGetLastError());
                return;
            }
            ++nlaunch;
            s0 = end;
        }
        cudaEventRecord(klast[k], ks[k]);
        kused[k] = true;
    }

    // copy one finished request's outputs back and release its arena (caller holds mu)
    void collect(Request* r) {
        const StaticLayout L(r->pk);
        char* base = d_arena + r->off;
        const Packed& pk = r->pk;
        std::vector<double> h_out(std::max<size_t>(pk.out.size(), 1));
        std::vector<int32_t> h_ost(std::max<size_t>(pk.ost.size(), 1));
        cudaError_t e = cudaMemcpyAsync(h_out.data(), base + L.out, h_out.size() * 8, cudaMemcpyDeviceToHost, cstream);
        if (!e) e = cudaMemcpyAsync(h_ost.data(), base + L.ost, h_ost.size() * 4, cudaMemcpyDeviceToHost, cstream);
        if (!e) e = cudaStreamSynchronize(cstream);
        const InstPlan& ip = pk.plans[0];
        if (e) { r->rc = MB_E_CUDA; r->err = cudaGetErrorString(e); r->state = RQ_FAILED; ++nfail; }
        else {
            r->p.assign(ip.n, 0.0); r->d.assign(ip.n, 0.0); r->y.assign(ip.m, 0.0);
            static_unpack(ip, h_out.data(), h_ost.data(), set.max_iter, r->p.data(), r->d.data(), r->y.data(), &r->res);
            std::memcpy(&r->dev_t0, &h_out[ip.scal + mb::SCAL_T0], 8);
            std::memcpy(&r->dev_t1, &h_out[ip.scal + mb::SCAL_T1], 8);
            r->state = RQ_DONE;
            ++ncomplete;
        }
        r->t_done = now_s() - t0;
        arena.release(r->off, r->bytes);
        r->pk = Packed();
    }

    void run_loop() {
        cudaSetDevice(ctx->device);
        for (;;) {
            bool busy = false;
            {
                std::lock_guard<std::mutex> lk(mu);
                if (quit && inflight.empty() && planned.empty()) return;
                // collect finished requests (any order)
                for (auto it = inflight.begin(); it != inflight.end();) {
                    Request* r = it->second;
                    volatile unsigned long long* dn = h_done + r->seq % cap;
                    if (*dn == r->seq + 1) {
                        collect(r);
                        it = inflight.erase(it);
                        busy = true;
                        cv_done.notify_all();
                    } else ++it;
                }
                // a failed launch shows up as an error on its stream's event
                for (int i = 0; i < SERVE_STREAMS && fatal.empty(); ++i)
                    if (kused[i]) {
                        cudaError_t e = cudaEventQuery(klast[i]);
                        if (e != cudaSuccess && e != cudaErrorNotReady) fatal = std::string("serve kernel: ") + cudaGetErrorString(e);
                    }
                // admit in planning order while the arena and the ring have room, then launch the wave
                uint64_t s0 = next_seq;
                while (!planned.empty() && fatal.empty()) {
                    Request* r = planned.front();
                    uint64_t oldest = inflight.empty() ? next_seq : inflight.begin()->first;
                    if (next_seq - oldest >= (uint64_t)cap) break;
                    if (!arena.alloc(r->bytes, r->off)) break;
                    planned.pop_front();
                    if (stage(r)) { arena.release(r->off, r->bytes); r->state = RQ_FAILED; r->rc = MB_E_CUDA; r->err = fatal; ++nfail; }
                    busy = true;
                }
                if (next_seq > s0 && fatal.empty()) launch(s0, next_seq);
                if (!fatal.empty()) {   // fail everything outstanding
                    for (auto& kv : inflight) { kv.second->state = RQ_FAILED; kv.second->rc = MB_E_CUDA; kv.second->err = fatal; ++nfail; }
                    inflight.clear();
                    for (Request* r : planned) { r->state = RQ_FAILED; r->rc = MB_E_CUDA; r->err = fatal; ++nfail; }
                    planned.clear();
                    cv_done.notify_all();
                    if (quit) return;
                }
            }
            if (!busy) std::this_thread::sleep_for(std::chrono::microseconds(20));
        }
    }
};

extern "C" {

int mb_server_create(mb_ctx* ctx, const mb_settings* settings, int64_t arena_bytes, int32_t capacity,
                     int32_t nplanners, mb_server** out) {
    if (!ctx || !out || arena_bytes <= 0 || capacity <= 0) return fail(ctx, MB_E_ARG, "bad arguments");
    mb_settings s;
    if (settings) s = *settings; else mb_settings_default(&s);
    if (s.stable && s.precision != MB_PREC_FP64)
        return fail(ctx, MB_E_UNSUPPORTED, "stable=true (StableUzawaSolver) factors in FP64: precision must be 0");
    if (s.precision < 0 || s.precision > 2) return fail(ctx, MB_E_ARG, "precision must be 0, 1 or 2");
    auto sv = std::make_unique<mb_server>();
    sv->ctx = ctx; sv->set = s; sv->cap = capacity;
    sv->grid_max = ctx->nsm * mb::CTA_PER_SM;
    sv->t0 = now_s();
    CUDA_TRY(ctx, cudaSetDevice(ctx->device));
    CUDA_TRY(ctx, cudaStreamCreateWithFlags(&sv->cstream, cudaStreamNonBlocking));
    for (int i = 0; i < SERVE_STREAMS; ++i) {
        CUDA_TRY(ctx, cudaStreamCreateWithFlags(&sv->ks[i], cudaStreamNonBlocking));
        CUDA_TRY(ctx, cudaEventCreateWithFlags(&sv->klast[i], cudaEventDisableTiming));
    }
    CUDA_TRY(ctx, cudaEventCreateWithFlags(&sv->evpub, cudaEventDisableTiming));
    CUDA_TRY(ctx, cudaMalloc((void**)&sv->d_arena, (size_t)arena_bytes));
    CUDA_TRY(ctx, cudaMalloc((void**)&sv->d_ring, sizeof(mb::DevInst) * capacity));
    CUDA_TRY(ctx, cudaMalloc((void**)&sv->d_cnt, sizeof(int) * SERVE_STREAMS));
    CUDA_TRY(ctx, cudaHostAlloc((void**)&sv->h_done, sizeof(unsigned long long) * capacity, cudaHostAllocMapped));
    std::memset(sv->h_done, 0, sizeof(unsigned long long) * capacity);
    CUDA_TRY(ctx, cudaMallocHost((void**)&sv->h_zero, mb_server::ZERO_WORDS * sizeof(int32_t)));
    std::memset(sv->h_zero, 0, mb_server::ZERO_WORDS * sizeof(int32_t));
    CUDA_TRY(ctx, cudaHostGetDevicePointer((void**)&sv->dv_done, sv->h_done, 0));
    sv->arena.init((size_t)arena_bytes);
    int np = nplanners > 0 ? nplanners : (int)std::max(1u, std::thread::hardware_concurrency() / 2);
    mb_server* raw = sv.get();
    for (int t = 0; t < np; ++t) sv->planners.emplace_back([raw] { raw->plan_worker(); });
    sv->loop = std::thread([raw] { raw->run_loop(); });
    *out = sv.release();
    return MB_OK;
}

int mb_server_submit(mb_server* s, mb_problem* prob, int64_t* ticket) {
    if (!s || !prob || !ticket) return MB_E_ARG;
    auto r = std::make_unique<Request>();
    r->prob = prob;
    std::lock_guard<std::mutex> lk(s->mu);
    if (!s->fatal.empty()) return fail(s->ctx, MB_E_CUDA, s->fatal);
    r->ticket = s->next_ticket++;
    r->t_submit = now_s() - s->t0;
    *ticket = r->ticket;
    s->queued.push_back(r.get());
    s->reqs[r->ticket] = std::move(r);
    s->cv_plan.notify_one();
    return MB_OK;
}

int mb_server_poll(mb_server* s, int64_t ticket, int32_t* state) {
    if (!s || !state) return MB_E_ARG;
    std::lock_guard<std::mutex> lk(s->mu);
    auto it = s->reqs.find(ticket);
    if (it == s->reqs.end()) return MB_E_ARG;
    *state = it->second->state;
    return MB_OK;
}

int mb_server_wait(mb_server* s, int64_t ticket, double timeout_s, int32_t* state) {
    if (!s || !state) return MB_E_ARG;
    std::unique_lock<std::mutex> lk(s->mu);
    auto it = s->reqs.find(ticket);
    if (it == s->reqs.end()) return MB_E_ARG;
    Request* r = it->second.get();
    s->cv_done.wait_for(lk, std::chrono::duration<double>(std::max(0.0, timeout_s)),
                        [&] { return r->state == RQ_DONE || r->state == RQ_FAILED; });
    *state = r->state;
    return MB_OK;
}

int mb_server_result(mb_server* s, int64_t ticket, double* p, double* d, double* y, mb_result* res, double* times5) {
    if (!s) return MB_E_ARG;
    std::unique_ptr<Request> r;
    {
        std::lock_guard<std::mutex> lk(s->mu);
        auto it = s->reqs.find(ticket);
        if (it == s->reqs.end()) return MB_E_ARG;
        if (it->second->state != RQ_DONE && it->second->state != RQ_FAILED) return fail(s->ctx, MB_E_STATE, "request not finished");
        r = std::move(it->second);
        s->reqs.erase(it);
    }
    if (times5) {
        times5[0] = r->t_submit; times5[1] = r->t_admit; times5[2] = r->t_done;
        times5[3] = (double)r->dev_t0; times5[4] = (double)r->dev_t1;
    }
    if (r->state == RQ_FAILED) return fail(s->ctx, r->rc, r->err);
    if (p) std::copy(r->p.begin(), r->p.end(), p);
    if (d) std::copy(r->d.begin(), r->d.end(), d);
    if (y) std::copy(r->y.begin(), r->y.end(), y);
    if (res) *res = r->res;
    return MB_OK;
}

int mb_server_stats(mb_server* s, int64_t* st) {
    if (!s || !st) return MB_E_ARG;
    std::lock_guard<std::mutex> lk(s->mu);
    st[0] = (int64_t)s->queued.size(); st[1] = (int64_t)s->planned.size(); st[2] = (int64_t)s->inflight.size();
    st[3] = s->ncomplete; st[4] = s->nfail; st[5] = s->nlaunch; st[6] = (int64_t)s->arena.used; st[7] = (int64_t)s->arena.cap;
    return MB_OK;
}

int mb_server_destroy(mb_server* s) {
    if (!s) return MB_E_ARG;
    delete s;
    return MB_OK;
}

}  // extern "C"
