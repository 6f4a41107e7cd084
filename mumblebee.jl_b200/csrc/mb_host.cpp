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
#include <memory>
#include <string>
#include <vector>

#include "../../include/mumblebee_gpu.h"
#include "mb_internal.h"
#include "mb_symbolic.hpp"

extern "C" int mb_launch_batch(const mb::DevInst* d_inst, int ninst, int mode, const mb::Settings* set,
                               int* d_counter, int grid, int fp32, cudaStream_t stream);

using mbh::i64;

struct mb_ctx {
    int device = 0;
    int nsm = 148;
    cudaStream_t stream = nullptr;
    std::string err;
};

struct mb_problem {
    mb_ctx* ctx = nullptr;
    mbh::BSM Q, B;
    std::vector<double> f, g;
    double mu = 0;
    std::vector<int32_t> kind;
    std::vector<double> param;
    std::vector<i64> P1, P2;   // 0-based user row / column of each problem row / column
    // symbolic analysis, computed once
    bool sym = false;
    std::vector<i64> vperm;    // problem vertex of each solver vertex
    mbh::Fronts fr;
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
static void do_symbolic(mb_problem* P) {
    if (P->sym) return;
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
    P->fr = mbh::analyze(adj2, w2);
    P->vperm.resize(nv);
    for (i64 k = 0; k < nv; ++k) P->vperm[k] = order[P->fr.postperm[k]];
    P->sym = true;
}

// ---------------------------------------------------------------------------------------------
// packing instances into device arenas
// ---------------------------------------------------------------------------------------------
template <class T>
struct Arena {
    std::vector<T> h;
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
    // i32
    size_t Bxsrc, Bxcol, Bxrow, Btgt, Brptr, Brarc, Brvtx, Browout, Bcolvtx;
    size_t Qxsrc, Qtgt, Qrptr, Qrarc, Qrvtx;
    size_t qdiag, hld, kind, fres0, fnres, fnsep, fparent, fsepp, fsep, frel, vfront, status;
    i64 Bnout, Bnarc, Qnarc;
    // i64
    size_t Bxblk, Qxblk, hpos, cxblk, fptr;
    // double in
    size_t Bval, Qval, f, g, kpar, p, d, y;
    // work
    size_t H, Finit, pscl, yscl, vn, vm, vv, work, uhist, cghist, cache;
    size_t wBval, wQval, wf, wg, wp, wd, wy;   // working copies
    // factor
    size_t F;
    // out
    size_t po, dout, yo, scal, hist;
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
    size_t fbytes = 0;        // factor arena, bytes
    std::vector<InstPlan> plans;
    Packed() { work.host = false; out.host = false; }
    size_t device_bytes() const {
        return i32.size() * 4 + i64a.size() * 8 + din.size() * 8 + work.size() * 8 + out.size() * 8 + fbytes;
    }
};

static void bsm_rowindex(const mbh::BSM& A, std::vector<i64>& rptr, std::vector<i64>& rarc, std::vector<i64>& rvtx,
                         std::vector<i64>& rowout, std::vector<i64>& colvtx) {
    rptr.assign(A.nout + 1, 0);
    for (i64 e = 0; e < A.narc; ++e) rptr[A.tgt[e] + 1]++;
    for (i64 u = 0; u < A.nout; ++u) rptr[u + 1] += rptr[u];
    rarc.assign(A.narc, 0); rvtx.assign(A.narc, 0);
    std::vector<i64> c(rptr.begin(), rptr.end() - 1);
    for (i64 v = 0; v < A.nvtx; ++v)
        for (i64 e = A.xsrc[v]; e < A.xsrc[v + 1]; ++e) { i64 k = c[A.tgt[e]]++; rarc[k] = e; rvtx[k] = v; }
    rowout.assign(A.nrow, 0);
    for (i64 u = 0; u < A.nout; ++u) for (i64 i = A.xrow[u]; i < A.xrow[u + 1]; ++i) rowout[i] = u;
    colvtx.assign(A.ncol, 0);
    for (i64 v = 0; v < A.nvtx; ++v) for (i64 j = A.xcol[v]; j < A.xcol[v + 1]; ++j) colvtx[j] = v;
}

static int64_t cone_cachesize(int k, i64 n) { return k == MB_CONE_SOC ? 5 + n : 0; }
static int64_t cone_workspacesize(int k, i64 n) { return k == MB_CONE_SOC ? 2 * n : 0; }
static int64_t cone_degree(int k, i64 n) { return k == MB_CONE_POS ? n : (k == MB_CONE_SOC ? 2 : 0); }

static int plan_instance(mb_problem* P, const mb_settings& set, const double* p0, const double* d0, const double* y0,
                         Packed& pk, std::string& err) {
    do_symbolic(P);
    const auto& vp = P->vperm;
    mbh::BSM B = mbh::selectvtxs(P->B, vp);
    mbh::BSM Q = mbh::halfselectvtxs(mbh::halfselectvtxs(P->Q, vp), vp);
    const mbh::Fronts& fr = P->fr;
    InstPlan ip;
    ip.n = B.ncol; ip.m = B.nrow; ip.nvtx = B.nvtx; ip.nfront = fr.nfront;
    ip.mut = P->mu;
    for (i64 v = 0; v < B.nvtx; ++v) {
        int k = P->kind[vp[v]];
        if (k != MB_CONE_FREE && k != MB_CONE_POS && k != MB_CONE_SOC) { err = "cone kind not supported by this build"; return MB_E_UNSUPPORTED; }
    }
    // column map: solver column -> problem column -> user column
    std::vector<i64> cperm;
    cperm.reserve(B.ncol);
    for (i64 k = 0; k < B.nvtx; ++k) for (i64 j = P->B.xcol[vp[k]]; j < P->B.xcol[vp[k] + 1]; ++j) cperm.push_back(j);
    ip.colmap.resize(B.ncol); ip.rowmap.resize(B.nrow);
    for (i64 i = 0; i < B.ncol; ++i) ip.colmap[i] = P->P2[cperm[i]];
    for (i64 i = 0; i < B.nrow; ++i) ip.rowmap[i] = P->P1[i];
    // index structures
    std::vector<i64> rptr, rarc, rvtx, rowout, colvtx;
    bsm_rowindex(B, rptr, rarc, rvtx, rowout, colvtx);
    ip.Bnout = B.nout; ip.Bnarc = B.narc; ip.Qnarc = Q.narc;
    ip.Bxsrc = pk.i32.put(to32(B.xsrc)); ip.Bxcol = pk.i32.put(to32(B.xcol)); ip.Bxrow = pk.i32.put(to32(B.xrow));
    ip.Btgt = pk.i32.put(to32(B.tgt)); ip.Brptr = pk.i32.put(to32(rptr)); ip.Brarc = pk.i32.put(to32(rarc));
    ip.Brvtx = pk.i32.put(to32(rvtx)); ip.Browout = pk.i32.put(to32(rowout)); ip.Bcolvtx = pk.i32.put(to32(colvtx));
    std::vector<i64> qrptr, qrarc, qrvtx, qrowout, qcolvtx;
    bsm_rowindex(Q, qrptr, qrarc, qrvtx, qrowout, qcolvtx);
    ip.Qxsrc = pk.i32.put(to32(Q.xsrc)); ip.Qtgt = pk.i32.put(to32(Q.tgt)); ip.Qrptr = pk.i32.put(to32(qrptr));
    ip.Qrarc = pk.i32.put(to32(qrarc)); ip.Qrvtx = pk.i32.put(to32(qrvtx));
    std::vector<i64> qdiag(B.nvtx, -1);
    for (i64 v = 0; v < Q.nvtx; ++v) for (i64 e = Q.xsrc[v]; e < Q.xsrc[v + 1]; ++e) if (Q.tgt[e] == v) qdiag[v] = e;
    // every non-free cone needs its diagonal block (cone.jl:146-174 errors otherwise)
    for (i64 v = 0; v < B.nvtx; ++v)
        if (qdiag[v] < 0 && P->kind[vp[v]] != MB_CONE_FREE) { err = "Q lacks the diagonal block of a cone vertex"; return MB_E_ARG; }
    // fronts
    std::vector<i64> fnsep(fr.nfront), fsepp(fr.nfront + 1, 0), fsep, frel;
    for (i64 f = 0; f < fr.nfront; ++f) {
        fnsep[f] = (i64)fr.sep[f].size();
        fsepp[f + 1] = fsepp[f] + fnsep[f];
        fsep.insert(fsep.end(), fr.sep[f].begin(), fr.sep[f].end());
        if (fr.parent[f] >= 0) frel.insert(frel.end(), fr.rel[f].begin(), fr.rel[f].end());
        else frel.insert(frel.end(), fr.sep[f].size(), 0);
    }
    // H placement in fronts: block (u, v) with u >= v lands at rows rowpos(f, xcol[u]) of front f(v)
    std::vector<i64> hpos(Q.narc, -1), hld(Q.narc, 0);
    for (i64 v = 0; v < Q.nvtx; ++v) {
        i64 f = fr.vfront[v], nres = fr.nres[f], nf = nres + (i64)fr.sep[f].size(), r0 = fr.res0[f];
        for (i64 e = Q.xsrc[v]; e < Q.xsrc[v + 1]; ++e) {
            i64 u = Q.tgt[e];
            if (u < v) continue;
            i64 s = B.xcol[u], rp;
            if (s >= r0 && s < r0 + nres) rp = s - r0;
            else {
                auto it = std::lower_bound(fr.sep[f].begin(), fr.sep[f].end(), s);
                if (it == fr.sep[f].end() || *it != s) { err = "internal: Q block outside the front structure"; return MB_E_ARG; }
                rp = nres + (i64)(it - fr.sep[f].begin());
            }
            hpos[e] = fr.fptr[f] + rp + (B.xcol[v] - r0) * nf;
            hld[e] = nf;
        }
    }
    std::vector<i64> kind(B.nvtx), cx(B.nvtx + 1, 0);
    std::vector<double> kpar(B.nvtx);
    i64 wmax = 1;
    ip.nu = 0;
    for (i64 v = 0; v < B.nvtx; ++v) {
        kind[v] = P->kind[vp[v]]; kpar[v] = P->param[vp[v]];
        cx[v + 1] = cx[v] + cone_cachesize((int)kind[v], B.ncols(v));
        wmax = std::max<i64>(wmax, cone_workspacesize((int)kind[v], B.ncols(v)));
        ip.nu += cone_degree((int)kind[v], B.ncols(v));
    }
    ip.wsize = (int)wmax;
    ip.qdiag = pk.i32.put(to32(qdiag)); ip.hld = pk.i32.put(to32(hld)); ip.kind = pk.i32.put(to32(kind));
    ip.fres0 = pk.i32.put(to32(fr.res0)); ip.fnres = pk.i32.put(to32(fr.nres)); ip.fnsep = pk.i32.put(to32(fnsep));
    ip.fparent = pk.i32.put(to32(fr.parent)); ip.fsepp = pk.i32.put(to32(fsepp)); ip.fsep = pk.i32.put(to32(fsep));
    ip.frel = pk.i32.put(to32(frel)); ip.vfront = pk.i32.put(to32(fr.vfront));
    ip.status = pk.i32.take(mb::NSTAT);
    ip.Bxblk = pk.i64a.put(B.xblk); ip.Qxblk = pk.i64a.put(Q.xblk); ip.hpos = pk.i64a.put(hpos);
    ip.cxblk = pk.i64a.put(cx); ip.fptr = pk.i64a.put(fr.fptr);
    // values
    std::vector<double> f(B.ncol), g(P->g);
    for (i64 i = 0; i < B.ncol; ++i) f[i] = P->f[cperm[i]];
    ip.Bval = pk.din.put(B.val); ip.Qval = pk.din.put(Q.val); ip.f = pk.din.put(f); ip.g = pk.din.put(g);
    ip.kpar = pk.din.put(kpar);
    std::vector<double> pv(B.ncol, 0.0), dv(B.ncol, 0.0), yv(B.nrow, 0.0);
    ip.has_p0 = p0 != nullptr; ip.has_d0 = d0 != nullptr; ip.has_y0 = y0 != nullptr;
    for (i64 i = 0; i < B.ncol; ++i) { if (p0) pv[i] = p0[ip.colmap[i]]; if (d0) dv[i] = d0[ip.colmap[i]]; }
    if (y0) for (i64 i = 0; i < B.nrow; ++i) yv[i] = y0[ip.rowmap[i]];
    ip.p = pk.din.put(pv); ip.d = pk.din.put(dv); ip.y = pk.din.put(yv);
    // workspace
    ip.fsize = fr.fsize;
    ip.H = pk.work.take(Q.nbnz); ip.Finit = pk.work.take(fr.fsize);
    ip.pscl = pk.work.take(B.ncol); ip.yscl = pk.work.take(B.nrow);
    ip.vn = pk.work.take((size_t)mb::NVEC_N * B.ncol); ip.vm = pk.work.take((size_t)mb::NVEC_M * B.nrow);
    ip.vv = pk.work.take((size_t)mb::NVEC_V * B.nvtx); ip.work = pk.work.take((size_t)(512 / 32) * wmax);
    ip.uhist = pk.work.take(set.refine_max_iter + 2); ip.cghist = pk.work.take(set.newton_max_iter + 1);
    ip.cache = pk.work.take(std::max<i64>(cx[B.nvtx], 1));
    ip.wBval = pk.work.take(B.nbnz); ip.wQval = pk.work.take(Q.nbnz);
    ip.wf = pk.work.take(B.ncol); ip.wg = pk.work.take(B.nrow);
    ip.wp = pk.work.take(B.ncol); ip.wd = pk.work.take(B.ncol); ip.wy = pk.work.take(B.nrow);
    size_t esz = set.precision == MB_PREC_FP32 ? 4 : 8;
    ip.F = (pk.fbytes + 255) / 256 * 256;
    pk.fbytes = ip.F + fr.fsize * esz;
    ip.po = pk.out.take(B.ncol); ip.dout = pk.out.take(B.ncol); ip.yo = pk.out.take(B.nrow);
    ip.scal = pk.out.take(mb::NSCAL); ip.hist = pk.out.take((size_t)(set.max_iter + 1) * mb::ROW_DOUBLES);
    pk.plans.push_back(std::move(ip));
    return MB_OK;
}

struct mb_batch {
    mb_ctx* ctx = nullptr;
    mb_settings set{};
    std::vector<mb_problem*> probs;
    Packed pk;
    int32_t* d_i32 = nullptr;
    i64* d_i64 = nullptr;
    double* d_din = nullptr;
    double* d_work = nullptr;
    double* d_out = nullptr;
    void* d_F = nullptr;
    mb::DevInst* d_inst = nullptr;
    int* d_counter = nullptr;
    int32_t* h_i32 = nullptr;   // pinned mirrors of the status words
    double* h_out = nullptr;    // pinned output staging
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    int64_t launches = 0;
    ~mb_batch() {
        cudaFree(d_i32); cudaFree(d_i64); cudaFree(d_din); cudaFree(d_work); cudaFree(d_out); cudaFree(d_F);
        cudaFree(d_inst); cudaFree(d_counter);
        cudaFreeHost(h_i32); cudaFreeHost(h_out);
        if (e0) cudaEventDestroy(e0);
        if (e1) cudaEventDestroy(e1);
    }
};

static int upload(mb_batch* b) {
    mb_ctx* ctx = b->ctx;
    Packed& pk = b->pk;
    cudaStream_t st = ctx->stream;
    auto alloc_copy = [&](auto*& dptr, auto& arena) -> int {
        using T = typename std::remove_reference<decltype(arena.h)>::type::value_type;
        size_t bytes = std::max<size_t>(arena.size(), 1) * sizeof(T);
        CUDA_TRY(ctx, cudaMalloc((void**)&dptr, bytes));
        if (arena.host && arena.size()) CUDA_TRY(ctx, cudaMemcpyAsync(dptr, arena.h.data(), arena.size() * sizeof(T), cudaMemcpyHostToDevice, st));
        return MB_OK;
    };
    int rc;
    if ((rc = alloc_copy(b->d_i32, pk.i32))) return rc;
    if ((rc = alloc_copy(b->d_i64, pk.i64a))) return rc;
    if ((rc = alloc_copy(b->d_din, pk.din))) return rc;
    CUDA_TRY(ctx, cudaMalloc((void**)&b->d_work, std::max<size_t>(pk.work.size(), 1) * sizeof(double)));
    CUDA_TRY(ctx, cudaMalloc((void**)&b->d_out, std::max<size_t>(pk.out.size(), 1) * sizeof(double)));
    CUDA_TRY(ctx, cudaMalloc(&b->d_F, std::max<size_t>(pk.fbytes, 256)));
    CUDA_TRY(ctx, cudaMalloc((void**)&b->d_counter, sizeof(int)));
    CUDA_TRY(ctx, cudaMallocHost((void**)&b->h_out, std::max<size_t>(pk.out.size(), 1) * sizeof(double)));
    CUDA_TRY(ctx, cudaMallocHost((void**)&b->h_i32, std::max<size_t>(pk.i32.size(), 1) * sizeof(int32_t)));
    std::vector<mb::DevInst> hi(pk.plans.size());
    for (size_t k = 0; k < pk.plans.size(); ++k) {
        const InstPlan& p = pk.plans[k];
        mb::DevInst& I = hi[k];
        int32_t* i32 = b->d_i32; i64* q64 = b->d_i64; double* dn = b->d_din; double* wk = b->d_work; double* ot = b->d_out;
        I.n = (int)p.n; I.m = (int)p.m; I.nvtx = (int)p.nvtx; I.nfront = (int)p.nfront; I.nu = (int)p.nu;
        I.has_p0 = p.has_p0; I.has_d0 = p.has_d0; I.has_y0 = p.has_y0; I.mut = p.mut;
        auto fillbsm = [&](mb::DevBSM& A, i64 nout, i64 narc, size_t xsrc, size_t xcol, size_t xrow, size_t tgt, size_t xblk,
                           size_t val, size_t rptr, size_t rarc, size_t rvtx, size_t rowout, size_t colvtx, i64 nrow) {
            A.nout = (int)nout; A.nvtx = (int)p.nvtx; A.narc = (int)narc; A.ncol = (int)p.n; A.nrow = (int)nrow;
            A.xsrc = i32 + xsrc; A.xcol = i32 + xcol; A.xrow = i32 + xrow; A.tgt = i32 + tgt;
            A.xblk = (const int64_t*)(q64 + xblk); A.val = wk + val;
            A.rptr = i32 + rptr; A.rarc = i32 + rarc; A.rvtx = i32 + rvtx; A.rowout = i32 + rowout; A.colvtx = i32 + colvtx;
        };
        fillbsm(I.B, p.Bnout, p.Bnarc, p.Bxsrc, p.Bxcol, p.Bxrow, p.Btgt, p.Bxblk, p.wBval, p.Brptr, p.Brarc, p.Brvtx,
                p.Browout, p.Bcolvtx, p.m);
        fillbsm(I.Q, p.nvtx, p.Qnarc, p.Qxsrc, p.Bxcol, p.Bxcol, p.Qtgt, p.Qxblk, p.wQval, p.Qrptr, p.Qrarc, p.Qrvtx,
                p.Bcolvtx, p.Bcolvtx, p.n);
        I.Bval0 = dn + p.Bval; I.Qval0 = dn + p.Qval; I.f0 = dn + p.f; I.g0 = dn + p.g;
        I.p0 = dn + p.p; I.d0 = dn + p.d; I.y0 = dn + p.y;
        I.H = wk + p.H;
        I.qdiag = i32 + p.qdiag; I.hpos = (const int64_t*)(q64 + p.hpos); I.hld = i32 + p.hld;
        I.kind = i32 + p.kind; I.kpar = dn + p.kpar; I.cxblk = (const int64_t*)(q64 + p.cxblk); I.cache = wk + p.cache;
        I.wsize = p.wsize;
        I.fres0 = i32 + p.fres0; I.fnres = i32 + p.fnres; I.fnsep = i32 + p.fnsep; I.fparent = i32 + p.fparent;
        I.fptr = (const int64_t*)(q64 + p.fptr); I.fsepp = i32 + p.fsepp; I.fsep = i32 + p.fsep; I.frel = i32 + p.frel;
        I.fsize = p.fsize;
        I.Finit = wk + p.Finit; I.F = (char*)b->d_F + p.F;
        I.f = wk + p.wf; I.g = wk + p.wg; I.pscl = wk + p.pscl; I.yscl = wk + p.yscl;
        I.p = wk + p.wp; I.d = wk + p.wd; I.y = wk + p.wy;
        I.vn = wk + p.vn; I.vm = wk + p.vm; I.vv = wk + p.vv; I.work = wk + p.work;
        I.vfront = i32 + p.vfront;
        I.po = ot + p.po; I.dout = ot + p.dout; I.yo = ot + p.yo;
        I.hist = ot + p.hist; I.uhist = wk + p.uhist; I.cghist = wk + p.cghist;
        I.status = i32 + p.status; I.scal = ot + p.scal;
    }
    CUDA_TRY(ctx, cudaMalloc((void**)&b->d_inst, hi.size() * sizeof(mb::DevInst)));
    CUDA_TRY(ctx, cudaMemcpyAsync(b->d_inst, hi.data(), hi.size() * sizeof(mb::DevInst), cudaMemcpyHostToDevice, st));
    CUDA_TRY(ctx, cudaEventCreate(&b->e0));
    CUDA_TRY(ctx, cudaEventCreate(&b->e1));
    CUDA_TRY(ctx, cudaStreamSynchronize(st));
    return MB_OK;
}

static int make_batch(mb_ctx* ctx, mb_problem* const* probs, int32_t nprob, const mb_settings* set,
                      const double* p0, const double* d0, const double* y0, mb_batch** out) {
    if (!ctx || !out || nprob < 0 || (nprob > 0 && !probs)) return fail(ctx, MB_E_ARG, "bad arguments");
    mb_settings s;
    if (set) s = *set; else mb_settings_default(&s);
    if (s.stable) return fail(ctx, MB_E_UNSUPPORTED, "stable=true (StableUzawaSolver) is not available");
    if (s.max_iter < 0 || s.refine_max_iter < 0 || s.newton_max_iter < 0) return fail(ctx, MB_E_ARG, "negative iteration limit");
    auto b = std::make_unique<mb_batch>();
    b->ctx = ctx; b->set = s;
    CUDA_TRY(ctx, cudaSetDevice(ctx->device));
    for (int32_t k = 0; k < nprob; ++k) {
        if (!probs[k]) return fail(ctx, MB_E_ARG, "null problem");
        std::string err;
        int rc = plan_instance(probs[k], s, p0, d0, y0, b->pk, err);
        if (rc) return fail(ctx, rc, err);
        b->probs.push_back(probs[k]);
    }
    int rc = upload(b.get());
    if (rc) return rc;
    *out = b.release();
    return MB_OK;
}

static int run_batch(mb_batch* b, int mode, int32_t grid, float* ms) {
    mb_ctx* ctx = b->ctx;
    int ninst = (int)b->pk.plans.size();
    if (ninst == 0) { if (ms) *ms = 0; return MB_OK; }
    int g = grid > 0 ? grid : ctx->nsm;
    g = std::min(g, ninst);
    mb::Settings s;
    static_assert(sizeof(mb::Settings) == sizeof(mb_settings), "settings layout");
    std::memcpy(&s, &b->set, sizeof(s));
    CUDA_TRY(ctx, cudaSetDevice(ctx->device));
    CUDA_TRY(ctx, cudaEventRecord(b->e0, ctx->stream));
    int rc = mb_launch_batch(b->d_inst, ninst, mode, &s, b->d_counter, g, b->set.precision == MB_PREC_FP32, ctx->stream);
    if (rc) return fail(ctx, MB_E_CUDA, std::string("launch failed: ") + cudaGetErrorString(cudaGetLastError()));
    b->launches++;
    CUDA_TRY(ctx, cudaEventRecord(b->e1, ctx->stream));
    CUDA_TRY(ctx, cudaEventSynchronize(b->e1));
    if (ms) CUDA_TRY(ctx, cudaEventElapsedTime(ms, b->e0, b->e1));
    return MB_OK;
}

static int fetch_batch(mb_batch* b) {
    mb_ctx* ctx = b->ctx;
    CUDA_TRY(ctx, cudaMemcpyAsync(b->h_out, b->d_out, std::max<size_t>(b->pk.out.size(), 1) * sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
    CUDA_TRY(ctx, cudaMemcpyAsync(b->h_i32, b->d_i32, std::max<size_t>(b->pk.i32.size(), 1) * sizeof(int32_t), cudaMemcpyDeviceToHost, ctx->stream));
    CUDA_TRY(ctx, cudaStreamSynchronize(ctx->stream));
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
        r->status = st[0]; r->niter = st[1]; r->nfactor_retry = st[2];
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
    s->stable = 0; s->precision = MB_PREC_FP64;
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
    mb_problem* P = const_cast<mb_problem*>(Pc);
    do_symbolic(P);
    if (vperm) for (size_t k = 0; k < P->vperm.size(); ++k) vperm[k] = P->vperm[k];
    if (nfront) *nfront = P->fr.nfront;
    for (i64 f = 0; f < P->fr.nfront && f < cap; ++f) {
        if (res0) res0[f] = P->fr.res0[f];
        if (nres) nres[f] = P->fr.nres[f];
        if (nsep) nsep[f] = (i64)P->fr.sep[f].size();
        if (parent) parent[f] = P->fr.parent[f];
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
    CUDA_TRY(s->prob->ctx, cudaMemcpy(&st, s->b->d_i32 + s->b->pk.plans[0].status, sizeof(int32_t), cudaMemcpyDeviceToHost));
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
    s[5] = (int64_t)(b->pk.out.size() * 8);
    s[6] = 0; s[7] = 0;
    return MB_OK;
}

int mb_batch_destroy(mb_batch* b) {
    if (!b) return MB_E_ARG;
    delete b;
    return MB_OK;
}

int mb_batch_solve(mb_ctx* ctx, mb_problem* const* probs, int32_t nprob, const mb_settings* settings, int32_t grid,
                   double* const* p_out, double* const* d_out, double* const* y_out, mb_result* results) {
    mb_batch* b = nullptr;
    int rc = make_batch(ctx, probs, nprob, settings, nullptr, nullptr, nullptr, &b);
    if (rc) return rc;
    std::unique_ptr<mb_batch> hold(b);
    rc = run_batch(b, mb::MODE_SOLVE, grid, nullptr);
    if (rc) return rc;
    return mb_batch_fetch(b, p_out, d_out, y_out, results);
}

}  // extern "C"
