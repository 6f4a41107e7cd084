// ============================================================================================
// ORACLE — test infrastructure only.
//
// A CPU, FP64 restatement of the interior-point hot path of Mumblebee.jl (src/IPM over
// src/BlockSparseArrays storage).  It is the parity checker for the CUDA path and the timed
// CPU baseline; nothing in the product links or calls it.  Only tests/, the smoke check and
// the CPU-baseline leg of bench.py load it.
//
// Parity status: the reference is pure Julia and ships no tests, fixtures or golden vectors,
// and Julia is not installed, so every restated function below is pinned only against the
// mathematics the reference documents (cone identities, shadow round trips, closed-form
// answers, KKT optimality certificates).  "Parity unpinned" in the sense of the build rules.
// The symbolic ordering that the reference takes from CliqueTrees (not vendored) is an input
// here (`vperm`); etree, supernodes and the multifrontal numeric factor are restated from the
// published algorithms (Liu 1990; Duff-Reid multifrontal) because CliqueTrees' source is absent.
//
// Every function cites the reference file:line it follows (paths inside the reference project).
// ============================================================================================
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <dlfcn.h>
#include <limits>
#include <algorithm>
#include <vector>
#include <chrono>

#include "oracle_cones.hpp"

using i64 = int64_t;
using i32 = int32_t;

namespace orc {

// --------------------------------------------------------------------------------------------
// Dense kernels: OpenBLAS (the scipy build in the image, `scipy_` prefixed symbols) when it is
// loaded with oracle_set_blas(); otherwise plain loops.  The reference reaches BLAS/LAPACK the
// same way through CliqueTrees' multifrontal kernels.
// --------------------------------------------------------------------------------------------
typedef void (*potrf_t)(const char*, const int*, double*, const int*, int*);
typedef void (*trsm_t)(const char*, const char*, const char*, const char*, const int*, const int*,
                       const double*, const double*, const int*, double*, const int*);
typedef void (*syrk_t)(const char*, const char*, const int*, const int*, const double*, const double*,
                       const int*, const double*, double*, const int*);
typedef void (*spotrf_t)(const char*, const int*, float*, const int*, int*);
typedef void (*strsm_t)(const char*, const char*, const char*, const char*, const int*, const int*,
                        const float*, const float*, const int*, float*, const int*);
typedef void (*ssyrk_t)(const char*, const char*, const int*, const int*, const float*, const float*,
                        const int*, const float*, float*, const int*);
typedef void (*setthr_t)(int);

static potrf_t g_dpotrf = nullptr;
static trsm_t g_dtrsm = nullptr;
static syrk_t g_dsyrk = nullptr;
static spotrf_t g_spotrf = nullptr;
static strsm_t g_strsm = nullptr;
static ssyrk_t g_ssyrk = nullptr;
static setthr_t g_setthr = nullptr;

template <class R>
static int potrf_loops(int n, R* a, int lda) {
    for (int j = 0; j < n; ++j) {
        R s = a[j + (i64)j * lda];
        for (int k = 0; k < j; ++k) s -= a[j + (i64)k * lda] * a[j + (i64)k * lda];
        if (!(s > 0)) return j + 1;
        R d = std::sqrt(s);
        a[j + (i64)j * lda] = d;
        for (int i = j + 1; i < n; ++i) {
            R t = a[i + (i64)j * lda];
            for (int k = 0; k < j; ++k) t -= a[i + (i64)k * lda] * a[j + (i64)k * lda];
            a[i + (i64)j * lda] = t / d;
        }
    }
    return 0;
}

// B (m x n) <- B * L^{-T}, L lower n x n
template <class R>
static void trsm_rlt_loops(int m, int n, const R* l, int ldl, R* b, int ldb) {
    for (int j = 0; j < n; ++j) {
        for (int k = 0; k < j; ++k) {
            R ljk = l[j + (i64)k * ldl];
            for (int i = 0; i < m; ++i) b[i + (i64)j * ldb] -= b[i + (i64)k * ldb] * ljk;
        }
        R d = l[j + (i64)j * ldl];
        for (int i = 0; i < m; ++i) b[i + (i64)j * ldb] /= d;
    }
}

// C (n x n, lower) -= A A^T, A n x k
template <class R>
static void syrk_ln_loops(int n, int k, const R* a, int lda, R* c, int ldc) {
    for (int j = 0; j < n; ++j)
        for (int p = 0; p < k; ++p) {
            R ajp = a[j + (i64)p * lda];
            for (int i = j; i < n; ++i) c[i + (i64)j * ldc] -= a[i + (i64)p * lda] * ajp;
        }
}

static int dpotrf_l(int n, double* a, int lda) {
    if (n == 0) return 0;
    if (g_dpotrf) { int info = 0; g_dpotrf("L", &n, a, &lda, &info); return info; }
    return potrf_loops(n, a, lda);
}
static int spotrf_l(int n, float* a, int lda) {
    if (n == 0) return 0;
    if (g_spotrf) { int info = 0; g_spotrf("L", &n, a, &lda, &info); return info; }
    return potrf_loops(n, a, lda);
}
static void dtrsm_rlt(int m, int n, const double* l, int ldl, double* b, int ldb) {
    if (m == 0 || n == 0) return;
    if (g_dtrsm) { double one = 1.0; g_dtrsm("R", "L", "T", "N", &m, &n, &one, l, &ldl, b, &ldb); return; }
    trsm_rlt_loops(m, n, l, ldl, b, ldb);
}
static void strsm_rlt(int m, int n, const float* l, int ldl, float* b, int ldb) {
    if (m == 0 || n == 0) return;
    if (g_strsm) { float one = 1.0f; g_strsm("R", "L", "T", "N", &m, &n, &one, l, &ldl, b, &ldb); return; }
    trsm_rlt_loops(m, n, l, ldl, b, ldb);
}
static void dsyrk_ln(int n, int k, const double* a, int lda, double* c, int ldc) {
    if (n == 0 || k == 0) return;
    if (g_dsyrk) { double al = -1.0, be = 1.0; g_dsyrk("L", "N", &n, &k, &al, a, &lda, &be, c, &ldc); return; }
    syrk_ln_loops(n, k, a, lda, c, ldc);
}
static void ssyrk_ln(int n, int k, const float* a, int lda, float* c, int ldc) {
    if (n == 0 || k == 0) return;
    if (g_ssyrk) { float al = -1.0f, be = 1.0f; g_ssyrk("L", "N", &n, &k, &al, a, &lda, &be, c, &ldc); return; }
    syrk_ln_loops(n, k, a, lda, c, ldc);
}

// --------------------------------------------------------------------------------------------
// BlockSparseMatrix, 0-based.  BlockSparseArrays/src/block_sparse_matrix.jl:10-158: vertices
// are column blocks, out-vertices row blocks, each arc a dense column-major block.
// --------------------------------------------------------------------------------------------
struct BSM {
    i64 nout = 0, nvtx = 0, narc = 0, ncol = 0, nrow = 0, nbnz = 0;
    std::vector<i64> xsrc, xcol, xrow, xblk, tgt;
    std::vector<double> val;
    i64 ncols(i64 v) const { return xcol[v + 1] - xcol[v]; }
    i64 nrows(i64 u) const { return xrow[u + 1] - xrow[u]; }
};

// y <- alpha A x + beta y  (blas/gemv.jl:321-343, :N)
static void gemvN(const BSM& A, const double* x, double* y, double alpha, double beta) {
    if (beta == 0) std::fill(y, y + A.nrow, 0.0);
    else if (beta != 1) for (i64 i = 0; i < A.nrow; ++i) y[i] *= beta;
    for (i64 v = 0; v < A.nvtx; ++v) {
        i64 c0 = A.xcol[v], nc = A.ncols(v);
        for (i64 e = A.xsrc[v]; e < A.xsrc[v + 1]; ++e) {
            i64 u = A.tgt[e], r0 = A.xrow[u], nr = A.nrows(u);
            const double* blk = A.val.data() + A.xblk[e];
            for (i64 j = 0; j < nc; ++j) {
                double xj = alpha * x[c0 + j];
                for (i64 i = 0; i < nr; ++i) y[r0 + i] += blk[i + j * nr] * xj;
            }
        }
    }
}

// y <- alpha A^T x + beta y  (blas/gemv.jl:321-343, :T)
static void gemvT(const BSM& A, const double* x, double* y, double alpha, double beta) {
    if (beta == 0) std::fill(y, y + A.ncol, 0.0);
    else if (beta != 1) for (i64 i = 0; i < A.ncol; ++i) y[i] *= beta;
    for (i64 v = 0; v < A.nvtx; ++v) {
        i64 c0 = A.xcol[v], nc = A.ncols(v);
        for (i64 j = 0; j < nc; ++j) {
            double acc = 0;
            for (i64 e = A.xsrc[v]; e < A.xsrc[v + 1]; ++e) {
                i64 u = A.tgt[e], r0 = A.xrow[u], nr = A.nrows(u);
                const double* blk = A.val.data() + A.xblk[e] + j * nr;
                for (i64 i = 0; i < nr; ++i) acc += blk[i] * x[r0 + i];
            }
            y[c0 + j] += alpha * acc;
        }
    }
}

// dot(x, A, y)  (block_sparse_matrix.jl:1094-1109)
static double bdot(const double* x, const BSM& A, const double* y) {
    double out = 0;
    for (i64 v = 0; v < A.nvtx; ++v) {
        i64 c0 = A.xcol[v], nc = A.ncols(v);
        for (i64 e = A.xsrc[v]; e < A.xsrc[v + 1]; ++e) {
            i64 u = A.tgt[e], r0 = A.xrow[u], nr = A.nrows(u);
            const double* blk = A.val.data() + A.xblk[e];
            double s = 0;
            for (i64 j = 0; j < nc; ++j) {
                double t = 0;
                for (i64 i = 0; i < nr; ++i) t += x[r0 + i] * blk[i + j * nr];
                s += t * y[c0 + j];
            }
            out += s;
        }
    }
    return out;
}

static double vnorm(const double* x, i64 n) {
    double s = 0;
    for (i64 i = 0; i < n; ++i) s += x[i] * x[i];
    return std::sqrt(s);
}
static double vdot(const double* x, const double* y, i64 n) {
    double s = 0;
    for (i64 i = 0; i < n; ++i) s += x[i] * y[i];
    return s;
}
// norm(A) over stored values  (block_sparse_matrix.jl:1084-1092)
static double bnorm(const BSM& A) { return vnorm(A.val.data(), A.nbnz); }

// selectvtxs(A, sel)  (block_sparse_matrix.jl:1111-1169)
static BSM selectvtxs(const BSM& A, const std::vector<i64>& sel) {
    BSM B;
    B.nout = A.nout; B.nrow = A.nrow; B.xrow = A.xrow;
    B.nvtx = (i64)sel.size();
    B.xcol.assign(B.nvtx + 1, 0); B.xsrc.assign(B.nvtx + 1, 0);
    i64 c = 0, ee = 0, bb = 0;
    for (i64 v = 0; v < B.nvtx; ++v) {
        i64 av = sel[v];
        B.xcol[v] = c; B.xsrc[v] = ee; c += A.ncols(av);
        for (i64 e = A.xsrc[av]; e < A.xsrc[av + 1]; ++e) {
            B.tgt.push_back(A.tgt[e]); B.xblk.push_back(bb); ++ee;
            for (i64 b = A.xblk[e]; b < A.xblk[e + 1]; ++b) { B.val.push_back(A.val[b]); ++bb; }
        }
    }
    B.xcol[B.nvtx] = c; B.xsrc[B.nvtx] = ee; B.xblk.push_back(bb);
    B.ncol = c; B.narc = ee; B.nbnz = bb;
    return B;
}

// halfselectvtxs(A, sel) with transposed blocks  (block_sparse_matrix.jl:787-874).  Out-vertices
// of the result are the selected vertices of A; vertices are A's out-vertices; arcs come out
// sorted by target.
static BSM halfselectvtxs(const BSM& A, const std::vector<i64>& sel) {
    BSM R;
    R.nout = (i64)sel.size(); R.nvtx = A.nout; R.ncol = A.nrow;
    R.nrow = 0; R.narc = 0; R.nbnz = 0;
    for (i64 av : sel) {
        R.nrow += A.ncols(av);
        for (i64 e = A.xsrc[av]; e < A.xsrc[av + 1]; ++e) { R.narc++; R.nbnz += A.xblk[e + 1] - A.xblk[e]; }
    }
    std::vector<i64> cnt(R.nvtx + 1, 0), bcnt(R.nvtx + 1, 0);
    for (i64 au = 0; au < R.nout; ++au) {
        i64 bv = sel[au];
        for (i64 e = A.xsrc[bv]; e < A.xsrc[bv + 1]; ++e) { cnt[A.tgt[e] + 1]++; bcnt[A.tgt[e] + 1] += A.xblk[e + 1] - A.xblk[e]; }
    }
    for (i64 v = 0; v < R.nvtx; ++v) { cnt[v + 1] += cnt[v]; bcnt[v + 1] += bcnt[v]; }
    R.xsrc = cnt; R.tgt.assign(R.narc, 0); R.xblk.assign(R.narc + 1, 0); R.val.assign(R.nbnz, 0);
    std::vector<i64> pe(cnt.begin(), cnt.end() - 1), pb(bcnt.begin(), bcnt.end() - 1);
    for (i64 au = 0; au < R.nout; ++au) {
        i64 bv = sel[au];
        i64 nc = A.ncols(bv);
        for (i64 e = A.xsrc[bv]; e < A.xsrc[bv + 1]; ++e) {
            i64 bu = A.tgt[e], nr = A.nrows(bu);
            i64 ae = pe[bu]++, ab = pb[bu];
            R.tgt[ae] = au; R.xblk[ae] = ab;
            const double* blk = A.val.data() + A.xblk[e];
            // transposed block: (nc x nr) column-major  <- blk (nr x nc)
            for (i64 i = 0; i < nr; ++i)
                for (i64 j = 0; j < nc; ++j) R.val[ab + j + i * nc] = blk[i + j * nr];
            pb[bu] += nr * nc;
        }
    }
    R.xblk[R.narc] = R.nbnz;
    R.xrow.assign(R.nout + 1, 0);
    i64 ar = 0;
    for (i64 au = 0; au < R.nout; ++au) { R.xrow[au] = ar; ar += A.ncols(sel[au]); }
    R.xrow[R.nout] = R.nrow;
    R.xcol = A.xrow;
    return R;
}

// C = A^T A pattern and values for the Uzawa factor  (uzawa.jl:29 `B' * B`;
// block_sparse_matrix.jl:1171-1256 matprod_dest; blas/gemm.jl:48-82)
static BSM gramian(const BSM& B) {
    // transpose of B as block-CSR: for each out-vertex u, the arcs (u, v)
    std::vector<std::vector<std::pair<i64, i64>>> rowarcs(B.nout);
    for (i64 v = 0; v < B.nvtx; ++v)
        for (i64 e = B.xsrc[v]; e < B.xsrc[v + 1]; ++e) rowarcs[B.tgt[e]].push_back({v, e});
    BSM C;
    C.nout = C.nvtx = B.nvtx; C.ncol = C.nrow = B.ncol;
    C.xcol = B.xcol; C.xrow = B.xcol;
    C.xsrc.assign(C.nvtx + 1, 0);
    std::vector<i64> marker(C.nout, -1);
    for (i64 v = 0; v < B.nvtx; ++v) {
        C.xsrc[v] = (i64)C.tgt.size();
        i64 s0 = (i64)C.tgt.size();
        for (i64 e = B.xsrc[v]; e < B.xsrc[v + 1]; ++e)
            for (auto& ua : rowarcs[B.tgt[e]]) {
                if (marker[ua.first] != v) { marker[ua.first] = v; C.tgt.push_back(ua.first); }
            }
        std::sort(C.tgt.begin() + s0, C.tgt.end());
    }
    C.narc = (i64)C.tgt.size(); C.xsrc[C.nvtx] = C.narc;
    C.xblk.assign(C.narc + 1, 0);
    i64 b = 0;
    for (i64 v = 0; v < C.nvtx; ++v)
        for (i64 e = C.xsrc[v]; e < C.xsrc[v + 1]; ++e) { C.xblk[e] = b; b += C.ncols(C.tgt[e]) * C.ncols(v); }
    C.xblk[C.narc] = b; C.nbnz = b; C.val.assign(b, 0.0);
    // values: C(w, v) += B(u, w)^T B(u, v)
    std::vector<i64> pos(C.nout, -1);
    for (i64 v = 0; v < C.nvtx; ++v) {
        for (i64 e = C.xsrc[v]; e < C.xsrc[v + 1]; ++e) pos[C.tgt[e]] = e;
        i64 ncv = C.ncols(v);
        for (i64 e = B.xsrc[v]; e < B.xsrc[v + 1]; ++e) {
            i64 u = B.tgt[e], nr = B.nrows(u);
            const double* bv = B.val.data() + B.xblk[e];
            for (auto& ua : rowarcs[u]) {
                i64 w = ua.first;
                const double* bw = B.val.data() + B.xblk[ua.second];
                i64 ncw = C.ncols(w);
                double* cb = C.val.data() + C.xblk[pos[w]];
                for (i64 j = 0; j < ncv; ++j)
                    for (i64 i = 0; i < ncw; ++i) {
                        double s = 0;
                        for (i64 k = 0; k < nr; ++k) s += bw[k + i * nr] * bv[k + j * nr];
                        cb[i + j * ncw] += s;
                    }
            }
        }
    }
    return C;
}

// --------------------------------------------------------------------------------------------
// Chordal symbolic analysis over vertices (restated from the published algorithms; the
// reference's CliqueTrees.symbolic is absent).  Elimination tree by Liu's path-compressed
// ancestor algorithm, postorder, vertex row structures, fundamental supernodes.
// --------------------------------------------------------------------------------------------
struct Symbolic {
    i64 nfront = 0;
    std::vector<i64> postperm;       // vertex order after postordering (indices into input order)
    std::vector<i64> fvtx;           // front f owns vertices fvtx[f] .. fvtx[f+1]-1 (postordered)
    std::vector<i64> res0, nres;     // scalar column range of each front
    std::vector<std::vector<i64>> sep;  // scalar separator rows, ascending
    std::vector<i64> parent;         // front parent (-1 root)
    std::vector<std::vector<i64>> rel;  // position of sep[f][k] in parent's row list
    std::vector<i64> fptr;           // offset of front f's (nf x nf) storage
    i64 fsize = 0;
    std::vector<i64> colfront;       // scalar column -> front
};

// adjacency over vertices: pattern of Q union B^T B (IPM/src/utils.jl:135-145 weightedgraph)
static std::vector<std::vector<i64>> vertexgraph(const BSM& Q, const BSM& L) {
    i64 nv = L.nvtx;
    std::vector<std::vector<i64>> adj(nv);
    auto add = [&](const BSM& A) {
        for (i64 v = 0; v < A.nvtx; ++v)
            for (i64 e = A.xsrc[v]; e < A.xsrc[v + 1]; ++e) {
                i64 u = A.tgt[e];
                if (u != v) { adj[v].push_back(u); adj[u].push_back(v); }
            }
    };
    add(Q); add(L);
    for (auto& a : adj) { std::sort(a.begin(), a.end()); a.erase(std::unique(a.begin(), a.end()), a.end()); }
    return adj;
}

static void etree(const std::vector<std::vector<i64>>& adj, std::vector<i64>& par) {
    i64 n = (i64)adj.size();
    par.assign(n, -1);
    std::vector<i64> anc(n, -1);
    for (i64 j = 0; j < n; ++j)
        for (i64 i : adj[j]) {
            if (i >= j) continue;
            i64 r = i;
            while (anc[r] != -1 && anc[r] != j) { i64 t = anc[r]; anc[r] = j; r = t; }
            if (anc[r] == -1) { anc[r] = j; par[r] = j; }
        }
}

// vertex-level analysis on a symmetric adjacency already permuted into elimination order.
static Symbolic analyze(const std::vector<std::vector<i64>>& adj0, const std::vector<i64>& w0) {
    i64 n = (i64)adj0.size();
    std::vector<i64> par0;
    etree(adj0, par0);
    // postorder: DFS from roots in increasing order, children in increasing order
    std::vector<std::vector<i64>> ch(n);
    std::vector<i64> roots;
    for (i64 v = 0; v < n; ++v) { if (par0[v] < 0) roots.push_back(v); else ch[par0[v]].push_back(v); }
    // children are visited in increasing size of their row structure (ties by index), so the child
    // with the largest structure, the one a chain of supernodes continues through, comes last and
    // can merge with its parent; any postorder of the etree gives the same factor
    {
        std::vector<i64> ssz0(n, 0), mk(n, -1);
        std::vector<std::vector<i64>> s0(n);
        for (i64 v = 0; v < n; ++v) {
            for (i64 u : adj0[v]) if (u > v && mk[u] != v) { mk[u] = v; s0[v].push_back(u); }
            for (i64 c : ch[v]) for (i64 u : s0[c]) if (u > v && mk[u] != v) { mk[u] = v; s0[v].push_back(u); }
            ssz0[v] = (i64)s0[v].size();
        }
        for (i64 v = 0; v < n; ++v)
            std::stable_sort(ch[v].begin(), ch[v].end(), [&](i64 a, i64 b) { return ssz0[a] < ssz0[b]; });
    }
    std::vector<i64> post; post.reserve(n);
    std::vector<std::pair<i64, size_t>> st;
    for (i64 r : roots) {
        st.push_back({r, 0});
        while (!st.empty()) {
            auto& t = st.back();
            if (t.second < ch[t.first].size()) { i64 c = ch[t.first][t.second++]; st.push_back({c, 0}); }
            else { post.push_back(t.first); st.pop_back(); }
        }
    }
    std::vector<i64> inv(n);
    for (i64 k = 0; k < n; ++k) inv[post[k]] = k;
    std::vector<std::vector<i64>> adj(n);
    std::vector<i64> w(n), par(n);
    for (i64 k = 0; k < n; ++k) {
        i64 v = post[k];
        w[k] = w0[v];
        par[k] = par0[v] < 0 ? -1 : inv[par0[v]];
        adj[k].reserve(adj0[v].size());
        for (i64 u : adj0[v]) adj[k].push_back(inv[u]);   // order is irrelevant below (mark arrays)
    }
    // vertex row structure struct(v) (vertices > v), by merging children
    std::vector<std::vector<i64>> sv(n);
    std::vector<std::vector<i64>> kids(n);
    for (i64 v = 0; v < n; ++v) if (par[v] >= 0) kids[par[v]].push_back(v);
    std::vector<i64> mark(n, -1);
    for (i64 v = 0; v < n; ++v) {
        std::vector<i64>& s = sv[v];
        for (i64 u : adj[v]) if (u > v && mark[u] != v) { mark[u] = v; s.push_back(u); }
        for (i64 c : kids[v])
            for (i64 u : sv[c]) if (u > v && mark[u] != v) { mark[u] = v; s.push_back(u); }
        std::sort(s.begin(), s.end());
    }
    // relaxed supernodes: v joins the front of its child v-1 (last child in postorder) when the
    // explicit zeros added to the front's columns stay within 5% of the merged front's lower
    // entries (CliqueTrees' own partition is not available here; the numeric factor does not
    // depend on the partition, only the storage does)
    Symbolic S;
    S.postperm = post;
    std::vector<i64> front(n, -1), ssw(n, 0);
    for (i64 v = 0; v < n; ++v) for (i64 u : sv[v]) ssw[v] += w[u];
    i64 fcols = 0, fzeros = 0;
    for (i64 v = 0; v < n; ++v) {
        bool merge = false;
        if (v > 0 && par[v - 1] == v) {
            const i64 add = fcols * (w[v] + ssw[v] - ssw[v - 1]);
            const i64 cols = fcols + w[v], nfm = cols + ssw[v];
            const double entries = (double)cols * (double)nfm - 0.5 * (double)cols * (double)(cols - 1);
            merge = add == 0 || (double)(fzeros + add) <= 0.05 * entries;
            if (merge) { fzeros += add; fcols = cols; }
        }
        if (merge) front[v] = front[v - 1];
        else { front[v] = S.nfront++; S.fvtx.push_back(v); fcols = w[v]; fzeros = 0; }
    }
    S.fvtx.push_back(n);
    // scalar columns of each vertex
    std::vector<i64> vcol(n + 1, 0);
    for (i64 v = 0; v < n; ++v) vcol[v + 1] = vcol[v] + w[v];
    i64 ncol = vcol[n];
    S.res0.resize(S.nfront); S.nres.resize(S.nfront); S.sep.resize(S.nfront); S.parent.assign(S.nfront, -1);
    S.colfront.assign(ncol, 0);
    for (i64 f = 0; f < S.nfront; ++f) {
        i64 v0 = S.fvtx[f], v1 = S.fvtx[f + 1];
        S.res0[f] = vcol[v0]; S.nres[f] = vcol[v1] - vcol[v0];
        for (i64 j = vcol[v0]; j < vcol[v1]; ++j) S.colfront[j] = f;
        for (i64 u : sv[v1 - 1])
            for (i64 j = vcol[u]; j < vcol[u + 1]; ++j) S.sep[f].push_back(j);
        i64 pv = par[v1 - 1];
        S.parent[f] = pv < 0 ? -1 : front[pv];
    }
    S.rel.resize(S.nfront);
    std::vector<i64> posmap(ncol, -1);
    for (i64 f = 0; f < S.nfront; ++f) {
        i64 p = S.parent[f];
        if (p < 0) continue;
        for (i64 k = 0; k < S.nres[p]; ++k) posmap[S.res0[p] + k] = k;
        for (size_t k = 0; k < S.sep[p].size(); ++k) posmap[S.sep[p][k]] = S.nres[p] + (i64)k;
        for (i64 r : S.sep[f]) S.rel[f].push_back(posmap[r]);
    }
    S.fptr.resize(S.nfront + 1);
    i64 off = 0;
    for (i64 f = 0; f < S.nfront; ++f) {
        S.fptr[f] = off;
        i64 nf = S.nres[f] + (i64)S.sep[f].size();
        off += nf * nf;
    }
    S.fptr[S.nfront] = off; S.fsize = off;
    return S;
}

// --------------------------------------------------------------------------------------------
// Multifrontal numeric factor.  F F^T = delta H + B^T B (+ rho I).  Fronts are full
// (nres+nsep)^2 column-major squares; the leading nres columns hold the factor, the trailing
// nsep x nsep block is the update matrix extend-added into the parent.
// --------------------------------------------------------------------------------------------
struct Factor {
    const Symbolic* S = nullptr;
    std::vector<double> val;   // FP64 fronts
    std::vector<float> fval;   // FP32 fronts (mixed-precision simulation)
    bool fp32 = false;
};

// Scatter alpha*A (lower part, by vertex blocks) into the fronts; chordal.jl:1-80
static void scatter_add(Factor& F, const BSM& A, double alpha) {
    const Symbolic& S = *F.S;
    for (i64 v = 0; v < A.nvtx; ++v) {
        i64 c0 = A.xcol[v], nc = A.ncols(v);
        if (nc == 0) continue;
        i64 f = S.colfront[c0];
        i64 nres = S.nres[f], nsep = (i64)S.sep[f].size(), nf = nres + nsep, r0 = S.res0[f];
        double* M = F.val.data() + S.fptr[f];
        for (i64 e = A.xsrc[v]; e < A.xsrc[v + 1]; ++e) {
            i64 u = A.tgt[e];
            if (u < v) continue;
            i64 ur0 = A.xrow[u], nr = A.nrows(u);
            const double* blk = A.val.data() + A.xblk[e];
            i64 rowpos;
            if (ur0 >= r0 && ur0 < r0 + nres) rowpos = ur0 - r0;
            else {
                auto it = std::lower_bound(S.sep[f].begin(), S.sep[f].end(), ur0);
                rowpos = nres + (i64)(it - S.sep[f].begin());
            }
            for (i64 j = 0; j < nc; ++j) {
                i64 fj = c0 - r0 + j;
                for (i64 i = 0; i < nr; ++i) M[(rowpos + i) + fj * nf] += alpha * blk[i + j * nr];
            }
        }
    }
}

static double factor_lower_norm(const Factor& F) {
    const Symbolic& S = *F.S;
    double s = 0;
    for (i64 f = 0; f < S.nfront; ++f) {
        i64 nres = S.nres[f], nf = nres + (i64)S.sep[f].size();
        const double* M = F.val.data() + S.fptr[f];
        for (i64 j = 0; j < nres; ++j)
            for (i64 i = j; i < nf; ++i) s += M[i + j * nf] * M[i + j * nf];
    }
    return std::sqrt(s);
}

template <class R>
static int factor_fronts(const Symbolic& S, R* val,
                         int (*potrf)(int, R*, int), void (*trsm)(int, int, const R*, int, R*, int),
                         void (*syrk)(int, int, const R*, int, R*, int)) {
    for (i64 f = 0; f < S.nfront; ++f) {
        i64 nres = S.nres[f], nsep = (i64)S.sep[f].size(), nf = nres + nsep;
        R* M = val + S.fptr[f];
        int info = potrf((int)nres, M, (int)nf);
        if (info != 0) return (int)(S.res0[f] + info);
        trsm((int)nsep, (int)nres, M, (int)nf, M + nres, (int)nf);
        syrk((int)nsep, (int)nres, M + nres, (int)nf, M + nres + nres * nf, (int)nf);
        i64 p = S.parent[f];
        if (p >= 0 && nsep > 0) {
            i64 np = S.nres[p] + (i64)S.sep[p].size();
            R* P = val + S.fptr[p];
            const std::vector<i64>& rel = S.rel[f];
            for (i64 j = 0; j < nsep; ++j)
                for (i64 i = j; i < nsep; ++i) {
                    i64 a = rel[i], b = rel[j];
                    R x = M[(nres + i) + (nres + j) * nf];
                    if (a >= b) P[a + b * np] += x; else P[b + a * np] += x;
                }
        }
    }
    return 0;
}

static int numeric_factor(Factor& F) {
    if (!F.fp32) return factor_fronts<double>(*F.S, F.val.data(), dpotrf_l, dtrsm_rlt, dsyrk_ln);
    F.fval.resize(F.val.size());
    for (size_t i = 0; i < F.val.size(); ++i) F.fval[i] = (float)F.val[i];
    return factor_fronts<float>(*F.S, F.fval.data(), spotrf_l, strsm_rlt, ssyrk_ln);
}

// forward solve L x = b in place (L!)
template <class R>
static void lsolve(const Symbolic& S, const R* val, double* x) {
    std::vector<double> t;
    for (i64 f = 0; f < S.nfront; ++f) {
        i64 nres = S.nres[f], nsep = (i64)S.sep[f].size(), nf = nres + nsep, r0 = S.res0[f];
        const R* M = val + S.fptr[f];
        for (i64 j = 0; j < nres; ++j) {
            double xj = x[r0 + j] / (double)M[j + j * nf];
            x[r0 + j] = xj;
            for (i64 i = j + 1; i < nres; ++i) x[r0 + i] -= (double)M[i + j * nf] * xj;
        }
        for (i64 k = 0; k < nsep; ++k) {
            double s = 0;
            for (i64 j = 0; j < nres; ++j) s += (double)M[nres + k + j * nf] * x[r0 + j];
            x[S.sep[f][k]] -= s;
        }
    }
}

// backward solve L^T x = b in place (U!)
template <class R>
static void usolve(const Symbolic& S, const R* val, double* x) {
    for (i64 f = S.nfront - 1; f >= 0; --f) {
        i64 nres = S.nres[f], nsep = (i64)S.sep[f].size(), nf = nres + nsep, r0 = S.res0[f];
        const R* M = val + S.fptr[f];
        for (i64 j = 0; j < nres; ++j) {
            double s = 0;
            for (i64 k = 0; k < nsep; ++k) s += (double)M[nres + k + j * nf] * x[S.sep[f][k]];
            x[r0 + j] -= s;
        }
        for (i64 j = nres - 1; j >= 0; --j) {
            double s = x[r0 + j];
            for (i64 i = j + 1; i < nres; ++i) s -= (double)M[i + j * nf] * x[r0 + i];
            x[r0 + j] = s / (double)M[j + j * nf];
        }
    }
}

static void Lsolve(const Factor& F, double* x) {
    if (F.fp32) lsolve<float>(*F.S, F.fval.data(), x); else lsolve<double>(*F.S, F.val.data(), x);
}
static void Usolve(const Factor& F, double* x) {
    if (F.fp32) usolve<float>(*F.S, F.fval.data(), x); else usolve<double>(*F.S, F.val.data(), x);
}

// --------------------------------------------------------------------------------------------
// Settings, statuses, history  (settings/ipm.jl:1-18; ipm/ipm.jl:1; kkt.jl:1; cg.jl:1-6)
// --------------------------------------------------------------------------------------------
enum IPMStatus { CONTINUE = 0, OPTIMAL, NEAR_OPTIMAL, STALLED, NUMERICAL_FAILURE, ITERATION_LIMIT,
                 PRIMAL_INFEASIBLE, DUAL_INFEASIBLE, ILL_POSED, NEAR_PRIMAL_INFEASIBLE,
                 NEAR_DUAL_INFEASIBLE, NEAR_ILL_POSED };
enum KKTStatus { KKT_CONTINUE = 0, KKT_SOLVED, KKT_STAGNATED, KKT_ITMAX, KKT_NUMERICAL_FAILURE, KKT_IRMAX };
enum CGStatus { CG_CONTINUE = 0, CG_SOLVED, CG_NUMERICAL_FAILURE, CG_ITMAX };

}  // namespace orc

extern "C" {
// Layout shared with include/mumblebee_gpu.h (mb_settings); checked by the tests.
typedef struct {
    int32_t verbose;
    int32_t max_iter;
    int32_t scale_max_iter;
    int32_t refine_max_iter;
    int32_t newton_max_iter;
    int32_t stable;
    int32_t precision;      // 0 = FP64 factor, 1 = FP32 factor (mixed)
    int32_t large;
    double step_frac;
    double feas_tol;
    double gap_tol;
    double near_factor;
    double stall_tol;
    double refine_stall_tol;
    double aug_tol;
    double infeas_abs;
    double infeas_rel;
} ob_settings;

typedef struct {
    int64_t nout, nvtx, narc, ncol, nrow, nbnz;
    const int64_t* xsrc;
    const int64_t* xcol;
    const int64_t* xrow;
    const int64_t* xblk;
    const int64_t* tgt;
    const double* val;
} ob_bsm;   // 1-based index arrays, as BlockSparseMatrix stores them

// history row, the 17 fields of IPMHistoryRow (history/ipm.jl:1-4), all as doubles
typedef struct {
    double pres, dres, pobj, dobj, step;
    double piter, ppass, pstat, citer, cpass, cstat;
    double dmin, dmax, rho, delta, mu, chi;
} ob_row;
}

namespace orc {

static BSM from_c(const ob_bsm* A) {
    BSM B;
    B.nout = A->nout; B.nvtx = A->nvtx; B.narc = A->narc; B.ncol = A->ncol; B.nrow = A->nrow; B.nbnz = A->nbnz;
    B.xsrc.resize(B.nvtx + 1); B.xcol.resize(B.nvtx + 1); B.xrow.resize(B.nout + 1);
    B.xblk.resize(B.narc + 1); B.tgt.resize(B.narc); B.val.assign(A->val, A->val + B.nbnz);
    for (i64 i = 0; i <= B.nvtx; ++i) { B.xsrc[i] = A->xsrc[i] - 1; B.xcol[i] = A->xcol[i] - 1; }
    for (i64 i = 0; i <= B.nout; ++i) B.xrow[i] = A->xrow[i] - 1;
    for (i64 i = 0; i <= B.narc; ++i) B.xblk[i] = A->xblk[i] - 1;
    for (i64 i = 0; i < B.narc; ++i) B.tgt[i] = A->tgt[i] - 1;
    return B;
}

struct Timers { double scale = 0, initkkt = 0, predictor = 0, corrector = 0, maxsteps = 0, solve = 0; };
using clk = std::chrono::steady_clock;
static double secs(clk::time_point a) { return std::chrono::duration<double>(clk::now() - a).count(); }

struct Solver {
    ob_settings set;
    BSM Q, H, B, L;
    std::vector<double> f, g, p, d, y;
    std::vector<i32> K;            // cone kind per (permuted) vertex
    std::vector<double> Kp;        // cone parameter per vertex
    std::vector<i64> P1, P2;       // user index of solver row / column
    std::vector<double> pscl, yscl;
    Symbolic S;
    Factor F;
    std::vector<i64> cxblk;        // cache offsets
    std::vector<double> cache;
    std::vector<double> cwork;     // cone workspace
    // workspace (workspace/ipm.jl:1-54)
    std::vector<double> Df, Dg, wf, Qp, Dpa, Dya, Dda, Dp, Dy, Dd, step, spsd;
    std::vector<char> flag;
    // Uzawa workspace (uzawa.jl:3-30; cg.jl:8-20)
    std::vector<double> uhist, df, dg, dx, dy, cgp, cgw, cghist;
    double delta = 0;
    std::vector<ob_row> hist;
    i64 nu = 0;
    double mut = 0;
    double nf = 0, ng = 0, sg = 0, sf = 0, nB = 0;
    i64 n = 0, m = 0;
    Timers tm;
    i64 nfactor_retry = 0;
    i64 nfallback = 0;      // iterations redone with the FP64 factor (precision 2)
    bool switched = false;  // moved to the FP64 factor after a solve-heavy FP32 iteration (precision 2)
    i64 stall0 = 0;         // history rows before the last precision switch (the stall window starts there)
    bool stallhit = false;  // the last step_ ended on the stall test
    i64 nfp32 = 0;          // iterations accepted with the FP32 factor
};

// --------------------------------------------------------------------------------------------
// cone fan-out  (cone.jl:146-553)
// --------------------------------------------------------------------------------------------
static bool scale_all(Solver& s, double& spsd_sum) {
    bool ok = true; spsd_sum = 0;
    for (i64 v = 0; v < s.B.nvtx; ++v) {
        i64 c0 = s.B.xcol[v], nc = s.B.ncols(v);
        i32 k = s.K[v];
        double sp = 0; bool fl = true;
        if (k != CONE_FREE) {
            // locate the diagonal block of H and Q (cone.jl:146-174)
            i64 ed = -1;
            for (i64 e = s.H.xsrc[v]; e < s.H.xsrc[v + 1]; ++e) if (s.H.tgt[e] == v) { ed = e; break; }
            if (ed < 0) { fprintf(stderr, "oracle: missing diagonal block for vertex %ld\n", (long)v); return false; }
            double* Hv = s.H.val.data() + s.H.xblk[ed];
            const double* Qv = s.Q.val.data() + s.Q.xblk[ed];
            std::copy(Qv, Qv + nc * nc, Hv);
            fl = cone_scale(k, s.Kp[v], nc, Hv, s.p.data() + c0, s.d.data() + c0,
                            s.cache.data() + s.cxblk[v], s.cwork.data(), &sp);
        }
        s.flag[v] = fl; s.spsd[v] = sp;
    }
    for (i64 v = 0; v < s.B.nvtx; ++v) { ok = ok && s.flag[v]; spsd_sum += s.spsd[v]; }
    return ok;
}

static void initcorrector(Solver& s, double* fr, const double* Dp, const double* Dd, double sm) {
    for (i64 v = 0; v < s.B.nvtx; ++v) {
        i64 c0 = s.B.xcol[v], nc = s.B.ncols(v);
        cone_corr(s.K[v], s.Kp[v], nc, fr + c0, s.p.data() + c0, s.d.data() + c0, Dp + c0, Dd + c0, sm,
                  s.cache.data() + s.cxblk[v], s.cwork.data());
    }
}

static void initpredictor(Solver& s, double* fr, double sm) {
    for (i64 v = 0; v < s.B.nvtx; ++v) {
        i64 c0 = s.B.xcol[v], nc = s.B.ncols(v);
        cone_corr0(s.K[v], s.Kp[v], nc, fr + c0, s.p.data() + c0, s.d.data() + c0, sm,
                   s.cache.data() + s.cxblk[v], s.cwork.data());
    }
}

static double maxsteps(Solver& s, const double* Dp, const double* Dd, double step_frac) {
    double mn = std::numeric_limits<double>::infinity();
    for (i64 v = 0; v < s.B.nvtx; ++v) {
        i64 c0 = s.B.xcol[v], nc = s.B.ncols(v);
        double tp = 1, td = 1;
        cone_maxsteps(s.K[v], s.Kp[v], nc, s.p.data() + c0, Dp + c0, s.d.data() + c0, Dd + c0,
                      s.cache.data() + s.cxblk[v], s.cwork.data(), &tp, &td);
        if (s.K[v] != CONE_FREE) { tp *= step_frac; td *= step_frac; }
        s.step[v] = std::min(tp, td);
        mn = std::min(mn, s.step[v]);
    }
    if (s.B.nvtx == 0) mn = 1;
    return mn;
}

static void zerofree(Solver& s, double* x) {
    for (i64 v = 0; v < s.B.nvtx; ++v)
        if (s.K[v] == CONE_FREE) std::fill(x + s.B.xcol[v], x + s.B.xcol[v + 1], 0.0);
}

// --------------------------------------------------------------------------------------------
// KKT: mulkkt!, initkkt!, cg!, solvekkt!, kktwindow  (kkt.jl:9-21; uzawa.jl:73-115,199-227,
// 319-507; cg.jl:69-167)
// --------------------------------------------------------------------------------------------
static void mulkkt(const Solver& s, double* u, double* v, const BSM& A, const double* x, const double* y) {
    gemvN(A, x, u, 1, 0);
    gemvT(s.B, y, u, -1, 1);
    gemvN(s.B, x, v, 1, 0);
}

// StableUzawaSolver's initkkt! (uzawa.jl:117-163; cholblockdiag! utils.jl:186-200): F Fᵀ = δH + BᵀB
// without forming BᵀB.  The reference factors each nonzero diagonal block of H (failing when one is
// not positive definite), scales by √δ and updates by the rows of B (CliqueTrees lowrankupdate!,
// absent here).  Restated as multifrontal Householder QR: front f stacks √δ U_v (U_vᵀU_v = H_vv) for
// its vertices, the rows of B whose first nonzero column lies in f, and each child's R triangle over
// its separator; R of that stack satisfies RᵀR = WᵀW, its first nres rows (signed to a positive
// diagonal) are the factor's columns and the trailing triangle passes to the parent.  In exact
// arithmetic this is the unique Cholesky factor the rank-m update produces.  Returns 0, the 1-based
// column of a zero pivot, or -1 for a diagonal block of H that is not positive definite.
static int stable_factor(Solver& s, double delta) {
    const Symbolic& S = s.S;
    const BSM& B = s.B;
    const BSM& H = s.H;
    const double sd = std::sqrt(delta);
    // rows of B: nonzeros in ascending column order, assigned to the front of the first column
    std::vector<std::vector<std::pair<i64, double>>> brow(B.nrow);
    for (i64 v = 0; v < B.nvtx; ++v)
        for (i64 jl = 0; jl < B.ncols(v); ++jl)
            for (i64 e = B.xsrc[v]; e < B.xsrc[v + 1]; ++e) {
                i64 u = B.tgt[e], nr = B.nrows(u);
                const double* blk = B.val.data() + B.xblk[e] + jl * nr;
                for (i64 il = 0; il < nr; ++il)
                    if (blk[il] != 0) brow[B.xrow[u] + il].push_back({B.xcol[v] + jl, blk[il]});
            }
    std::vector<std::vector<i64>> frows(S.nfront), fch(S.nfront);
    for (i64 i = 0; i < B.nrow; ++i) {
        if (brow[i].empty()) continue;
        std::sort(brow[i].begin(), brow[i].end());
        frows[S.colfront[brow[i][0].first]].push_back(i);
    }
    for (i64 f = 0; f < S.nfront; ++f) if (S.parent[f] >= 0) fch[S.parent[f]].push_back(f);
    std::vector<double> W;
    for (i64 f = 0; f < S.nfront; ++f) {
        const i64 nres = S.nres[f], nsep = (i64)S.sep[f].size(), nf = nres + nsep, r0 = S.res0[f];
        i64 rows = nres + (i64)frows[f].size();
        for (i64 c : fch[f]) rows += (i64)S.sep[c].size();
        const i64 ld = rows;
        W.assign((size_t)(ld * nf), 0.0);
        auto w = [&](i64 i, i64 j) -> double& { return W[(size_t)(i + j * ld)]; };
        auto pos = [&](i64 col) -> i64 {
            if (col >= r0 && col < r0 + nres) return col - r0;
            auto it = std::lower_bound(S.sep[f].begin(), S.sep[f].end(), col);
            return nres + (i64)(it - S.sep[f].begin());
        };
        for (i64 v = S.fvtx[f]; v < S.fvtx[f + 1]; ++v) {
            const i64 c0 = B.xcol[v] - r0, nc = B.ncols(v);
            const double* h = nullptr;
            for (i64 e = H.xsrc[v]; e < H.xsrc[v + 1]; ++e) if (H.tgt[e] == v) h = H.val.data() + H.xblk[e];
            if (!h) continue;
            bool nz = false;
            for (i64 j = 0; j < nc; ++j) for (i64 i = j; i < nc; ++i) nz |= h[i + j * nc] != 0.0;
            if (!nz) continue;
            for (i64 j = 0; j < nc; ++j) for (i64 i = 0; i <= j; ++i) w(c0 + i, c0 + j) = h[j + i * nc];
            for (i64 j = 0; j < nc; ++j) {   // upper Cholesky in place: UᵀU = H_vv
                const double dd = w(c0 + j, c0 + j);
                if (!(dd > 0.0)) return -1;
                const double u = std::sqrt(dd), ru = 1.0 / u;
                bool nzr = false;
                for (i64 k = j + 1; k < nc; ++k) { w(c0 + j, c0 + k) *= ru; nzr |= w(c0 + j, c0 + k) != 0.0; }
                w(c0 + j, c0 + j) = u;
                if (!nzr) continue;   // an empty row updates nothing (a diagonal block)
                for (i64 k = j + 1; k < nc; ++k)
                    for (i64 i = j + 1; i <= k; ++i) w(c0 + i, c0 + k) -= w(c0 + j, c0 + i) * w(c0 + j, c0 + k);
            }
            for (i64 j = 0; j < nc; ++j) for (i64 i = 0; i <= j; ++i) w(c0 + i, c0 + j) *= sd;
        }
        i64 rc = nres;
        for (i64 i : frows[f]) {
            for (const auto& e : brow[i]) w(rc, pos(e.first)) = e.second;
            ++rc;
        }
        for (i64 c : fch[f]) {
            const i64 cres = S.nres[c], cs = (i64)S.sep[c].size(), cn = cres + cs;
            const double* Mc = s.F.val.data() + S.fptr[c];
            for (i64 j = 0; j < cs; ++j)
                for (i64 r = 0; r <= j; ++r) w(rc + r, S.rel[c][j]) = Mc[(cres + r) + (cres + j) * cn];
            rc += cs;
        }
        if (rows < nres) return (int)(r0 + rows + 1);
        const i64 jmax = std::min(rows, nf);
        // Householder: v = (a − β, w[j+1..]), β = −sign(a)‖w[j..]‖.  The vertex rows form an upper
        // triangle that no reflector fills, so v lives on row j and rows [lo, rows), lo = max(j + 1, nres).
        for (i64 j = 0; j < jmax; ++j) {
            const double a = w(j, j);
            const i64 lo = std::max(j + 1, nres);
            double ss = 0.0;
            for (i64 i = lo; i < rows; ++i) ss += w(i, j) * w(i, j);
            double beta = a;
            if (ss > 0.0) {
                const double nrm = std::sqrt(a * a + ss);
                beta = a > 0.0 ? -nrm : nrm;
                const double cf = 1.0 / (beta * (beta - a));
                w(j, j) = a - beta;
                for (i64 k = j + 1; k < nf; ++k) {
                    double dt = w(j, j) * w(j, k);
                    for (i64 i = lo; i < rows; ++i) dt += w(i, j) * w(i, k);
                    dt *= cf;
                    w(j, k) -= dt * w(j, j);
                    for (i64 i = lo; i < rows; ++i) w(i, k) -= dt * w(i, j);
                }
                w(j, j) = beta;
            }
            if (j < nres && !(std::fabs(beta) > 0.0)) return (int)(r0 + j + 1);
        }
        double* M = s.F.val.data() + S.fptr[f];
        for (i64 j = 0; j < nres; ++j) {
            const double sg = w(j, j) < 0.0 ? -1.0 : 1.0;
            for (i64 i = j; i < nf; ++i) M[i + j * nf] = sg * w(j, i);
        }
        for (i64 c = 0; c < nsep; ++c)
            for (i64 r = 0; r <= c; ++r) M[(nres + r) + (nres + c) * nf] = nres + r < jmax ? w(nres + r, nres + c) : 0.0;
    }
    return 0;
}

static bool initkkt(Solver& s, double delta, double& rho) {
    s.delta = delta;
    if (s.set.stable) {   // no ρ retry (uzawa.jl:162)
        rho = 0;
        return stable_factor(s, delta) == 0;
    }
    auto assemble = [&]() {
        std::fill(s.F.val.begin(), s.F.val.end(), 0.0);
        scatter_add(s.F, s.L, 1.0);
        scatter_add(s.F, s.H, delta);
    };
    assemble();
    int info = numeric_factor(s.F);
    rho = 0;
    if (info != 0) {
        assemble();
        rho = std::numeric_limits<double>::epsilon() * factor_lower_norm(s.F);
        const Symbolic& S = s.S;
        for (i64 f = 0; f < S.nfront; ++f) {
            i64 nres = S.nres[f], nf = nres + (i64)S.sep[f].size();
            double* M = s.F.val.data() + S.fptr[f];
            for (i64 j = 0; j < nres; ++j) M[j + j * nf] += rho;
        }
        info = numeric_factor(s.F);
        s.nfactor_retry++;
    }
    return info == 0;
}

typedef bool (*stopfn)(const Solver&, const double*);
static bool never(const Solver&, const double*) { return false; }

static void kktwindow(const double* rhist, const double* chist, double delta, i64 nir, i64 ncg,
                      double ftol, double gtol, double& dmin, double& dmax) {
    dmin = dmax = std::numeric_limits<double>::quiet_NaN();
    if (nir >= 1) {
        double logd = std::log(delta), logfres = std::log(rhist[1]);
        double loggtol = std::log(gtol), logftol = std::log(ftol);
        i64 i = 0;
        double logdmax = -std::numeric_limits<double>::infinity();
        double logdmin = logd + logfres - logftol;
        while (logdmin > logdmax && i < ncg + 1) {
            i += 1;
            double loggres = std::log(chist[i - 1]);
            logdmax = logd + (loggtol - loggres) / (double)i;
        }
        dmin = std::exp(logdmin);
        dmax = std::exp(logdmax);
    }
}

static int cg(Solver& s, stopfn stop, double* x, double* y, double* u, double atol, i64 itmax, i64& niter) {
    const double eps = std::numeric_limits<double>::epsilon();
    i64 m = s.m, n = s.n;
    double* p = s.cgp.data();
    double* w = s.cgw.data();
    niter = 0;
    double nu2 = vdot(u, u, m), nu = std::sqrt(nu2);
    s.cghist[0] = nu;
    double np2 = nu2;
    std::fill(y, y + m, 0.0);
    int status = CG_SOLVED;
    if (nu > atol && !stop(s, u)) {
        status = CG_ITMAX;
        if (itmax > 0) {
            std::copy(u, u + m, p);
            status = CG_CONTINUE;
            while (status == CG_CONTINUE) {
                niter += 1;
                gemvT(s.B, p, w, 1, 0);
                Lsolve(s.F, w);
                double ep2 = vdot(w, w, n);
                if (ep2 <= eps * np2) status = CG_NUMERICAL_FAILURE;
                else {
                    Usolve(s.F, w);
                    double a = nu2 / ep2;
                    for (i64 i = 0; i < m; ++i) y[i] += a * p[i];
                    for (i64 i = 0; i < n; ++i) x[i] += a * w[i];
                    gemvN(s.B, w, u, -a, 1);
                    double pnu2 = nu2;
                    nu2 = vdot(u, u, m); nu = std::sqrt(nu2);
                    s.cghist[niter] = nu;
                    if (nu <= atol || 1.0 + nu <= 1.0 || stop(s, u)) status = CG_SOLVED;
                    else if (niter >= itmax) status = CG_ITMAX;
                    else {
                        double b = nu2 / pnu2;
                        for (i64 i = 0; i < m; ++i) p[i] = u[i] + b * p[i];
                        np2 = nu2 + b * b * np2;
                    }
                }
            }
        }
    }
    return status;
}

struct KKTOut { i64 ncg, nir; int status; double dmin, dmax; };

static KKTOut solvekkt(Solver& s, stopfn fstop, stopfn gstop, double* x, double* y, const BSM& A,
                       const double* f, const double* g, bool warm, double ftol, double gtol,
                       double stall, i64 irmax, i64 cgmax, i64 irmin) {
    i64 m = s.m, n = s.n;
    double delta = s.delta, alpha = 1.0 / delta;
    double* df = s.df.data(); double* dg = s.dg.data(); double* dx = s.dx.data(); double* dyv = s.dy.data();
    i64 nir = 0, ncg = 0;
    if (warm) {
        mulkkt(s, df, dg, A, x, y);
        for (i64 i = 0; i < n; ++i) df[i] = f[i] - df[i];
        for (i64 i = 0; i < m; ++i) dg[i] = g[i] - dg[i];
    } else {
        std::copy(f, f + n, df); std::copy(g, g + m, dg);
        std::fill(x, x + n, 0.0); std::fill(y, y + m, 0.0);
    }
    double fres = vnorm(df, n), fprv = fres;
    s.uhist[0] = fres;
    int irstat;
    if (nir >= irmin && (fres <= ftol || fstop(s, df))) irstat = KKT_SOLVED;
    else if (nir >= irmax) irstat = KKT_IRMAX;
    else irstat = KKT_CONTINUE;
    while (irstat == KKT_CONTINUE) {
        nir += 1;
        for (i64 i = 0; i < n; ++i) dx[i] = df[i] * delta;
        gemvT(s.B, dg, dx, 1, 1);
        Lsolve(s.F, dx);
        Usolve(s.F, dx);
        gemvN(s.B, dx, dg, -1, 1);
        for (i64 i = 0; i < n; ++i) x[i] += dx[i];
        for (i64 i = 0; i < m; ++i) y[i] += alpha * dg[i];
        mulkkt(s, df, dg, A, x, y);
        for (i64 i = 0; i < n; ++i) df[i] = f[i] - df[i];
        for (i64 i = 0; i < m; ++i) dg[i] = g[i] - dg[i];
        fres = vnorm(df, n);
        s.uhist[nir] = fres;
        if (nir >= irmin && (fres <= ftol || fstop(s, df))) irstat = KKT_SOLVED;
        else if (nir > 1 && fres > (1 - stall) * fprv) irstat = KKT_STAGNATED;
        else if (nir >= irmax) irstat = KKT_IRMAX;
        else irstat = KKT_CONTINUE;
        fprv = fres;
    }
    for (i64 i = 0; i < m; ++i) y[i] -= alpha * dg[i];
    int cgstat = cg(s, gstop, x, dyv, dg, gtol, cgmax, ncg);
    for (i64 i = 0; i < m; ++i) y[i] += alpha * dyv[i];
    for (i64 i = 0; i < m; ++i) y[i] += alpha * dg[i];
    int status;
    if (cgstat == CG_NUMERICAL_FAILURE) status = KKT_NUMERICAL_FAILURE;
    else if (irstat == KKT_STAGNATED) status = KKT_STAGNATED;
    else if (irstat == KKT_IRMAX || cgstat == CG_ITMAX) status = KKT_ITMAX;
    else status = KKT_SOLVED;
    KKTOut o{ncg, nir, status, 0, 0};
    kktwindow(s.uhist.data(), s.cghist.data(), delta, nir, ncg, ftol, gtol, o.dmin, o.dmax);
    return o;
}

// --------------------------------------------------------------------------------------------
// solver pieces  (solver/ipm.jl, solver/solver.jl, solver/utils.jl, history/history.jl)
// --------------------------------------------------------------------------------------------
static double scalenorm(const double* v, const double* sc, i64 n) {
    double o = 0;
    for (i64 i = 0; i < n; ++i) { double t = v[i] / sc[i]; o += t * t; }
    return std::sqrt(o);
}
static double fnorm(const Solver& s, const double* Df) { return scalenorm(Df, s.pscl.data(), s.n) / (1 + s.sf); }
static double gnorm(const Solver& s, const double* Dg) { return scalenorm(Dg, s.yscl.data(), s.m) / (1 + s.sg); }
static bool fstop_exact(const Solver& s, const double* df) { return fnorm(s, df) <= s.set.feas_tol; }
static bool gstop_exact(const Solver& s, const double* dg) { return gnorm(s, dg) <= s.set.feas_tol; }

static void residuals(Solver& s) {
    mulkkt(s, s.Df.data(), s.Dg.data(), s.Q, s.p.data(), s.y.data());
    for (i64 i = 0; i < s.n; ++i) s.Df[i] = s.d[i] + s.f[i] - s.Df[i];
    for (i64 i = 0; i < s.m; ++i) s.Dg[i] = s.g[i] - s.Dg[i];
}

static bool isoptimal_(double mu, double mus, double mut, double pobj, double dobj, double pres,
                       double dres, i64 nu, double gap_tol, double feas_tol) {
    if (!(pres < feas_tol && dres < feas_tol)) return false;
    double tol = gap_tol * std::max(1.0, std::min(std::fabs(pobj), std::fabs(dobj)));
    if (mut > 0 && nu > 0) return (double)nu * (mu - mut + mut * std::log1p(mus * mut - 1.0)) <= tol;
    return pobj - dobj < tol;
}
static bool isoptimal(const Solver& s, double mu, double mus, double pobj, double dobj, double pres, double dres) {
    return isoptimal_(mu, mus, s.mut, pobj, dobj, pres, dres, s.nu, s.set.gap_tol, s.set.feas_tol);
}
static bool isnearoptimal(const Solver& s, double mu, double mus, double pobj, double dobj, double pres, double dres) {
    double fct = s.set.near_factor;
    return isoptimal_(mu, mus, s.mut, pobj, dobj, pres, dres, s.nu, fct * s.set.gap_tol, fct * s.set.feas_tol);
}

static bool isprimalinfeasible(Solver& s, double rtol, double atol) {
    double gy = vdot(s.g.data(), s.y.data(), s.m), ny = vnorm(s.y.data(), s.m);
    bool fl = gy > atol * ny * (1 + s.ng);
    if (fl) {
        double nQp = vnorm(s.Qp.data(), s.n);
        for (i64 i = 0; i < s.n; ++i) s.wf[i] = s.Qp[i] - s.d[i];
        gemvT(s.B, s.y.data(), s.wf.data(), -1, 1);
        fl = std::max(nQp, vnorm(s.wf.data(), s.n)) < rtol * gy * (1 + vnorm(s.d.data(), s.n) / ny);
    }
    return fl;
}
static bool isdualinfeasible(Solver& s, double rtol, double atol) {
    double fp = vdot(s.f.data(), s.p.data(), s.n), np = vnorm(s.p.data(), s.n);
    bool fl = fp > atol * np * (1 + s.nf);
    if (fl) {
        gemvN(s.B, s.p.data(), s.Dya.data(), 1, 0);
        fl = std::max(vnorm(s.Dya.data(), s.m), vnorm(s.Qp.data(), s.n)) < rtol * std::fabs(fp);
    }
    return fl;
}

static int nearstatus(Solver& s, int status, double mu, double mus, double pobj, double dobj, double pres, double dres) {
    double fct = s.set.near_factor;
    if (isnearoptimal(s, mu, mus, pobj, dobj, pres, dres)) status = NEAR_OPTIMAL;
    else if (isprimalinfeasible(s, fct * s.set.infeas_rel, s.set.infeas_abs)) status = NEAR_PRIMAL_INFEASIBLE;
    else if (isdualinfeasible(s, fct * s.set.infeas_rel, s.set.infeas_abs)) status = NEAR_DUAL_INFEASIBLE;
    return status;
}

static bool isstalled(const Solver& s) {
    const i64 window = 5;
    i64 n = (i64)s.hist.size();
    double tol = s.set.stall_tol;
    if (n - s.stall0 > window) {
        for (i64 i = n - window; i < n; ++i) {
            bool muok = s.hist[i].mu < (1 - tol) * s.hist[i - 1].mu;
            bool pok = s.hist[i].pres < (1 - tol) * s.hist[i - 1].pres;
            bool dok = s.hist[i].dres < (1 - tol) * s.hist[i - 1].dres;
            if (muok || pok || dok) return false;
        }
        return true;
    }
    return false;
}

static double getaug(const Solver& s) {
    double nH = bnorm(s.H);
    if (s.nB == 0 || nH == 0) return 1.0;
    if (s.hist.empty()) return s.set.aug_tol * s.nB * s.nB / nH;
    const ob_row& r = s.hist.back();
    double delta = r.delta, dmin = r.dmin, dmax = r.dmax;
    if (r.ppass > 1) {
        if (std::isfinite(dmin)) delta = std::max(delta, dmin);
        delta *= 10;
    } else if (std::isfinite(dmin) && std::isfinite(dmax) && dmin > 0 && dmax > 0) {
        delta = std::sqrt(dmin) * std::sqrt(dmax);
    }
    return delta;
}

static const double FORCING_FRAC = 0.1;

static int step_(Solver& s);

// precision 2 (mixed): iterate with an FP32 factor until a KKT solve misses its tolerance; that
// iteration is redone from the saved iterate with the FP64 factor, which is kept from then on.
// An accepted FP32 iteration that needed more than MIXED_MAX_SOLVES KKT solves (IR passes + CG
// steps) also moves the solve to the FP64 factor for the remaining iterations, without a redo.  A
// stall while on the FP32 factor is redone with the FP64 factor, and the stall window restarts.
static const double MIXED_MAX_SOLVES = 4;
static int step(Solver& s) {
    if (s.set.precision != 2 || s.nfallback > 0 || s.switched) { if (s.set.precision == 2) s.F.fp32 = false; return step_(s); }
    std::vector<double> p0 = s.p, d0 = s.d, y0 = s.y;
    std::vector<double> c0 = s.cache;
    s.F.fp32 = true;
    s.stallhit = false;
    int st = step_(s);
    const ob_row& r = s.hist.back();
    bool kktfail = (r.pstat != KKT_SOLVED || r.cstat != KKT_SOLVED) && !std::isnan(r.rho);
    if (!kktfail && !s.stallhit) {
        s.nfp32++;
        if (r.piter + r.ppass + r.citer + r.cpass > MIXED_MAX_SOLVES) s.switched = true;
        return st;
    }
    // a KKT solve missed its tolerance, or the FP32 iterates stalled: redo from the saved iterate
    // with the FP64 factor, kept from now on (after a stall the stall window restarts)
    s.hist.pop_back();
    if (s.stallhit) { s.switched = true; s.stall0 = (i64)s.hist.size(); }
    s.p = p0; s.d = d0; s.y = y0; s.cache = c0;
    s.F.fp32 = false;
    s.nfallback++;
    return step_(s);
}

static int step_(Solver& s) {
    const double NaN = std::numeric_limits<double>::quiet_NaN();
    int status = CONTINUE;
    ob_row row{NaN, NaN, NaN, NaN, 0.0, 0, 0, (double)KKT_SOLVED, 0, 0, (double)KKT_SOLVED,
               NaN, NaN, NaN, 0.0, NaN, NaN};
    i64 n = s.n, m = s.m;
    double delta = getaug(s);
    double pd = vdot(s.p.data(), s.d.data(), n);
    auto t0 = clk::now();
    double spsd = 0;
    bool ok = scale_all(s, spsd);
    s.tm.scale += secs(t0);
    if (!ok) {
        status = NUMERICAL_FAILURE;
    } else {
        residuals(s);
        double nuf = (double)std::max<i64>(s.nu, 1);
        double mu = pd / nuf, mus = spsd / nuf, chi = mu * mus - 1;
        double pres = gnorm(s, s.Dg.data()), dres = fnorm(s, s.Df.data());
        gemvN(s.Q, s.p.data(), s.Qp.data(), 1, 0);
        double pQp = vdot(s.p.data(), s.Qp.data(), n);
        double pobj = pQp / 2 - vdot(s.f.data(), s.p.data(), n);
        double dobj = vdot(s.g.data(), s.y.data(), m) - pQp / 2;
        row.mu = mu; row.chi = chi; row.pres = pres; row.dres = dres; row.pobj = pobj; row.dobj = dobj;
        if (isoptimal(s, mu, mus, pobj, dobj, pres, dres)) status = OPTIMAL;
        else if (isprimalinfeasible(s, s.set.infeas_rel, s.set.infeas_abs)) status = PRIMAL_INFEASIBLE;
        else if (isdualinfeasible(s, s.set.infeas_rel, s.set.infeas_abs)) status = DUAL_INFEASIBLE;
        else if ((i64)s.hist.size() >= s.set.max_iter) status = nearstatus(s, ITERATION_LIMIT, mu, mus, pobj, dobj, pres, dres);
        else if (isstalled(s)) { s.stallhit = true; status = nearstatus(s, STALLED, mu, mus, pobj, dobj, pres, dres); }
        else if (s.nu == 0) {
            double rho;
            t0 = clk::now();
            bool iok = initkkt(s, delta, rho);
            s.tm.initkkt += secs(t0);
            row.rho = rho;
            if (!iok) status = nearstatus(s, NUMERICAL_FAILURE, mu, mus, pobj, dobj, pres, dres);
            else {
                t0 = clk::now();
                double eps = std::numeric_limits<double>::epsilon();
                KKTOut o = solvekkt(s, fstop_exact, gstop_exact, s.Dpa.data(), s.Dya.data(), s.H,
                                    s.Df.data(), s.Dg.data(), false, eps, eps, s.set.refine_stall_tol,
                                    s.set.refine_max_iter, s.set.newton_max_iter, 0);
                s.tm.solve += secs(t0);
                row.piter = (double)o.ncg; row.ppass = (double)o.nir; row.pstat = o.status;
                row.dmin = o.dmin; row.dmax = o.dmax;
                for (i64 i = 0; i < n; ++i) s.p[i] += s.Dpa[i];
                for (i64 i = 0; i < m; ++i) s.y[i] += s.Dya[i];
            }
        } else if (!(mu > 0)) {
            status = nearstatus(s, NUMERICAL_FAILURE, mu, mus, pobj, dobj, pres, dres);
        } else {
            double rho;
            t0 = clk::now();
            bool iok = initkkt(s, delta, rho);
            s.tm.initkkt += secs(t0);
            row.rho = rho;
            if (!iok) status = nearstatus(s, NUMERICAL_FAILURE, mu, mus, pobj, dobj, pres, dres);
            else {
                double mu1 = s.hist.empty() ? mu : s.hist.front().mu;
                double tol;
                if (s.mut > 0) {
                    double dmu = std::fabs(mu - s.mut), dmu1 = std::fabs(mu1 - s.mut);
                    tol = FORCING_FRAC * std::min(dmu / dmu1, 1.0);
                } else tol = FORCING_FRAC * mu / mu1;
                double ftol = tol * (1 + s.nf), gtol = tol * (1 + s.ng);
                // predictor (solver/ipm.jl:119-163)
                t0 = clk::now();
                if (s.mut > 0) initpredictor(s, s.wf.data(), s.mut);
                else for (i64 i = 0; i < n; ++i) s.wf[i] = -s.d[i];
                for (i64 i = 0; i < n; ++i) s.wf[i] += s.Df[i];
                KKTOut po = solvekkt(s, never, never, s.Dpa.data(), s.Dya.data(), s.H, s.wf.data(), s.Dg.data(),
                                     false, ftol, gtol, s.set.refine_stall_tol, s.set.refine_max_iter,
                                     s.set.newton_max_iter, 1);
                std::copy(s.Df.begin(), s.Df.end(), s.Dda.begin());
                gemvT(s.B, s.Dya.data(), s.Dda.data(), -1, -1);
                gemvN(s.Q, s.Dpa.data(), s.Dda.data(), 1, 1);
                s.tm.predictor += secs(t0);
                row.piter = (double)po.ncg; row.ppass = (double)po.nir; row.pstat = po.status;
                row.dmin = po.dmin; row.dmax = po.dmax;
                zerofree(s, s.Dda.data());
                // corrector (solver/ipm.jl:181-272)
                t0 = clk::now();
                auto t1 = clk::now();
                double taua = maxsteps(s, s.Dpa.data(), s.Dda.data(), 1.0);
                s.tm.maxsteps += secs(t1);
                double sm = 0;
                for (i64 j = 0; j < n; ++j) sm += (s.p[j] + taua * s.Dpa[j]) * (s.d[j] + taua * s.Dda[j]);
                double mua = sm / (double)s.nu;
                if (s.mut > 0) {
                    double dmu = mu - s.mut;
                    if (dmu > 0) {
                        double dmua = std::min(std::max(mua - s.mut, 0.0), dmu);
                        sm = s.mut + std::min(std::max(dmua * (dmua / dmu) * (dmua / dmu), 0.0), dmu);
                    } else sm = s.mut;
                } else {
                    sm = std::min(std::max(mua * (mua / mu) * (mua / mu), 0.0), mu);
                }
                initcorrector(s, s.wf.data(), s.Dpa.data(), s.Dda.data(), sm);
                for (i64 i = 0; i < n; ++i) s.wf[i] += s.Df[i];
                std::copy(s.Dpa.begin(), s.Dpa.end(), s.Dp.begin());
                std::copy(s.Dya.begin(), s.Dya.end(), s.Dy.begin());
                KKTOut co = solvekkt(s, never, never, s.Dp.data(), s.Dy.data(), s.H, s.wf.data(), s.Dg.data(),
                                     true, ftol, gtol, s.set.refine_stall_tol, s.set.refine_max_iter,
                                     s.set.newton_max_iter, 1);
                std::copy(s.Df.begin(), s.Df.end(), s.Dd.begin());
                gemvT(s.B, s.Dy.data(), s.Dd.data(), -1, -1);
                gemvN(s.Q, s.Dp.data(), s.Dd.data(), 1, 1);
                s.tm.corrector += secs(t0);
                row.citer = (double)co.ncg; row.cpass = (double)co.nir; row.cstat = co.status;
                zerofree(s, s.Dd.data());
                if (po.status != KKT_SOLVED || co.status != KKT_SOLVED) {
                    status = nearstatus(s, NUMERICAL_FAILURE, mu, mus, pobj, dobj, pres, dres);
                } else {
                    t1 = clk::now();
                    double st = maxsteps(s, s.Dp.data(), s.Dd.data(), s.set.step_frac);
                    s.tm.maxsteps += secs(t1);
                    row.step = st;
                    for (i64 i = 0; i < n; ++i) { s.p[i] += st * s.Dp[i]; s.d[i] += st * s.Dd[i]; }
                    for (i64 i = 0; i < m; ++i) s.y[i] += st * s.Dy[i];
                }
            }
        }
    }
    row.delta = delta;
    s.hist.push_back(row);
    if (s.set.verbose > 0) {
        i64 i = (i64)s.hist.size();
        fprintf(stderr, "| %4ld | %8.2e | %8.2e | %9.2e | %9.2e | %6.4f | %5d | %8.2e | %8.2e | %8.2e | %8.2e |\n",
                (long)i, row.pres, row.dres, row.pobj, row.dobj, row.step,
                (int)(row.piter + row.ppass + row.citer + row.cpass), row.rho, row.delta, row.mu, row.chi);
    }
    return status;
}

// --------------------------------------------------------------------------------------------
// construction  (solver/ipm.jl:431-478; kkt.jl:23-53; scaling.jl:52-184; solver/ipm.jl:321-429)
// --------------------------------------------------------------------------------------------
static void infnorms(std::vector<double>& rnrm, std::vector<double>& vnrm, const BSM& B, const BSM& Q) {
    std::fill(rnrm.begin(), rnrm.end(), 0.0);
    for (i64 v = 0; v < B.nvtx; ++v) {
        double nv = 0;
        for (i64 e = Q.xsrc[v]; e < Q.xsrc[v + 1]; ++e)
            for (i64 b = Q.xblk[e]; b < Q.xblk[e + 1]; ++b) nv = std::max(nv, std::fabs(Q.val[b]));
        i64 nc = B.ncols(v);
        for (i64 e = B.xsrc[v]; e < B.xsrc[v + 1]; ++e) {
            i64 u = B.tgt[e], r0 = B.xrow[u], nr = B.nrows(u);
            const double* blk = B.val.data() + B.xblk[e];
            for (i64 j = 0; j < nc; ++j)
                for (i64 i = 0; i < nr; ++i) {
                    double a = std::fabs(blk[i + j * nr]);
                    nv = std::max(nv, a);
                    rnrm[r0 + i] = std::max(rnrm[r0 + i], a);
                }
        }
        vnrm[v] = nv;
    }
}

static void applyscaling(BSM& B, BSM& Q, const std::vector<double>& ys, const std::vector<double>& vs) {
    for (i64 v = 0; v < B.nvtx; ++v) {
        double sv = vs[v];
        i64 nc = B.ncols(v);
        for (i64 e = B.xsrc[v]; e < B.xsrc[v + 1]; ++e) {
            i64 u = B.tgt[e], r0 = B.xrow[u], nr = B.nrows(u);
            double* blk = B.val.data() + B.xblk[e];
            for (i64 j = 0; j < nc; ++j)
                for (i64 i = 0; i < nr; ++i) blk[i + j * nr] *= ys[r0 + i] * sv;
        }
        for (i64 e = Q.xsrc[v]; e < Q.xsrc[v + 1]; ++e) {
            double sc = vs[Q.tgt[e]] * sv;
            for (i64 b = Q.xblk[e]; b < Q.xblk[e + 1]; ++b) Q.val[b] *= sc;
        }
    }
}

static void equilibrate(Solver& s, int itmax, double tol) {
    BSM& B = s.B; BSM& Q = s.Q;
    i64 nrow = B.nrow, nvtx = B.nvtx;
    std::vector<double> vscl(nvtx, 1.0), vnrm(nvtx, 0.0), rnrm(nrow, 0.0), vswp(nvtx, 1.0), rswp(nrow, 1.0);
    for (int it = 0; it < itmax; ++it) {
        infnorms(rnrm, vnrm, B, Q);
        double dd = 0;
        for (i64 v = 0; v < nvtx; ++v) {
            double nn = std::sqrt(vnrm[v]);
            dd = std::max(dd, std::fabs(1.0 - nn));
            if (nn != 0) { vswp[v] = 1.0 / nn; vscl[v] *= vswp[v]; }
        }
        for (i64 i = 0; i < nrow; ++i) {
            double nn = std::sqrt(rnrm[i]);
            dd = std::max(dd, std::fabs(1.0 - nn));
            if (nn != 0) { rswp[i] = 1.0 / nn; s.yscl[i] *= rswp[i]; }
        }
        applyscaling(B, Q, rswp, vswp);
        if (dd < tol) break;
    }
    for (i64 v = 0; v < nvtx; ++v)
        for (i64 j = B.xcol[v]; j < B.xcol[v + 1]; ++j) { s.pscl[j] = vscl[v]; s.f[j] *= s.pscl[j]; }
    for (i64 i = 0; i < nrow; ++i) s.g[i] *= s.yscl[i];
}

static void startingpoint(Solver& s) {
    i64 n = s.n, m = s.m;
    for (i64 v = 0; v < s.B.nvtx; ++v) {
        i64 c0 = s.B.xcol[v], nc = s.B.ncols(v);
        cone_identity(s.K[v], s.Kp[v], nc, s.p.data() + c0);
        cone_identity(s.K[v], s.Kp[v], nc, s.d.data() + c0);
    }
    std::vector<double> z(m), w(n);
    gemvN(s.B, s.p.data(), z.data(), 1, 0);
    gemvN(s.Q, s.p.data(), w.data(), 1, 0);
    double eps = std::numeric_limits<double>::epsilon();
    double np = vnorm(s.p.data(), n), nz = vnorm(z.data(), m), nw = vnorm(w.data(), n);
    double sp = nz > eps * np ? std::max(1.0, vnorm(s.g.data(), m) / nz) : 1.0;
    double sd = np > eps ? std::max(1.0, (vnorm(s.f.data(), n) + sp * nw) / np) : 1.0;
    for (i64 i = 0; i < n; ++i) { s.p[i] *= sp; s.d[i] *= sd; }
}

#include "oracle_comp.hpp"

}  // namespace orc

using namespace orc;

extern "C" {

// extmul! (pair = 0) / twomul! (pair = 1) of BlockSparseArrays on the host (comp.jl:280-311):
// c ← α op(A) b + β c with op = transpose when trans; s, cs (nullable) get phase 1's pair
int oracle_twomul(const ob_bsm* Ac, int trans, const double* b, double alpha, double beta, double* c, double* cc,
                  double* s, double* cs) {
    const BSM A = from_c(Ac);
    const i64 nout = trans ? A.ncol : A.nrow;
    std::vector<double> sv(nout), csv(nout);
    c_twogemv(A, trans != 0, b, sv.data(), csv.data());
    if (s) { std::copy(sv.begin(), sv.end(), s); std::copy(csv.begin(), csv.end(), cs); }
    c_epilogue(nout, c, cc, alpha, sv.data(), csv.data(), beta, cc != nullptr);
    return 0;
}

int oracle_set_blas(const char* path, int nthreads) {
    void* h = dlopen(path, RTLD_NOW | RTLD_LOCAL);
    if (!h) return -1;
    g_dpotrf = (potrf_t)dlsym(h, "scipy_dpotrf_");
    g_dtrsm = (trsm_t)dlsym(h, "scipy_dtrsm_");
    g_dsyrk = (syrk_t)dlsym(h, "scipy_dsyrk_");
    g_spotrf = (spotrf_t)dlsym(h, "scipy_spotrf_");
    g_strsm = (strsm_t)dlsym(h, "scipy_strsm_");
    g_ssyrk = (ssyrk_t)dlsym(h, "scipy_ssyrk_");
    g_setthr = (setthr_t)dlsym(h, "scipy_openblas_set_num_threads");
    if (g_setthr && nthreads > 0) g_setthr(nthreads);
    return (g_dpotrf && g_dtrsm && g_dsyrk) ? 0 : -2;
}

int oracle_set_threads(int nthreads) {
    if (g_setthr && nthreads > 0) { g_setthr(nthreads); return 0; }
    return -1;
}

// the starting-point part of reinit! (solver/ipm.jl:390-427): from the cone identity scaled by
// startingpoint!, or the given p0/d0 (user order) completed by shadows; y from y0 or zero; the cone
// caches reset and the history emptied
static void reinit_start(Solver& s, const double* p0, const double* d0, const double* y0) {
    i64 n = s.n, m = s.m, nv = s.B.nvtx;
    std::fill(s.y.begin(), s.y.end(), 0.0);
    if (!p0 && !d0) {
        startingpoint(s);
        if (y0) for (i64 i = 0; i < m; ++i) s.y[i] = y0[s.P1[i]] / s.yscl[i];
    } else {
        if (p0) for (i64 i = 0; i < n; ++i) s.p[i] = p0[s.P2[i]];
        if (d0) for (i64 i = 0; i < n; ++i) s.d[i] = d0[s.P2[i]];
        for (i64 v = 0; v < nv; ++v) {
            i64 c0 = s.B.xcol[v], nc = s.B.ncols(v);
            double* cv = s.cache.data() + s.cxblk[v];
            if (!d0) cone_shadow(s.K[v], s.Kp[v], nc, s.d.data() + c0, s.p.data() + c0, cv, s.cwork.data());
            else if (!p0) cone_pshadow(s.K[v], s.Kp[v], nc, s.p.data() + c0, s.d.data() + c0, cv, s.cwork.data());
        }
        if (y0) for (i64 i = 0; i < m; ++i) s.y[i] = y0[s.P1[i]];
        for (i64 i = 0; i < n; ++i) { s.p[i] /= s.pscl[i]; s.d[i] *= s.pscl[i]; }
        for (i64 i = 0; i < m; ++i) s.y[i] /= s.yscl[i];
    }
    for (i64 v = 0; v < nv; ++v)
        cone_initcache(s.K[v], s.Kp[v], s.B.ncols(v), s.cache.data() + s.cxblk[v]);
    s.hist.clear();
}

// Build a solver: IPMSolver(prob, settings; p0, d0, y0) with the vertex elimination order
// `vperm` (0-based, length nvtx; NULL = identity) standing in for CliqueTrees.symbolic.
void* oracle_create(const ob_bsm* Qc, const ob_bsm* Bc, const double* f, const double* g, double mu,
                    const int32_t* cone_kind, const double* cone_param, const int64_t* P1,
                    const int64_t* P2, const int64_t* vperm, const ob_settings* set,
                    const double* p0, const double* d0, const double* y0) {
    Solver* s = new Solver();
    s->set = *set;
    BSM Q0 = from_c(Qc), B0 = from_c(Bc);
    i64 nv = B0.nvtx;
    s->n = B0.ncol; s->m = B0.nrow; s->mut = mu;
    // initial vertex order, then etree postorder on top (kkt.jl:23-53 symbkkt)
    std::vector<i64> perm(nv);
    for (i64 i = 0; i < nv; ++i) perm[i] = vperm ? vperm[i] : i;
    {
        BSM Bs = selectvtxs(B0, perm);
        BSM Qs = halfselectvtxs(halfselectvtxs(Q0, perm), perm);
        BSM Ls = gramian(Bs);
        auto adj = vertexgraph(Qs, Ls);
        std::vector<i64> w(nv);
        for (i64 v = 0; v < nv; ++v) w[v] = Bs.ncols(v);
        Symbolic S0 = analyze(adj, w);
        std::vector<i64> p2(nv);
        for (i64 k = 0; k < nv; ++k) p2[k] = perm[S0.postperm[k]];
        perm = p2;
    }
    s->B = selectvtxs(B0, perm);
    s->Q = halfselectvtxs(halfselectvtxs(Q0, perm), perm);
    // column permutation: P * P2 (solver column -> user column)
    std::vector<i64> cperm;
    for (i64 k = 0; k < nv; ++k)
        for (i64 j = B0.xcol[perm[k]]; j < B0.xcol[perm[k] + 1]; ++j) cperm.push_back(j);
    s->P2.resize(s->n); s->P1.resize(s->m);
    s->f.resize(s->n); s->g.resize(s->m);
    for (i64 i = 0; i < s->n; ++i) { s->P2[i] = (P2 ? P2[cperm[i]] - 1 : cperm[i]); s->f[i] = f[cperm[i]]; }
    for (i64 i = 0; i < s->m; ++i) { s->P1[i] = (P1 ? P1[i] - 1 : i); s->g[i] = g[i]; }
    s->K.resize(nv); s->Kp.resize(nv);
    for (i64 k = 0; k < nv; ++k) { s->K[k] = cone_kind[perm[k]]; s->Kp[k] = cone_param ? cone_param[perm[k]] : 0.0; }
    // conedegree (solver/utils.jl:1-9)
    s->nu = 0;
    for (i64 v = 0; v < nv; ++v) s->nu += cone_degree(s->K[v], s->B.ncols(v));
    s->pscl.assign(s->n, 1.0); s->yscl.assign(s->m, 1.0);
    if (s->set.scale_max_iter > 0) equilibrate(*s, s->set.scale_max_iter, 1e-3);
    s->L = gramian(s->B);
    {
        auto adj = vertexgraph(s->Q, s->L);
        std::vector<i64> w(nv);
        for (i64 v = 0; v < nv; ++v) w[v] = s->B.ncols(v);
        s->S = analyze(adj, w);
    }
    s->F.S = &s->S;
    s->F.val.assign(s->S.fsize, 0.0);
    s->F.fp32 = s->set.precision >= 1;
    s->H = s->Q;
    // caches (cone.jl:46-65) and workspaces
    s->cxblk.assign(nv + 1, 0);
    i64 wmax = 0;
    for (i64 v = 0; v < nv; ++v) {
        s->cxblk[v + 1] = s->cxblk[v] + cone_cachesize(s->K[v], s->B.ncols(v));
        wmax = std::max<i64>(wmax, cone_workspacesize(s->K[v], s->B.ncols(v)));
    }
    s->cache.assign(s->cxblk[nv], 0.0); s->cwork.assign(std::max<i64>(wmax, 1), 0.0);
    i64 n = s->n, m = s->m;
    for (auto* v : {&s->Df, &s->wf, &s->Qp, &s->Dpa, &s->Dda, &s->Dp, &s->Dd, &s->df, &s->dx, &s->cgw, &s->p, &s->d})
        v->assign(n, 0.0);
    for (auto* v : {&s->Dg, &s->Dya, &s->Dy, &s->dg, &s->dy, &s->cgp, &s->y}) v->assign(m, 0.0);
    s->step.assign(nv, 0.0); s->spsd.assign(nv, 0.0); s->flag.assign(nv, 1);
    s->uhist.assign(s->set.refine_max_iter + 2, 0.0);
    s->cghist.assign(s->set.newton_max_iter + 1, 0.0);
    s->nB = bnorm(s->B);
    s->nf = vnorm(s->f.data(), n); s->ng = vnorm(s->g.data(), m);
    s->sg = scalenorm(s->g.data(), s->yscl.data(), m);
    s->sf = scalenorm(s->f.data(), s->pscl.data(), n);
    reinit_start(*s, p0, d0, y0);
    return s;
}

// reinit!(s; p0, d0, y0, f, g) (solver/ipm.jl:371-429): f and g (user order) replace the solver's
// in its scaling; H, the equilibration and BᵀB stay as they are
int oracle_reinit(void* h, const double* p0, const double* d0, const double* y0, const double* f, const double* g) {
    Solver& s = *(Solver*)h;
    const i64 n = s.n, m = s.m;
    if (f) {
        for (i64 i = 0; i < n; ++i) s.f[i] = f[s.P2[i]] * s.pscl[i];
        s.nf = vnorm(s.f.data(), n);
        s.sf = scalenorm(s.f.data(), s.pscl.data(), n);
    }
    if (g) {
        for (i64 i = 0; i < m; ++i) s.g[i] = g[s.P1[i]] * s.yscl[i];
        s.ng = vnorm(s.g.data(), m);
        s.sg = scalenorm(s.g.data(), s.yscl.data(), m);
    }
    reinit_start(s, p0, d0, y0);
    s.nfactor_retry = 0; s.nfallback = 0; s.switched = false; s.stall0 = 0; s.stallhit = false; s.nfp32 = 0;
    return 0;
}

// ---- sensitivities (ipm/differential.jl) ---------------------------------------------------
// d*(p): the dual shadow of every cone at p (dualshadow!, cone.jl:562-608)
static void dualshadow_all(Solver& s, double* ds) {
    for (i64 v = 0; v < s.B.nvtx; ++v) {
        i64 c0 = s.B.xcol[v], nc = s.B.ncols(v);
        cone_shadow(s.K[v], s.Kp[v], nc, ds + c0, s.p.data() + c0, s.cache.data() + s.cxblk[v], s.cwork.data());
    }
}

// the factorization and tolerances every rule starts from (differential.jl:5-14): δ = getaug(s),
// initkkt!(s, δ), tol from the history's first and last μ
static bool sens_setup(Solver& s, double& ftol, double& gtol) {
    double rho;
    if (!initkkt(s, getaug(s), rho)) return false;
    const double mu0 = s.hist.empty() ? 0.0 : s.hist.front().mu;
    const double tol = mu0 == 0 ? FORCING_FRAC * s.set.gap_tol : FORCING_FRAC * s.hist.back().mu / mu0;
    ftol = tol * (1 + s.nf); gtol = tol * (1 + s.ng);
    return true;
}

// r = F2(p) Δp and r = F3(p)[u, w] per cone (primalhess!, primalthird!; cone.jl:579-607): pos.jl:193-219,
// soc.jl:510-560 (det(p) from the cache), tdc.jl:509-521, sdp.jl:696-790 (the cached R)
static void primalhess_all(Solver& s, double* r, const double* dp) {
    for (i64 v = 0; v < s.B.nvtx; ++v) {
        const i64 c0 = s.B.xcol[v], nc = s.B.ncols(v);
        const double* p = s.p.data() + c0; const double* x = dp + c0; double* o = r + c0;
        const double* C = s.cache.data() + s.cxblk[v];
        const int k = s.K[v];
        if (k == CONE_POS) { for (i64 i = 0; i < nc; ++i) o[i] = x[i] / (p[i] * p[i]); }
        else if (k == CONE_SOC) {
            double hi, lo;
            socdot(p, x, nc, hi, lo);
            const double pdet = C[1], t = hi / pdet, gm = 2 / pdet, t2 = 2 * t;
            o[0] = gm * std::fma(t2, p[0], -x[0]);
            for (i64 i = 1; i < nc; ++i) o[i] = gm * std::fma(-t2, p[i], x[i]);
        } else if (k == CONE_EXP || k == CONE_POW) tdhessmul(o, C + TD_L, x);
        else if (k == CONE_SDP) {
            const int d = (int)triroot(nc);
            std::vector<double> U((size_t)d * d), A((size_t)d * d);
            sdp_smat(U.data(), x, d); sdp_symm(U.data(), d);
            sdp_mul(A.data(), C, true, U.data(), false, d); sdp_mul(U.data(), A.data(), false, C, false, d);
            sdp_mul(A.data(), C, false, U.data(), false, d); sdp_mul(U.data(), A.data(), false, C, true, d);
            sdp_svec(o, U.data(), d);
        } else { for (i64 i = 0; i < nc; ++i) o[i] = 0; }
    }
}

static void primalthird_all(Solver& s, double* r, const double* u, const double* w) {
    for (i64 v = 0; v < s.B.nvtx; ++v) {
        const i64 c0 = s.B.xcol[v], nc = s.B.ncols(v);
        const double* p = s.p.data() + c0; const double* a = u + c0; const double* b = w + c0; double* o = r + c0;
        const double* C = s.cache.data() + s.cxblk[v];
        const int k = s.K[v];
        if (k == CONE_POS) { for (i64 i = 0; i < nc; ++i) o[i] = -2 * a[i] * b[i] / (p[i] * p[i] * p[i]); }
        else if (k == CONE_SOC) {
            double a1, a2, a3, lo;
            socdot(p, a, nc, a1, lo); socdot(p, b, nc, a2, lo); socdot(a, b, nc, a3, lo);
            const double pdet = C[1], u1 = a1 / pdet, u2 = a2 / pdet, vv = a3 / pdet, gm = 4 / pdet;
            const double cc = std::fma(-4 * u1, u2, vv);
            for (i64 i = 0; i < nc; ++i) {
                const double t = std::fma(u1, b[i], std::fma(u2, a[i], cc * p[i]));
                o[i] = i == 0 ? gm * t : -gm * t;
            }
        } else if (k == CONE_EXP || k == CONE_POW) {
            double D[9];
            tdbarrthird(TD{k, s.Kp[v]}, D, p, a, C);
            for (int i = 0; i < 3; ++i) o[i] = D[i] * b[0] + D[i + 3] * b[1] + D[i + 6] * b[2];
        } else if (k == CONE_SDP) {
            const int d = (int)triroot(nc);
            std::vector<double> U((size_t)d * d), V((size_t)d * d), A((size_t)d * d);
            sdp_smat(U.data(), a, d); sdp_symm(U.data(), d); sdp_smat(V.data(), b, d); sdp_symm(V.data(), d);
            sdp_mul(A.data(), C, true, U.data(), false, d); sdp_mul(U.data(), A.data(), false, C, false, d);
            sdp_mul(A.data(), C, true, V.data(), false, d); sdp_mul(V.data(), A.data(), false, C, false, d);
            sdp_mul(A.data(), U.data(), false, V.data(), false, d);
            for (int j = 0; j < d; ++j)
                for (int i = 0; i < d; ++i) V[i + (size_t)j * d] = i == j ? 2 * A[i + (size_t)j * d] : A[i + (size_t)j * d] + A[j + (size_t)i * d];
            sdp_mul(U.data(), C, false, V.data(), false, d); sdp_mul(A.data(), U.data(), false, C, true, d);
            sdp_svec(o, A.data(), d);
            for (i64 i = 0; i < nc; ++i) o[i] = -o[i];
        } else { for (i64 i = 0; i < nc; ++i) o[i] = 0; }
    }
}

// frule2! (ipm/differential.jl:82-260); every vector in user order, NULL seed = 0; outputs
// p1 y1 d1 p2 y2 d2 p12 y12 d12 (each may be NULL).  Returns 0, or -1 when the factorization fails.
int oracle_frule2(void* h, const double* Df1, const double* Dg1, double Dmu1, const double* Df2,
                  const double* Dg2, double Dmu2, double* const* out) {
    Solver& s = *(Solver*)h;
    const i64 n = s.n, m = s.m;
    double ftol, gtol;
    if (!sens_setup(s, ftol, gtol)) return -1;
    std::vector<double> ds(n), fx(n), gx(m), p1(n, 0.0), y1(m, 0.0), d1(n), p2(n, 0.0), y2(m, 0.0), d2(n);
    dualshadow_all(s, ds.data());
    for (int k = 0; k < 2; ++k) {
        const double* Df = k ? Df2 : Df1; const double* Dg = k ? Dg2 : Dg1; const double dm = k ? Dmu2 : Dmu1;
        std::vector<double>& px = k ? p2 : p1; std::vector<double>& yx = k ? y2 : y1; std::vector<double>& dx = k ? d2 : d1;
        for (i64 i = 0; i < n; ++i) fx[i] = std::fma(dm, ds[i], (Df ? Df[s.P2[i]] : 0.0) * s.pscl[i]);
        for (i64 i = 0; i < m; ++i) gx[i] = (Dg ? Dg[s.P1[i]] : 0.0) * s.yscl[i];
        solvekkt(s, never, never, px.data(), yx.data(), s.H, fx.data(), gx.data(), false, ftol, gtol,
                 s.set.refine_stall_tol, s.set.refine_max_iter, s.set.newton_max_iter, 1);
        gemvN(s.H, px.data(), dx.data(), 1, 0);            // Δd = Δμ d* − (H − Q) Δp
        gemvN(s.Q, px.data(), dx.data(), -1, 1);
        for (i64 i = 0; i < n; ++i) dx[i] = std::fma(dm, ds[i], -dx[i]);
    }
    primalthird_all(s, fx.data(), p1.data(), p2.data());
    for (i64 i = 0; i < n; ++i) fx[i] *= s.mut;
    if (Dmu1 != 0) { primalhess_all(s, ds.data(), p2.data()); for (i64 i = 0; i < n; ++i) fx[i] = std::fma(Dmu1, ds[i], fx[i]); }
    if (Dmu2 != 0) { primalhess_all(s, ds.data(), p1.data()); for (i64 i = 0; i < n; ++i) fx[i] = std::fma(Dmu2, ds[i], fx[i]); }
    for (i64 i = 0; i < n; ++i) fx[i] = -fx[i];
    auto pull = [&](double* o, const std::vector<double>& v, bool col, int how) {   // how: 0 ×scl, 1 ÷scl
        if (!o) return;
        if (col) for (i64 i = 0; i < n; ++i) o[s.P2[i]] = how ? v[i] / s.pscl[i] : v[i] * s.pscl[i];
        else for (i64 i = 0; i < m; ++i) o[s.P1[i]] = v[i] * s.yscl[i];
    };
    pull(out[0], p1, true, 0); pull(out[1], y1, false, 0); pull(out[2], d1, true, 1);
    pull(out[3], p2, true, 0); pull(out[4], y2, false, 0); pull(out[5], d2, true, 1);
    std::fill(gx.begin(), gx.end(), 0.0);
    std::fill(p2.begin(), p2.end(), 0.0); std::fill(y2.begin(), y2.end(), 0.0);
    solvekkt(s, never, never, p2.data(), y2.data(), s.H, fx.data(), gx.data(), false, ftol, gtol,
             s.set.refine_stall_tol, s.set.refine_max_iter, s.set.newton_max_iter, 1);
    gemvN(s.H, p2.data(), fx.data(), -1, 1);               // Δd12 = rhs − (H − Q) Δp12
    gemvN(s.Q, p2.data(), fx.data(), 1, 1);
    pull(out[6], p2, true, 0); pull(out[7], y2, false, 0); pull(out[8], fx, true, 1);
    return 0;
}

// frule!(Δp, Δy, Δd, s, Δf, Δg, Δμ) (differential.jl:5-79); every vector in user order, NULL = 0.
// Returns 0, or -1 when the factorization fails (the reference errors).
int oracle_frule(void* h, const double* Df, const double* Dg, double Dmu, double* Dp, double* Dy, double* Dd) {
    Solver& s = *(Solver*)h;
    const i64 n = s.n, m = s.m;
    double ftol, gtol;
    if (!sens_setup(s, ftol, gtol)) return -1;
    std::vector<double> fx(n), gx(m), px(n, 0.0), yx(m, 0.0), dx(n);
    for (i64 i = 0; i < n; ++i) fx[i] = (Df ? Df[s.P2[i]] : 0.0) * s.pscl[i];
    for (i64 i = 0; i < m; ++i) gx[i] = (Dg ? Dg[s.P1[i]] : 0.0) * s.yscl[i];
    dualshadow_all(s, dx.data());
    for (i64 i = 0; i < n; ++i) { dx[i] *= Dmu; fx[i] += dx[i]; }
    solvekkt(s, never, never, px.data(), yx.data(), s.H, fx.data(), gx.data(), false, ftol, gtol,
             s.set.refine_stall_tol, s.set.refine_max_iter, s.set.newton_max_iter, 1);
    gemvN(s.H, px.data(), dx.data(), -1, 1);           // Δd = Δμ d* − (H − Q) Δp
    gemvN(s.Q, px.data(), dx.data(), 1, 1);
    for (i64 i = 0; i < n; ++i) { Dp[s.P2[i]] = px[i] * s.pscl[i]; Dd[s.P2[i]] = dx[i] / s.pscl[i]; }
    for (i64 i = 0; i < m; ++i) Dy[s.P1[i]] = yx[i] * s.yscl[i];
    return 0;
}

// rrule!(Δf, Δg, s, Δp, Δy, Δd) (differential.jl:263-334); *Dmu = the μ cotangent
int oracle_rrule(void* h, const double* Dp, const double* Dy, const double* Dd, double* Df, double* Dg, double* Dmu) {
    Solver& s = *(Solver*)h;
    const i64 n = s.n, m = s.m;
    double ftol, gtol;
    if (!sens_setup(s, ftol, gtol)) return -1;
    std::vector<double> px(n), dx(n), yx(m), fx(n, 0.0), gx(m, 0.0);
    for (i64 i = 0; i < n; ++i) {
        px[i] = (Dp ? Dp[s.P2[i]] : 0.0) * s.pscl[i];
        dx[i] = (Dd ? Dd[s.P2[i]] : 0.0) / s.pscl[i];
    }
    for (i64 i = 0; i < m; ++i) yx[i] = (Dy ? Dy[s.P1[i]] : 0.0) * -s.yscl[i];
    gemvN(s.H, dx.data(), px.data(), -1, 1);           // Δp −= (H − Q) Δd
    gemvN(s.Q, dx.data(), px.data(), 1, 1);
    solvekkt(s, never, never, fx.data(), gx.data(), s.H, px.data(), yx.data(), false, ftol, gtol,
             s.set.refine_stall_tol, s.set.refine_max_iter, s.set.newton_max_iter, 1);
    for (i64 i = 0; i < n; ++i) dx[i] += fx[i];         // λd = Δd + λp
    for (i64 i = 0; i < n; ++i) Df[s.P2[i]] = fx[i] * s.pscl[i];
    for (i64 i = 0; i < m; ++i) Dg[s.P1[i]] = -gx[i] * s.yscl[i];
    dualshadow_all(s, px.data());
    *Dmu = vdot(dx.data(), px.data(), n);
    return 0;
}

int oracle_step(void* h) { return step(*(Solver*)h); }

int oracle_solve(void* h) {
    Solver& s = *(Solver*)h;
    int status = CONTINUE;
    while (status == CONTINUE) status = step(s);
    return status;
}

// result(s, status)  (solver/ipm.jl:30-74).  scal = {mu, pres, dres, pobj, dobj}.
int oracle_result(void* h, int status, double* p, double* d, double* y, double* scal, int32_t* niter, int32_t* nsolve) {
    Solver& s = *(Solver*)h;
    i64 n = s.n, m = s.m;
    const double NaN = std::numeric_limits<double>::quiet_NaN();
    double mu = NaN, pres = NaN, dres = NaN, pobj = NaN, dobj = NaN;
    bool infeas = status == PRIMAL_INFEASIBLE || status == NEAR_PRIMAL_INFEASIBLE ||
                  status == DUAL_INFEASIBLE || status == NEAR_DUAL_INFEASIBLE;
    if (!(infeas || s.hist.empty())) {
        residuals(s);
        double pQp = bdot(s.p.data(), s.Q, s.p.data());
        pobj = pQp / 2 - vdot(s.f.data(), s.p.data(), n);
        dobj = vdot(s.g.data(), s.y.data(), m) - pQp / 2;
        mu = s.nu == 0 ? NaN : vdot(s.p.data(), s.d.data(), n) / (double)s.nu;
        pres = gnorm(s, s.Dg.data());
        dres = fnorm(s, s.Df.data());
    }
    for (i64 i = 0; i < n; ++i) { p[s.P2[i]] = s.p[i] * s.pscl[i]; d[s.P2[i]] = s.d[i] / s.pscl[i]; }
    for (i64 i = 0; i < m; ++i) y[s.P1[i]] = s.y[i] * s.yscl[i];
    scal[0] = mu; scal[1] = pres; scal[2] = dres; scal[3] = pobj; scal[4] = dobj;
    i64 ni = 0, ns = 0;
    for (auto& r : s.hist) { ni++; ns += (i64)(r.piter + r.ppass + r.citer + r.cpass); }
    *niter = (int32_t)ni; *nsolve = (int32_t)ns;
    return 0;
}

int oracle_history(void* h, ob_row* rows, int32_t cap) {
    Solver& s = *(Solver*)h;
    int32_t k = 0;
    for (auto& r : s.hist) { if (k >= cap) break; rows[k++] = r; }
    return (int32_t)s.hist.size();
}

// section timers, seconds: scale, initkkt, predictor, corrector, maxsteps, exact-solve
int oracle_timers(void* h, double* t) {
    Solver& s = *(Solver*)h;
    t[0] = s.tm.scale; t[1] = s.tm.initkkt; t[2] = s.tm.predictor; t[3] = s.tm.corrector;
    t[4] = s.tm.maxsteps; t[5] = s.tm.solve;
    return 0;
}

// the solver-frame vertex order (0-based user vertex per solver vertex) and front partition,
// for cross-checking the product's host symbolic analysis
int oracle_symbolic(void* h, int64_t* nfront, int64_t* res0, int64_t* nres, int64_t* nsep, int64_t* parent, int64_t cap) {
    Solver& s = *(Solver*)h;
    *nfront = s.S.nfront;
    for (i64 f = 0; f < s.S.nfront && f < cap; ++f) {
        res0[f] = s.S.res0[f]; nres[f] = s.S.nres[f]; nsep[f] = (i64)s.S.sep[f].size(); parent[f] = s.S.parent[f];
    }
    return 0;
}

int64_t oracle_nfactor_retry(void* h) { return ((Solver*)h)->nfactor_retry; }

// TDC cone primitives at a point x (for the known-answer tests): out = [grad(3), hess(9, from the
// pivoted factor), third(9, along u), dual shadow d*(3), primal shadow of d*(3), det chain d1..d4,
// two-word log(x1/x2) (2)], returns the tdfact flag
// Tunçel scaling block at (p, d) and the certified steps along (Δp, Δd): out = [M(9), p*(3), d*(3),
// τp, τd], returns the scale flag
int oracle_tdc_scale_step(int kind, double alpha, const double* p, const double* d, const double* Dp,
                          const double* Dd, double* out) {
    TD c{kind, alpha};
    double C[19] = {0};
    tdinitcache(c, C);
    double H[9] = {0}, spsd = 0;
    bool ok = tdscale(c, H, p, d, C, spsd);
    for (int i = 0; i < 9; ++i) out[i] = H[i];
    double sp[3], C2[19] = {0};
    tdprimalshadow(c, sp, d, C2);
    for (int i = 0; i < 3; ++i) { out[9 + i] = sp[i]; out[12 + i] = C[TD_SD + i]; }
    double tp, td;
    tdmaxsteps(c, p, Dp, d, Dd, C, tp, td);
    out[15] = tp; out[16] = td;
    return ok ? 1 : 0;
}

int oracle_tdc_eval(int kind, double alpha, const double* x, const double* u, double* out) {
    TD c{kind, alpha};
    double C[19] = {0};
    tdinitcache(c, C);
    tddet(c, C, x);
    double g[3];
    tdbarrgrad(c, g, x, C);
    bool ok = tdfact(c, C + TD_L, x, C);
    double H[9];
    for (int j = 0; j < 3; ++j) {
        double e[3] = {0, 0, 0}, col[3];
        e[j] = 1;
        tdhessmul(col, C + TD_L, e);
        for (int i = 0; i < 3; ++i) H[i + 3 * j] = col[i];
    }
    double D[9];
    tdbarrthird(c, D, x, u, C);
    double sd[3], sp[3];
    tddualshadow(c, sd, x, C);
    double C2[19] = {0};
    tdprimalshadow(c, sp, sd, C2);
    for (int i = 0; i < 3; ++i) out[i] = g[i];
    for (int i = 0; i < 9; ++i) out[3 + i] = H[i];
    for (int i = 0; i < 9; ++i) out[12 + i] = D[i];
    for (int i = 0; i < 3; ++i) { out[21 + i] = sd[i]; out[24 + i] = sp[i]; }
    out[27] = C[TD_D1]; out[28] = C[TD_D2]; out[29] = C[TD_D3]; out[30] = C[TD_D4];
    DD l = twolograt(x[0], x[1]);
    out[31] = l.h; out[32] = l.l;
    return ok ? 1 : 0;
}
// Semidefinite cone primitives on svec vectors of length n = d(d+1)/2 (known-answer tests):
// H (n×n) += W ⊗ₛ W and the cache [R | S | s] at (p, d), ⟨p*, d*⟩, the corrector along (Δp, Δd)
// and the zero corrector at σμ, the steps τp/τd, and the shadow X⁻¹ of p.  Returns bit 0 = scale
// succeeded, bit 1 = shadow succeeded.
int oracle_sdp_probe(int64_t n, const double* p, const double* d, const double* Dp, const double* Dd, double sm,
                     double* H, double* cache, double* spsd, double* r, double* r0, double* steps, double* shp) {
    std::vector<double> work(std::max<int64_t>(sdp_workspacesize(n), 1));
    bool ok = sdp_scale(H, n, cache, p, d, work.data(), *spsd);
    int flags = ok ? 1 : 0;
    if (ok) {
        sdp_corr(r, cache, Dp, Dd, sm, n, work.data());
        sdp_corr0(r0, cache, sm, n, work.data());
        double tp, td;
        cone_maxsteps(CONE_SDP, 0.0, n, p, Dp, d, Dd, cache, work.data(), &tp, &td);
        steps[0] = tp; steps[1] = td;
    }
    if (sdp_shadow(shp, p, n, work.data())) flags |= 2;
    return flags;
}

// smallest eigenvalue of the symmetric d×d M (column-major): out[0] through the tridiagonal
// Laguerre path capped at lmax, out[1] through the analytic path (d ≤ 3 only); and the Jacobi SVD
// of A: U (d×d), s (d); returns the SVD's convergence flag
int oracle_sdp_eig(int d, const double* M, double lmax, const double* A, double* out, double* U, double* sv) {
    std::vector<double> W(M, M + (size_t)d * d), a(d), b(std::max(d, 1));
    out[0] = sdp_eigminsturm(W.data(), a.data(), b.data(), d, lmax);
    out[1] = d <= 3 ? sdp_eigmin_small(M, d) : NAN;
    std::copy(A, A + (size_t)d * d, U);
    return sdp_svdjacobi(U, sv, d) ? 1 : 0;
}

int64_t oracle_nfallback(void* h) { return ((Solver*)h)->nfallback; }
int64_t oracle_nfp32(void* h) { return ((Solver*)h)->nfp32; }

void oracle_destroy(void* h) { delete (Solver*)h; }

}  // extern "C"
