// Host-side symbolic work of the solver (integer and pattern work, done once per problem).
//
//  * the CSC front-end of IPMProblem: dropoffdz, colpartition, colcompress, twins (exact and
//    cosine-τ), compress2  — src/IPM/src/ipm/problem.jl:84-349,
//    src/BlockSparseArrays/src/compress.jl:9-483
//  * selectvtxs / halfselectvtxs (symbkkt's permutation of B and Q)
//    — src/BlockSparseArrays/src/block_sparse_matrix.jl:787-874,1111-1169
//  * the elimination ordering that the reference takes from CliqueTrees.symbolic
//    (src/IPM/src/kkt/kkt.jl:36): minimum weighted external degree on the elimination graph,
//    ties to the smallest vertex index; elimination tree (Liu), postorder, vertex row structures
//    and fundamental supernodes (the fronts of the multifrontal factor).
#pragma once
#include <algorithm>
#include <cstdint>
#include <vector>
#include "mb_internal.h"

namespace mbh {

using i64 = int64_t;

struct BSM {  // 0-based BlockSparseMatrix
    i64 nout = 0, nvtx = 0, narc = 0, ncol = 0, nrow = 0, nbnz = 0;
    std::vector<i64> xsrc, xcol, xrow, xblk, tgt;
    std::vector<double> val;
    i64 ncols(i64 v) const { return xcol[v + 1] - xcol[v]; }
    i64 nrows(i64 u) const { return xrow[u + 1] - xrow[u]; }
};

struct CSC {  // 0-based
    i64 m = 0, n = 0;
    std::vector<i64> colptr, rowval;
    std::vector<double> nzval;
};

// ------------------------------------------------------------------------------- front-end
// problem.jl:133-186
inline CSC dropoffdz(const CSC& Q) {
    CSC R; R.m = Q.m; R.n = Q.n;
    R.colptr.assign(Q.n + 1, 0);
    for (i64 j = 0; j < Q.n; ++j) {
        R.colptr[j] = (i64)R.rowval.size();
        i64 iprv = -1;
        for (i64 p = Q.colptr[j]; p < Q.colptr[j + 1]; ++p) {
            i64 i = Q.rowval[p]; double x = Q.nzval[p];
            if (x != 0 && iprv < j && j < i) { R.rowval.push_back(j); R.nzval.push_back(0.0); iprv = j; }
            if (x != 0 || i == j) { R.rowval.push_back(i); R.nzval.push_back(x); iprv = i; }
        }
        if (iprv < j) { R.rowval.push_back(j); R.nzval.push_back(0.0); }
    }
    R.colptr[Q.n] = (i64)R.rowval.size();
    return R;
}

inline CSC dropzeros(const CSC& A) {
    CSC R; R.m = A.m; R.n = A.n; R.colptr.assign(A.n + 1, 0);
    for (i64 j = 0; j < A.n; ++j) {
        R.colptr[j] = (i64)R.rowval.size();
        for (i64 p = A.colptr[j]; p < A.colptr[j + 1]; ++p)
            if (A.nzval[p] != 0) { R.rowval.push_back(A.rowval[p]); R.nzval.push_back(A.nzval[p]); }
    }
    R.colptr[A.n] = (i64)R.rowval.size();
    return R;
}

inline void sort_csc(CSC& A) {
    std::vector<std::pair<i64, double>> t;
    for (i64 j = 0; j < A.n; ++j) {
        t.clear();
        for (i64 p = A.colptr[j]; p < A.colptr[j + 1]; ++p) t.push_back({A.rowval[p], A.nzval[p]});
        std::sort(t.begin(), t.end(), [](auto& a, auto& b) { return a.first < b.first; });
        for (i64 k = 0; k < (i64)t.size(); ++k) { A.rowval[A.colptr[j] + k] = t[k].first; A.nzval[A.colptr[j] + k] = t[k].second; }
    }
}

// twins over the rows of a pattern given as CSC (xsrc/tgt, 0-based): compress.jl:28-116.
// Returns nsv and, 1-based, xptr[1..nsv+1] and perm[1..nout] (stored 0-indexed in the vectors).
inline i64 twins_exact(i64 nout, i64 nvtx, const std::vector<i64>& xsrc, const std::vector<i64>& tgt,
                       std::vector<i64>& xptr, std::vector<i64>& perm) {
    std::vector<i64> var(nout + 2, 0), svar(nout + 1, 0), flag(nout + 1, 0), card(nout + 1, 0),
        head(nout + 1, 0), prev(nout + 1, 0), nxt(nout + 1, 0);
    i64 fhead = 0;
    auto set_pushfirst = [&](i64 s, i64 i) { i64 n = nxt[i] = head[s]; head[s] = i; if (n > 0) prev[n] = i; };
    auto set_delete = [&](i64 s, i64 i) {
        i64 h = head[s], n = nxt[i];
        if (i == h) head[s] = n;
        else { i64 p = prev[i]; nxt[p] = n; if (n > 0) prev[n] = p; }
    };
    i64 nsv = 0;
    // free list = 1..nout
    if (nout > 0) { fhead = 1; for (i64 i = 1; i < nout; ++i) var[i] = i + 1; var[nout] = 0; }
    if (nout > 0) {
        i64 s = fhead; fhead = var[s]; nsv += 1;
        head[s] = 1;
        for (i64 i = 1; i <= nout; ++i) { if (i > 1) prev[i] = i - 1; nxt[i] = (i < nout) ? i + 1 : 0; svar[i] = s; }
        card[s] = nout;
    }
    for (i64 j = 1; j <= nvtx; ++j) {
        for (i64 e = xsrc[j - 1]; e < xsrc[j]; ++e) {
            i64 i = tgt[e] + 1;
            i64 s = svar[i];
            if (flag[s] < j) {
                flag[s] = j;
                if (card[s] > 1) {
                    set_delete(s, i); card[s] -= 1;
                    var[s] = i;
                    i64 ns = fhead; fhead = var[ns]; svar[i] = ns; nsv += 1;
                    set_pushfirst(ns, i); card[ns] += 1;
                }
            } else {
                set_delete(s, i); card[s] -= 1;
                i64 k = var[s];
                i64 ns = svar[k]; svar[i] = ns;
                set_pushfirst(ns, i); card[ns] += 1;
                if (head[s] == 0) { var[s] = fhead; fhead = s; nsv -= 1; }
            }
        }
    }
    xptr.assign(nsv + 1, 0); perm.assign(nout, 0);
    i64 t = 0, p = 1;
    xptr[0] = 1;
    for (i64 s = 1; s <= nout; ++s) {
        if (head[s] == 0) continue;
        for (i64 i = head[s]; i > 0; i = nxt[i]) { perm[p - 1] = i; ++p; }
        ++t; xptr[t] = p;
    }
    return nsv;
}

// cosine-τ twins over the rows of A (nout x nvtx): compress.jl:169-265
inline i64 twins_cosine(i64 nout, i64 nvtx, const std::vector<i64>& xcol, const std::vector<i64>& radj,
                        double tau, std::vector<i64>& xptr, std::vector<i64>& perm) {
    // row-wise pattern (At)
    std::vector<i64> xrow(nout + 1, 0), cadj(xcol[nvtx]);
    for (i64 e = 0; e < xcol[nvtx]; ++e) xrow[radj[e] + 1]++;
    for (i64 i = 0; i < nout; ++i) xrow[i + 1] += xrow[i];
    { std::vector<i64> c(xrow.begin(), xrow.end() - 1);
      for (i64 j = 0; j < nvtx; ++j) for (i64 e = xcol[j]; e < xcol[j + 1]; ++e) cadj[c[radj[e]]++] = j; }
    std::vector<i64> adjmap(nout + 1, 0), cosine(nout + 1, 0), degree(nout + 1, 0);
    for (i64 i = 1; i <= nout; ++i) degree[i] = xrow[i] - xrow[i - 1];
    i64 nb = 0;
    std::vector<i64> lst;
    for (i64 i = 1; i <= nout; ++i) {
        if (adjmap[i] != 0) continue;
        adjmap[i] = ++nb;
        lst.clear();
        for (i64 e = xrow[i - 1]; e < xrow[i]; ++e) {
            i64 j = cadj[e] + 1;
            for (i64 f = xcol[j] - 1; f >= xcol[j - 1]; --f) {
                i64 k = radj[f] + 1;
                if (!(k > i)) break;
                if (adjmap[k] == 0) { if (cosine[k] == 0) lst.push_back(k); cosine[k] += 1; }
            }
        }
        for (i64 k : lst) {
            double c = (double)cosine[k], nzi = (double)degree[i], nzk = (double)degree[k];
            if (c * c >= tau * tau * nzi * nzk) adjmap[k] = nb;
            cosine[k] = 0;
        }
    }
    std::vector<i64> xp(nb + 2, 0);
    for (i64 i = 1; i <= nout; ++i) xp[adjmap[i] + 1]++;
    xp[1] = 1;
    for (i64 t = 1; t <= nb; ++t) xp[t + 1] += xp[t];
    std::vector<i64> cur(xp);
    perm.assign(nout, 0);
    for (i64 i = 1; i <= nout; ++i) { i64 t = adjmap[i]; perm[cur[t] - 1] = i; cur[t]++; }
    xptr.assign(xp.begin() + 1, xp.begin() + nb + 2);
    return nb;
}

// twins over the rows of a CSC pattern, dispatching like compress.jl:118-167
inline i64 twins_rows(const CSC& A, double tau, std::vector<i64>& xptr, std::vector<i64>& perm) {
    if (tau == 1.0) return twins_exact(A.m, A.n, A.colptr, A.rowval, xptr, perm);
    return twins_cosine(A.m, A.n, A.colptr, A.rowval, tau, xptr, perm);
}

// compress2  (compress.jl:359-483).  xcol/xrow 0-based offsets (nvtx+1 / nout+1).
inline BSM compress2(const CSC& A, i64 nvtx, i64 nout, const std::vector<i64>& xcol, const std::vector<i64>& xrow) {
    BSM R;
    R.nout = nout; R.nvtx = nvtx; R.ncol = A.n; R.nrow = A.m;
    R.xcol = xcol; R.xrow = xrow;
    std::vector<i64> row(A.m), arcpos(nout, -1);
    for (i64 u = 0; u < nout; ++u) for (i64 i = xrow[u]; i < xrow[u + 1]; ++i) row[i] = u;
    R.xsrc.assign(nvtx + 1, 0);
    std::vector<i64> us;
    i64 b = 0;
    for (i64 v = 0; v < nvtx; ++v) {
        R.xsrc[v] = (i64)R.tgt.size();
        us.clear();
        for (i64 j = xcol[v]; j < xcol[v + 1]; ++j)
            for (i64 p = A.colptr[j]; p < A.colptr[j + 1]; ++p) us.push_back(row[A.rowval[p]]);
        std::sort(us.begin(), us.end());
        us.erase(std::unique(us.begin(), us.end()), us.end());
        i64 nc = xcol[v + 1] - xcol[v];
        for (i64 u : us) { R.tgt.push_back(u); R.xblk.push_back(b); b += (xrow[u + 1] - xrow[u]) * nc; }
    }
    R.narc = (i64)R.tgt.size(); R.xsrc[nvtx] = R.narc; R.xblk.push_back(b); R.nbnz = b;
    R.val.assign(b, 0.0);
    for (i64 v = 0; v < nvtx; ++v) {
        for (i64 e = R.xsrc[v]; e < R.xsrc[v + 1]; ++e) arcpos[R.tgt[e]] = e;
        for (i64 j = xcol[v]; j < xcol[v + 1]; ++j)
            for (i64 p = A.colptr[j]; p < A.colptr[j + 1]; ++p) {
                i64 i = A.rowval[p], u = row[i], e = arcpos[u], nr = xrow[u + 1] - xrow[u];
                R.val[R.xblk[e] + (i - xrow[u]) + (j - xcol[v]) * nr] = A.nzval[p];
            }
    }
    return R;
}

// A[rp, cp] for CSC A (rp/cp 0-based "new -> old"), sorted rows
inline CSC permute(const CSC& A, const std::vector<i64>& rp, const std::vector<i64>& cp) {
    std::vector<i64> rinv(A.m);
    for (i64 i = 0; i < A.m; ++i) rinv[rp[i]] = i;
    CSC R; R.m = A.m; R.n = A.n; R.colptr.assign(A.n + 1, 0);
    for (i64 j = 0; j < A.n; ++j) {
        R.colptr[j] = (i64)R.rowval.size();
        i64 oj = cp[j];
        for (i64 p = A.colptr[oj]; p < A.colptr[oj + 1]; ++p) { R.rowval.push_back(rinv[A.rowval[p]]); R.nzval.push_back(A.nzval[p]); }
    }
    R.colptr[A.n] = (i64)R.rowval.size();
    sort_csc(R);
    return R;
}

// ------------------------------------------------------------------------------- symbkkt
// selectvtxs(A, sel)  (block_sparse_matrix.jl:1111-1169)
inline BSM selectvtxs(const BSM& A, const std::vector<i64>& sel) {
    BSM B;
    B.nout = A.nout; B.nrow = A.nrow; B.xrow = A.xrow;
    B.nvtx = (i64)sel.size();
    B.xcol.assign(B.nvtx + 1, 0); B.xsrc.assign(B.nvtx + 1, 0);
    i64 c = 0, ee = 0, bb = 0;
    B.tgt.reserve(A.narc); B.xblk.reserve(A.narc + 1); B.val.reserve(A.val.size());
    for (i64 v = 0; v < B.nvtx; ++v) {
        i64 av = sel[v];
        B.xcol[v] = c; B.xsrc[v] = ee; c += A.ncols(av);
        for (i64 e = A.xsrc[av]; e < A.xsrc[av + 1]; ++e) {
            B.tgt.push_back(A.tgt[e]); B.xblk.push_back(bb); ++ee;
            B.val.insert(B.val.end(), A.val.begin() + A.xblk[e], A.val.begin() + A.xblk[e + 1]);
            bb += A.xblk[e + 1] - A.xblk[e];
        }
    }
    B.xcol[B.nvtx] = c; B.xsrc[B.nvtx] = ee; B.xblk.push_back(bb);
    B.ncol = c; B.narc = ee; B.nbnz = bb;
    return B;
}

// halfselectvtxs(A, sel) with transposed blocks  (block_sparse_matrix.jl:787-874)
inline BSM halfselectvtxs(const BSM& A, const std::vector<i64>& sel) {
    BSM R;
    R.nout = (i64)sel.size(); R.nvtx = A.nout; R.ncol = A.nrow;
    for (i64 av : sel) {
        R.nrow += A.ncols(av);
        for (i64 e = A.xsrc[av]; e < A.xsrc[av + 1]; ++e) { R.narc++; R.nbnz += A.xblk[e + 1] - A.xblk[e]; }
    }
    std::vector<i64> cnt(R.nvtx + 1, 0), bcnt(R.nvtx + 1, 0);
    for (i64 au = 0; au < R.nout; ++au)
        for (i64 e = A.xsrc[sel[au]]; e < A.xsrc[sel[au] + 1]; ++e) { cnt[A.tgt[e] + 1]++; bcnt[A.tgt[e] + 1] += A.xblk[e + 1] - A.xblk[e]; }
    for (i64 v = 0; v < R.nvtx; ++v) { cnt[v + 1] += cnt[v]; bcnt[v + 1] += bcnt[v]; }
    R.xsrc = cnt; R.tgt.assign(R.narc, 0); R.xblk.assign(R.narc + 1, 0); R.val.assign(R.nbnz, 0);
    std::vector<i64> pe(cnt.begin(), cnt.end() - 1), pb(bcnt.begin(), bcnt.end() - 1);
    for (i64 au = 0; au < R.nout; ++au) {
        i64 bv = sel[au], nc = A.ncols(bv);
        for (i64 e = A.xsrc[bv]; e < A.xsrc[bv + 1]; ++e) {
            i64 bu = A.tgt[e], nr = A.nrows(bu);
            i64 ae = pe[bu]++, ab = pb[bu];
            R.tgt[ae] = au; R.xblk[ae] = ab;
            const double* blk = A.val.data() + A.xblk[e];
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

// halfselectvtxs(halfselectvtxs(Q, sel), sel) for a square Q whose only arcs are diagonal blocks:
// the two block transposes cancel, so vertex v takes the diagonal block of sel[v] as it is stored,
// with row and column splits both the sizes of the selected vertices in order
inline bool blockdiag(const BSM& Q) {
    for (i64 v = 0; v < Q.nvtx; ++v)
        for (i64 e = Q.xsrc[v]; e < Q.xsrc[v + 1]; ++e)
            if (Q.tgt[e] != v) return false;
    return Q.nout == Q.nvtx;
}
inline BSM select_blockdiag(const BSM& Q, const std::vector<i64>& sel) {
    BSM R;
    R.nout = R.nvtx = (i64)sel.size();
    R.xcol.assign(R.nvtx + 1, 0); R.xsrc.assign(R.nvtx + 1, 0);
    R.tgt.reserve(Q.narc); R.xblk.reserve(Q.narc + 1); R.val.reserve(Q.val.size());
    i64 c = 0, ee = 0, bb = 0;
    for (i64 v = 0; v < R.nvtx; ++v) {
        const i64 w = sel[v];
        R.xcol[v] = c; R.xsrc[v] = ee; c += Q.ncols(w);
        for (i64 e = Q.xsrc[w]; e < Q.xsrc[w + 1]; ++e) {
            R.tgt.push_back(v); R.xblk.push_back(bb); ++ee;
            R.val.insert(R.val.end(), Q.val.begin() + Q.xblk[e], Q.val.begin() + Q.xblk[e + 1]);
            bb += Q.xblk[e + 1] - Q.xblk[e];
        }
    }
    R.xcol[R.nvtx] = c; R.xsrc[R.nvtx] = ee; R.xblk.push_back(bb);
    R.xrow = R.xcol;
    R.ncol = R.nrow = c; R.narc = ee; R.nbnz = bb;
    return R;
}

// vertex adjacency: pattern of Q ∪ BᵀB  (IPM/src/utils.jl:135-145 weightedgraph), sorted lists
inline std::vector<std::vector<i64>> vertex_graph(const BSM& B, const BSM& Q) {
    i64 nv = B.nvtx;
    if (nv > 0 && nv <= 8192) {
        // bitset form: a vertex's neighbours are the union of its rows' vertex sets
        const i64 W = (nv + 63) / 64;
        std::vector<uint64_t> rb((size_t)B.nout * W, 0), ab((size_t)W);
        for (i64 v = 0; v < nv; ++v)
            for (i64 e = B.xsrc[v]; e < B.xsrc[v + 1]; ++e) rb[(size_t)B.tgt[e] * W + (v >> 6)] |= 1ull << (v & 63);
        std::vector<std::vector<i64>> adj(nv);
        for (i64 v = 0; v < nv; ++v) {
            std::fill(ab.begin(), ab.end(), 0ull);
            for (i64 e = B.xsrc[v]; e < B.xsrc[v + 1]; ++e) {
                const uint64_t* r = rb.data() + (size_t)B.tgt[e] * W;
                for (i64 q = 0; q < W; ++q) ab[q] |= r[q];
            }
            ab[v >> 6] |= 1ull << (v & 63);
            for (i64 e = Q.xsrc[v]; e < Q.xsrc[v + 1]; ++e) { i64 u = Q.tgt[e]; ab[u >> 6] |= 1ull << (u & 63); }
            for (i64 q = 0; q < W; ++q) { uint64_t x = ab[q]; while (x) { int b = __builtin_ctzll(x); x &= x - 1; adj[v].push_back(q * 64 + b); } }
        }
        bool extra = false;            // Q pattern is used symmetrically
        for (i64 v = 0; v < nv; ++v)
            for (i64 e = Q.xsrc[v]; e < Q.xsrc[v + 1]; ++e) { i64 u = Q.tgt[e]; if (u != v) { adj[u].push_back(v); extra = true; } }
        if (extra)   // the bitset lists are sorted and unique already
            for (auto& a : adj) { std::sort(a.begin(), a.end()); a.erase(std::unique(a.begin(), a.end()), a.end()); }
        return adj;
    }
    std::vector<std::vector<i64>> rows(B.nout), adj(nv);
    for (i64 v = 0; v < nv; ++v) for (i64 e = B.xsrc[v]; e < B.xsrc[v + 1]; ++e) rows[B.tgt[e]].push_back(v);
    std::vector<i64> mark(nv, -1);
    for (i64 v = 0; v < nv; ++v) {
        mark[v] = v;
        for (i64 e = B.xsrc[v]; e < B.xsrc[v + 1]; ++e)
            for (i64 w : rows[B.tgt[e]]) if (mark[w] != v) { mark[w] = v; adj[v].push_back(w); }
        for (i64 e = Q.xsrc[v]; e < Q.xsrc[v + 1]; ++e) {
            i64 u = Q.tgt[e];
            if (mark[u] != v) { mark[u] = v; adj[v].push_back(u); }
        }
    }
    // Q pattern is used symmetrically
    for (i64 v = 0; v < nv; ++v)
        for (i64 e = Q.xsrc[v]; e < Q.xsrc[v + 1]; ++e) { i64 u = Q.tgt[e]; if (u != v) adj[u].push_back(v); }
    for (auto& a : adj) { std::sort(a.begin(), a.end()); a.erase(std::unique(a.begin(), a.end()), a.end()); }
    return adj;
}

// Minimum weighted external degree on the elimination graph, ties to the smallest index; exact
// incremental degree updates on a bitset graph, and a closed form once the remaining graph is a
// clique (every remaining degree then drops by the same amount per elimination, so the order is by
// weight descending, index ascending).  Returns the elimination order (0-based vertices).
inline std::vector<i64> minimum_degree(const std::vector<std::vector<i64>>& adj, const std::vector<i64>& w) {
    const i64 nv = (i64)adj.size();
    std::vector<i64> order; order.reserve(nv);
    if (nv == 0) return order;
    const i64 W = (nv + 63) / 64;
    std::vector<uint64_t> bits((size_t)nv * W, 0);
    auto row = [&](i64 v) { return bits.data() + (size_t)v * W; };
    std::vector<i64> deg(nv, 0), cnt(nv, 0);
    std::vector<char> alive(nv, 1);
    i64 S = 0;
    for (i64 v = 0; v < nv; ++v)
        for (i64 u : adj[v]) if (u != v) { row(v)[u >> 6] |= 1ull << (u & 63); }
    for (i64 v = 0; v < nv; ++v) {
        uint64_t* r = row(v);
        for (i64 k = 0; k < W; ++k) { uint64_t x = r[k]; while (x) { int b = __builtin_ctzll(x); x &= x - 1; deg[v] += w[k * 64 + b]; cnt[v]++; } }
        S += cnt[v];
    }
    std::vector<uint64_t> nb(W);
    std::vector<i64> nbl;
    i64 k = nv;
    while (k > 0) {
        if (S == k * (k - 1)) {  // the remaining graph is a clique
            std::vector<i64> rest;
            for (i64 v = 0; v < nv; ++v) if (alive[v]) rest.push_back(v);
            std::stable_sort(rest.begin(), rest.end(), [&](i64 a, i64 b) { return deg[a] < deg[b]; });
            order.insert(order.end(), rest.begin(), rest.end());
            break;
        }
        i64 v = -1;
        for (i64 u = 0; u < nv; ++u) if (alive[u] && (v < 0 || deg[u] < deg[v])) v = u;
        order.push_back(v);
        alive[v] = 0;
        uint64_t* rv = row(v);
        for (i64 q = 0; q < W; ++q) nb[q] = rv[q];
        nbl.clear();
        for (i64 q = 0; q < W; ++q) { uint64_t x = nb[q]; while (x) { int b = __builtin_ctzll(x); x &= x - 1; nbl.push_back(q * 64 + b); } }
        S -= cnt[v] + (i64)nbl.size();
        for (i64 u : nbl) {
            uint64_t* ru = row(u);
            ru[v >> 6] &= ~(1ull << (v & 63));
            cnt[u] -= 1; deg[u] -= w[v];
            for (i64 q = 0; q < W; ++q) {
                uint64_t nw = nb[q] & ~ru[q];
                if (q == (u >> 6)) nw &= ~(1ull << (u & 63));
                if (!nw) continue;
                ru[q] |= nw;
                while (nw) { int b = __builtin_ctzll(nw); nw &= nw - 1; deg[u] += w[q * 64 + b]; cnt[u]++; S++; }
            }
        }
        for (i64 q = 0; q < W; ++q) rv[q] = 0;
        cnt[v] = 0;
        --k;
    }
    return order;
}

// ------------------------------------------------------------------------------- fronts
struct Fronts {
    i64 nfront = 0;
    std::vector<i64> postperm;           // vertex order after postordering (indices into the input order)
    std::vector<i64> fvtx;               // front f owns (postordered) vertices fvtx[f] .. fvtx[f+1]-1
    std::vector<i64> res0, nres, parent;
    std::vector<std::vector<i64>> sep;   // scalar separator rows, ascending
    std::vector<std::vector<i64>> rel;   // positions of sep rows in the parent's row list
    std::vector<i64> fptr;               // storage offsets of the fronts (order nres+nsep, leading dimension front_ld)
    i64 fsize = 0;
    std::vector<i64> vfront;             // per postordered vertex
};

inline void etree(const std::vector<std::vector<i64>>& adj, std::vector<i64>& par) {
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

// adj0: vertex graph in elimination order (vertex k = k-th eliminated); w0: column counts
inline Fronts analyze(const std::vector<std::vector<i64>>& adj0, const std::vector<i64>& w0) {
    i64 n = (i64)adj0.size();
    std::vector<i64> par0;
    etree(adj0, par0);
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
    std::vector<std::vector<i64>> sv(n), kids(n);
    for (i64 v = 0; v < n; ++v) if (par[v] >= 0) kids[par[v]].push_back(v);
    std::vector<i64> mark(n, -1);
    for (i64 v = 0; v < n; ++v) {
        auto& s = sv[v];
        for (i64 u : adj[v]) if (u > v && mark[u] != v) { mark[u] = v; s.push_back(u); }
        for (i64 c : kids[v]) for (i64 u : sv[c]) if (u > v && mark[u] != v) { mark[u] = v; s.push_back(u); }
        std::sort(s.begin(), s.end());
    }
    Fronts S;
    S.postperm = post;
    S.vfront.assign(n, -1);
    // relaxed supernodes: v joins the front of its child v-1 (its last child in postorder, so the
    // columns stay contiguous) when the explicit zeros this adds to the front's columns stay within
    // 5% of the merged front's lower-triangle entries; with no zero added this is the maximal
    // supernode.  struct(v-1) ⊆ {v} ∪ struct(v) (etree property), so the merged front's rows hold
    // every column's structure and the added entries are zeros of L.
    std::vector<i64> ssw(n, 0);   // scalar rows of struct(v)
    for (i64 v = 0; v < n; ++v) for (i64 u : sv[v]) ssw[v] += w[u];
    i64 fcols = 0, fzeros = 0;    // the open front: scalar columns, zeros added so far
    for (i64 v = 0; v < n; ++v) {
        bool merge = false;
        if (v > 0 && par[v - 1] == v) {
            const i64 add = fcols * (w[v] + ssw[v] - ssw[v - 1]);
            const i64 cols = fcols + w[v], nfm = cols + ssw[v];
            const double entries = (double)cols * (double)nfm - 0.5 * (double)cols * (double)(cols - 1);
            merge = add == 0 || (double)(fzeros + add) <= 0.05 * entries;
            if (merge) { fzeros += add; fcols = cols; }
        }
        if (merge) S.vfront[v] = S.vfront[v - 1];
        else { S.vfront[v] = S.nfront++; S.fvtx.push_back(v); fcols = w[v]; fzeros = 0; }
    }
    S.fvtx.push_back(n);
    std::vector<i64> vcol(n + 1, 0);
    for (i64 v = 0; v < n; ++v) vcol[v + 1] = vcol[v] + w[v];
    i64 ncol = vcol[n];
    S.res0.resize(S.nfront); S.nres.resize(S.nfront); S.sep.resize(S.nfront); S.parent.assign(S.nfront, -1);
    for (i64 f = 0; f < S.nfront; ++f) {
        i64 v0 = S.fvtx[f], v1 = S.fvtx[f + 1];
        S.res0[f] = vcol[v0]; S.nres[f] = vcol[v1] - vcol[v0];
        for (i64 u : sv[v1 - 1]) for (i64 j = vcol[u]; j < vcol[u + 1]; ++j) S.sep[f].push_back(j);
        i64 pv = par[v1 - 1];
        S.parent[f] = pv < 0 ? -1 : S.vfront[pv];
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
        off += (mb::front_ld(nf) * nf + 31) / 32 * 32;   // column-major, leading dimension front_ld(nf)
    }
    S.fptr[S.nfront] = off; S.fsize = off;
    return S;
}

}  // namespace mbh
