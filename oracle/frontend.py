"""ORACLE — test infrastructure only.

Pure-Python restatement of the reference's problem front-end and host symbolic steps, used as
the independent checker of the product's C++ host code (bit-exact integer comparison) and to
feed block-form problems to the FP64 oracle.  Paths cited are inside the Mumblebee.jl project.

  * dropoffdz, colcompress, colpartition, IPMProblem(CSC…)   src/IPM/src/ipm/problem.jl:84-349
  * twins (exact partition refinement)                          src/BlockSparseArrays/src/compress.jl:9-116
  * twins (cosine-τ row similarity)                             src/BlockSparseArrays/src/compress.jl:134-265
  * compress2                                                   src/BlockSparseArrays/src/compress.jl:359-483
  * minimum_degree: the elimination ordering.  The reference takes it from CliqueTrees
    (`symbolic(weights, graph; alg)`, src/IPM/src/kkt/kkt.jl:36), which is not vendored; this
    restates the classical minimum-degree algorithm (Tinney–Walker / Rose) on the weighted
    vertex graph with the tie rule "smallest vertex index".  Parity with CliqueTrees is
    unpinned.

Indices returned by the block-form routines are 1-based, like BlockSparseMatrix.
"""
from __future__ import annotations

import numpy as np
import scipy.sparse as sp

CONE_FREE, CONE_POS, CONE_SOC, CONE_SDP, CONE_EXP, CONE_POW = 0, 1, 2, 3, 4, 5


def dropoffdz(Q: sp.csc_matrix) -> sp.csc_matrix:
    """problem.jl:133-186 — drop zero off-diagonals, keep (or insert) every diagonal entry."""
    Q = sp.csc_matrix(Q)
    Q.sort_indices()
    n = Q.shape[0]
    colptr = [0]
    rows, vals = [], []
    for j in range(n):
        iprv = -1
        for p in range(Q.indptr[j], Q.indptr[j + 1]):
            i = int(Q.indices[p]); x = float(Q.data[p])
            if x != 0 and iprv < j < i:
                rows.append(j); vals.append(0.0); iprv = j
            if x != 0 or i == j:
                rows.append(i); vals.append(x); iprv = i
        if iprv < j:
            rows.append(j); vals.append(0.0)
        colptr.append(len(rows))
    return sp.csc_matrix((np.array(vals, dtype=np.float64), np.array(rows, dtype=np.int64),
                          np.array(colptr, dtype=np.int64)), shape=(n, n))


def twins_exact(nout: int, nvtx: int, xsrc, tgt):
    """compress.jl:28-116.  Rows (1..nout) with identical column patterns, by partition
    refinement over the columns.  `xsrc`/`tgt` are a 0-based CSC (colptr, rowval).  Returns
    (nsv, xptr, perm), 1-based, in the reference's exact set and element order."""
    var = [0] * (nout + 2)          # doubles as the free list's `next`
    svar = [0] * (nout + 1)
    flag = [0] * (nout + 1)
    card = [0] * (nout + 1)
    head = [0] * (nout + 1)
    prev = [0] * (nout + 1)
    nxt = [0] * (nout + 1)
    new = [0]

    def free_prepend(seq):
        if len(seq):
            h = new[0]
            i = seq[0]; new[0] = i
            for j in seq[1:]:
                var[i] = j; i = j
            var[i] = h

    def free_popfirst():
        i = new[0]; new[0] = var[i]; return i

    def free_pushfirst(i):
        var[i] = new[0]; new[0] = i

    def set_pushfirst(s, i):
        n = nxt[i] = head[s]
        head[s] = i
        if n > 0:
            prev[n] = i

    def set_delete(s, i):
        h = head[s]; n = nxt[i]
        if i == h:
            head[s] = n
        else:
            p = prev[i]; nxt[p] = n
            if n > 0:
                prev[n] = p

    def set_prepend(s, seq):
        if len(seq):
            i = seq[0]; h = head[s]; head[s] = i
            for j in seq[1:]:
                prev[j] = i; nxt[i] = j; i = j
            nxt[i] = h

    nsv = 0
    free_prepend(list(range(1, nout + 1)))
    if nout > 0:
        s = free_popfirst(); nsv += 1
        set_prepend(s, list(range(1, nout + 1))); card[s] = nout
        for i in range(1, nout + 1):
            svar[i] = s
    for j in range(1, nvtx + 1):
        for e in range(xsrc[j - 1], xsrc[j]):
            i = int(tgt[e]) + 1
            s = svar[i]
            if flag[s] < j:
                flag[s] = j
                if card[s] > 1:
                    set_delete(s, i); card[s] -= 1
                    var[s] = i
                    ns = svar[i] = free_popfirst(); nsv += 1
                    set_pushfirst(ns, i); card[ns] += 1
            else:
                set_delete(s, i); card[s] -= 1
                k = var[s]
                ns = svar[i] = svar[k]
                set_pushfirst(ns, i); card[ns] += 1
                if head[s] == 0:
                    free_pushfirst(s); nsv -= 1
    t = 1; p = 1
    xptr = [0] * (nout + 2)
    perm = [0] * (nout + 1)
    xptr[t] = p
    for s in range(1, nout + 1):
        if head[s] == 0:
            continue
        i = head[s]
        while i > 0:
            svar[i] = t
            perm[p] = i; p += 1
            i = nxt[i]
        t += 1; xptr[t] = p
    return nsv, np.array(xptr[1:nsv + 2], dtype=np.int64), np.array(perm[1:nout + 1], dtype=np.int64)


def twins_cosine(A: sp.csc_matrix, tau: float):
    """compress.jl:169-265.  Rows of A (nout x nvtx) whose patterns have cosine >= tau with the
    first row of their part.  Returns (nb, xptr, perm), 1-based."""
    A = sp.csc_matrix(A); A.sort_indices()
    At = sp.csc_matrix(A.T); At.sort_indices()
    nout = A.shape[0]
    xrow, cadj = At.indptr, At.indices
    xcol, radj = A.indptr, A.indices
    adjmap = [0] * (nout + 1)
    cosine = [0] * (nout + 1)
    degree = [0] * (nout + 1)
    for i in range(1, nout + 1):
        degree[i] = int(xrow[i] - xrow[i - 1])
    nb = 0
    for i in range(1, nout + 1):
        if adjmap[i] != 0:
            continue
        nb += 1; adjmap[i] = nb
        lst = []
        for e in range(xrow[i - 1], xrow[i]):
            j = int(cadj[e]) + 1
            for f in range(xcol[j] - 1, xcol[j - 1] - 1, -1):
                k = int(radj[f]) + 1
                if not (k > i):
                    break
                if adjmap[k] == 0:
                    if cosine[k] == 0:
                        lst.insert(0, k)
                    cosine[k] += 1
        for k in lst:
            c = float(cosine[k]); nzi = float(degree[i]); nzk = float(degree[k])
            if c * c >= tau * tau * nzi * nzk:
                adjmap[k] = nb
            cosine[k] = 0
    xptr = [0] * (nb + 2)
    for i in range(1, nout + 1):
        xptr[adjmap[i] + 1] += 1
    xptr[1] = 1
    for t in range(1, nb + 1):
        xptr[t + 1] += xptr[t]
    cur = list(xptr)
    perm = [0] * (nout + 1)
    for i in range(1, nout + 1):
        t = adjmap[i]
        perm[cur[t]] = i; cur[t] += 1
    return nb, np.array(xptr[1:nb + 2], dtype=np.int64), np.array(perm[1:], dtype=np.int64)


def twins_rows(A: sp.csc_matrix, tau: float = 1.0):
    """twins over the rows of A, dispatching like compress.jl:118-167."""
    A = sp.csc_matrix(A); A.sort_indices()
    if tau == 1.0:
        return twins_exact(A.shape[0], A.shape[1], A.indptr, A.indices)
    return twins_cosine(A, tau)


def colpartition(B, Q, kinds, sizes, params, tau):
    """problem.jl:262-349.  POS columns, then free columns (each group compressed by twins on
    the pattern of [Q; B]), then the other cones in their given order.  Returns
    (nvtx, xcol, perm, cone kinds, cone params), xcol/perm 1-based."""
    ncol = B.shape[1]
    ncolP = sum(s for k, s in zip(kinds, sizes) if k == CONE_POS)
    ncolC = sum(s for k, s in zip(kinds, sizes) if k == CONE_FREE)
    work = [0] * (ncol + 1)
    p = c = r = 1; j = 1
    for k, s in zip(kinds, sizes):
        for _ in range(s):
            if k == CONE_POS:
                work[p] = j; p += 1
            elif k == CONE_FREE:
                work[ncolP + c] = j; c += 1
            else:
                work[ncolP + ncolC + r] = j; r += 1
            j += 1
    indP = [w - 1 for w in work[1:ncolP + 1]]
    indC = [w - 1 for w in work[ncolP + 1:ncolP + ncolC + 1]]
    QB = sp.vstack([sp.csc_matrix(Q), sp.csc_matrix(B)]).tocsc()
    XP = sp.csc_matrix(QB[:, indP]); XC = sp.csc_matrix(QB[:, indC])
    nvP, xcP, pmP = twins_rows(sp.csc_matrix(XP.T), tau)
    nvC, xcC, pmC = twins_rows(sp.csc_matrix(XC.T), tau)
    nvR = sum(1 for k in kinds if k not in (CONE_POS, CONE_FREE))
    nvtx = nvP + nvC + nvR
    perm = [0] * (ncol + 1)
    xcol = [0] * (nvtx + 2)
    cone = [0] * (nvtx + 1)
    cpar = [0.0] * (nvtx + 1)
    for jj in range(1, ncolP + 1):
        perm[jj] = work[pmP[jj - 1]]
    for v in range(1, nvP + 1):
        xcol[v] = int(xcP[v - 1]); cone[v] = CONE_POS
    for jj in range(1, ncolC + 1):
        perm[ncolP + jj] = work[ncolP + pmC[jj - 1]]
    for v in range(1, nvC + 1):
        xcol[nvP + v] = ncolP + int(xcC[v - 1]); cone[nvP + v] = CONE_FREE
    for jj in range(ncolP + ncolC + 1, ncol + 1):
        perm[jj] = work[jj]
    r = 1; j = 1
    for k, s, prm in zip(kinds, sizes, params):
        if k not in (CONE_POS, CONE_FREE):
            xcol[nvP + nvC + r] = ncolP + ncolC + j
            cone[nvP + nvC + r] = k; cpar[nvP + nvC + r] = prm
            r += 1; j += s
    xcol[nvtx + 1] = ncol + 1
    return nvtx, xcol, perm, cone, cpar


def colcompress(A, nvtx, xcol, colperm):
    """problem.jl:188-260: the vertex-pattern matrix (m x nvtx) of A's column groups."""
    A = sp.csc_matrix(A); A.sort_indices()
    m = A.shape[0]
    indptr = [0]; indices = []
    for v in range(1, nvtx + 1):
        rows = set()
        for j in range(xcol[v], xcol[v + 1]):
            k = colperm[j] - 1
            rows.update(A.indices[A.indptr[k]:A.indptr[k + 1]].tolist())
        indices.extend(sorted(rows)); indptr.append(len(indices))
    return sp.csc_matrix((np.ones(len(indices)), np.array(indices, dtype=np.int64),
                          np.array(indptr, dtype=np.int64)), shape=(m, nvtx))


def compress2(A, nvtx, nout, xcol, xrow):
    """compress.jl:359-483: block-CSC with dense blocks (explicit zeros), 1-based arrays."""
    A = sp.csc_matrix(A); A.sort_indices()
    nrow, ncol = A.shape
    row = np.zeros(nrow + 1, dtype=np.int64)
    for u in range(1, nout + 1):
        row[xrow[u]:xrow[u + 1]] = u
    xsrc = [0] * (nvtx + 2); tgt = []; xblk = []
    b = 0
    for v in range(1, nvtx + 1):
        xsrc[v] = len(tgt) + 1
        rows = set()
        for j in range(xcol[v], xcol[v + 1]):
            rows.update((A.indices[A.indptr[j - 1]:A.indptr[j]] + 1).tolist())
        t = 0
        for i in sorted(rows):
            u = int(row[i])
            if t < u:
                t = u; tgt.append(u); xblk.append(b + 1)
                b += (xrow[u + 1] - xrow[u]) * (xcol[v + 1] - xcol[v])
    narc = len(tgt)
    xsrc[nvtx + 1] = narc + 1
    xblk.append(b + 1)
    val = np.zeros(b)
    Ad = A.tocsc()
    for v in range(1, nvtx + 1):
        jstrt, jstop = xcol[v], xcol[v + 1] - 1
        for e in range(xsrc[v], xsrc[v + 1]):
            u = tgt[e - 1]; bb = xblk[e - 1] - 1
            istrt, istop = xrow[u], xrow[u + 1] - 1
            for j in range(jstrt, jstop + 1):
                col = Ad.indices[Ad.indptr[j - 1]:Ad.indptr[j]] + 1
                dat = Ad.data[Ad.indptr[j - 1]:Ad.indptr[j]]
                lookup = dict(zip(col.tolist(), dat.tolist()))
                for i in range(istrt, istop + 1):
                    val[bb] = lookup.get(i, 0.0); bb += 1
    return dict(nout=nout, nvtx=nvtx, narc=narc, ncol=ncol, nrow=nrow, nbnz=b,
                xsrc=np.array(xsrc[1:], dtype=np.int64), xcol=np.array(xcol[1:nvtx + 2], dtype=np.int64),
                xrow=np.array(xrow[1:nout + 2], dtype=np.int64), xblk=np.array(xblk, dtype=np.int64),
                tgt=np.array(tgt, dtype=np.int64), val=val)


def ipmproblem_from_csc(Q, B, f, g, mu, kinds, sizes, params=None, compress=1.0):
    """IPMProblem{T,I,V}(Q::SparseMatrixCSC, B::SparseMatrixCSC, f, g, μ, K, s; compress),
    problem.jl:84-127.  Returns the block-form problem dict with P1/P2 (1-based)."""
    m, n = B.shape
    assert Q.shape == (n, n) and len(f) == n and len(g) == m and sum(sizes) == n
    assert 0 < compress <= 1
    params = list(params) if params is not None else [0.0] * len(kinds)
    Q = dropoffdz(Q)
    B = sp.csc_matrix(B); B.eliminate_zeros(); B.sort_indices()
    nvtx, xcol, colperm, cone, cpar = colpartition(B, Q, kinds, sizes, params, compress)
    Bc = colcompress(B, nvtx, xcol, colperm)
    nout, xrow, rowperm = twins_rows(Bc, compress)
    cp = np.array(colperm[1:], dtype=np.int64) - 1
    rp = np.array(rowperm, dtype=np.int64) - 1
    Bp = sp.csc_matrix(sp.csc_matrix(B)[rp, :][:, cp])
    Qp = sp.csc_matrix(sp.csc_matrix(Q)[cp, :][:, cp])
    xrow_full = [0] + list(xrow)
    Bb = compress2(Bp, nvtx, nout, xcol, xrow_full)
    Qb = compress2(Qp, nvtx, nvtx, xcol, xcol)
    return dict(Q=Qb, B=Bb, f=np.asarray(f, dtype=np.float64)[cp], g=np.asarray(g, dtype=np.float64)[rp],
                mu=float(mu), kind=np.array(cone[1:], dtype=np.int32),
                param=np.array(cpar[1:], dtype=np.float64),
                P1=np.array(rowperm, dtype=np.int64), P2=np.array(colperm[1:], dtype=np.int64))


def vertex_graph(prob):
    """Pattern of Q ∪ BᵀB over vertices and the column-count weights (IPM/src/utils.jl:135-145)."""
    B, Q = prob["B"], prob["Q"]
    nv = B["nvtx"]
    adj = [set() for _ in range(nv)]
    rows = [[] for _ in range(B["nout"])]
    for v in range(nv):
        for e in range(B["xsrc"][v] - 1, B["xsrc"][v + 1] - 1):
            rows[B["tgt"][e] - 1].append(v)
    for r in rows:
        for a in r:
            for b in r:
                if a != b:
                    adj[a].add(b)
    for v in range(nv):
        for e in range(Q["xsrc"][v] - 1, Q["xsrc"][v + 1] - 1):
            u = Q["tgt"][e] - 1
            if u != v:
                adj[v].add(u); adj[u].add(v)
    w = np.diff(B["xcol"]).astype(np.int64)
    return adj, w


def minimum_degree(adj, w):
    """Exact minimum (weighted external) degree on the elimination graph, ties to the smallest
    index.  Returns the 0-based elimination order."""
    nv = len(adj)
    if nv == 0:
        return np.zeros(0, dtype=np.int64)
    A = np.zeros((nv, nv), dtype=bool)
    for v, s in enumerate(adj):
        if s:
            A[v, list(s)] = True
    np.fill_diagonal(A, False)
    wv = np.asarray(w, dtype=np.int64)
    alive = np.ones(nv, dtype=bool)
    deg = A.astype(np.int64) @ wv
    order = []
    big = np.iinfo(np.int64).max
    for _ in range(nv):
        d = np.where(alive, deg, big)
        v = int(np.argmin(d))
        order.append(v)
        nb = np.nonzero(A[v] & alive)[0]
        alive[v] = False
        A[v, :] = False; A[:, v] = False
        if len(nb):
            A[np.ix_(nb, nb)] = True
            A[nb, nb] = False
            deg[nb] = A[nb].astype(np.int64) @ wv
    return np.array(order, dtype=np.int64)
