"""Seeded synthetic problem generators for the benchmark workloads.

Each generator returns the reference's native CSC input of
``IPMProblem(Q, B, f, g, μ, K, s; compress)`` (src/IPM/src/ipm/problem.jl:84-127):
``min ½pᵀQp − fᵀp  s.t.  Bp = g,  p ∈ K`` with the cone list given as (kind, size, param).

Standard-form data (min cᵀx s.t. Ax = b, x ∈ K) maps to it as Q = 0, B = A, g = b, f = −c, so the
dual slack of the reference, d = Qp − f − Bᵀy, is c − Aᵀy.
"""
from __future__ import annotations

import numpy as np
import scipy.sparse as sp

CONE_FREE, CONE_POS, CONE_SOC, CONE_SDP, CONE_EXP, CONE_POW = 0, 1, 2, 3, 4, 5


def _soc_interior(rng, k):
    u = rng.standard_normal(k - 1)
    t = np.linalg.norm(u) + 1.0 + rng.uniform()
    return np.concatenate([[t], u])


def socp(n=500, m=200, ncone=25, density=0.05, seed=0):
    """Plain SOCP: A sparse with N(0,1) entries at the given density; ``ncone`` second-order
    cones of dimension n/ncone; feasible by construction: x0, s0 in cone interiors
    (t = ‖u‖ + 1 + U(0,1)), y0 ~ N(0,1), b = A x0, c = Aᵀ y0 + s0."""
    rng = np.random.default_rng(seed)
    k = n // ncone
    assert k * ncone == n
    A = sp.random(m, n, density=density, format="csc", random_state=rng,
                  data_rvs=lambda s: rng.standard_normal(s))
    x0 = np.concatenate([_soc_interior(rng, k) for _ in range(ncone)])
    s0 = np.concatenate([_soc_interior(rng, k) for _ in range(ncone)])
    y0 = rng.standard_normal(m)
    b = A @ x0
    c = A.T @ y0 + s0
    Q = sp.csc_matrix((n, n))
    return dict(Q=Q, B=sp.csc_matrix(A), f=-c, g=b, mu=0.0,
                kinds=[CONE_SOC] * ncone, sizes=[k] * ncone, params=[0.0] * ncone,
                name=f"socp n={n} m={m} {ncone}xSOC({k}) density={density} seed={seed}")


def portfolio(n_assets, nfac=10, gamma=1.0, seed=0, rng=None):
    """Long-only factor-model portfolio with a risk budget (lifted form keeps Q and the SOC
    sparse).  Variables p = [x (n, POS); y (nfac, free); s = (t, u, w) (SOC of dim 1+n+nfac)]:

        min  γ (xᵀ D x + yᵀ y) − μᵀ x
        s.t. Fᵀ x − y = 0,  1ᵀ x = 1,  t = σ,  u − D^{1/2} x = 0,  w − y = 0,
             x ≥ 0,  ‖(u, w)‖ ≤ t.

    Covariance F Fᵀ + D with F (n x nfac) N(0,1), D ~ U(0.1, 1); expected returns μ ~ N(0, 1)/10;
    σ = 0.8 · risk of the equal-weight portfolio, so the risk bound binds on most instances."""
    rng = rng if rng is not None else np.random.default_rng(seed)
    n, k = n_assets, nfac
    F = rng.standard_normal((n, k))
    D = rng.uniform(0.1, 1.0, n)
    mu_r = rng.standard_normal(n) / 10
    xe = np.full(n, 1.0 / n)
    sigma = 0.8 * np.sqrt(xe @ (D * xe) + np.sum((F.T @ xe) ** 2))
    nx, ny, ns = n, k, 1 + n + k
    N = nx + ny + ns
    ox, oy, os_ = 0, nx, nx + ny
    Qd = np.zeros(N)
    Qd[ox:ox + nx] = 2 * gamma * D
    Qd[oy:oy + ny] = 2 * gamma
    Q = sp.diags(Qd).tocsc()
    f = np.zeros(N)
    f[ox:ox + nx] = mu_r
    rows, cols, vals = [], [], []
    g = []
    r = 0
    for j in range(k):                       # Fᵀx − y = 0
        rows += [r] * n; cols += list(range(ox, ox + nx)); vals += list(F[:, j])
        rows.append(r); cols.append(oy + j); vals.append(-1.0)
        g.append(0.0); r += 1
    rows += [r] * n; cols += list(range(ox, ox + nx)); vals += [1.0] * n   # budget
    g.append(1.0); r += 1
    rows.append(r); cols.append(os_); vals.append(1.0); g.append(sigma); r += 1   # t = σ
    sD = np.sqrt(D)
    for i in range(n):                       # u_i − √D_i x_i = 0
        rows += [r, r]; cols += [os_ + 1 + i, ox + i]; vals += [1.0, -sD[i]]
        g.append(0.0); r += 1
    for j in range(k):                       # w_j − y_j = 0
        rows += [r, r]; cols += [os_ + 1 + n + j, oy + j]; vals += [1.0, -1.0]
        g.append(0.0); r += 1
    B = sp.csc_matrix((vals, (rows, cols)), shape=(r, N))
    kinds = [CONE_POS] * nx + [CONE_FREE] * ny + [CONE_SOC]
    sizes = [1] * nx + [1] * ny + [ns]
    return dict(Q=Q, B=B, f=f, g=np.array(g), mu=0.0, kinds=kinds, sizes=sizes,
                params=[0.0] * len(kinds), name=f"portfolio n={n} nfac={k} seed={seed}")


def portfolio_batch(count=4096, nmin=50, nmax=400, nfac=10, seed=0):
    """``count`` portfolio instances with n_assets ~ U[nmin, nmax] (integers), one stream."""
    rng = np.random.default_rng(seed)
    sizes = rng.integers(nmin, nmax + 1, size=count)
    return [portfolio(int(s), nfac=nfac, rng=np.random.default_rng([seed, i])) for i, s in enumerate(sizes)]


def _exp_interior(rng):
    x1, x2 = rng.uniform(0.5, 2.0, 2)
    return [x1, x2, x2 * np.log(x1 / x2) - rng.uniform(0.1, 1.0)]


def _exp_dual_interior(rng):
    z1, mz3 = rng.uniform(0.5, 2.0, 2)
    z2 = mz3 * (np.log(mz3 / z1) - 1.0) + rng.uniform(0.1, 1.0)
    return [z1, z2, -mz3]


def _pow_interior(rng, a):
    x1, x2 = rng.uniform(0.5, 2.0, 2)
    return [x1, x2, rng.uniform(-0.9, 0.9) * x1 ** a * x2 ** (1 - a)]


def _pow_dual_interior(rng, a):
    s1, s2 = rng.uniform(0.5, 2.0, 2)
    return [s1, s2, rng.uniform(-0.9, 0.9) * (s1 / a) ** a * (s2 / (1 - a)) ** (1 - a)]


def exppow(nexp=3000, npow=1000, nfree=4000, npos=4000, m=5000, density=0.001, seed=0, determined_free=True):
    """Exponential / power cone problem (defaults: n = 20000, m = 5000): ``nexp`` exponential cones and
    ``npow`` 3-d power cones with α ~ U(0.2, 0.8), plus free and nonnegative columns (the
    log-sum-exp / relative-entropy epigraph variables), A sparse N(0,1) at the given density.
    Feasible by construction: x0 in the cone interior, s0 in the dual-cone interior (0 on free
    columns), y0 ~ U(-1, 1), b = A x0, c = Aᵀ y0 + s0.  Free columns each carry an entry in a row of
    their own, so the free variables are determined by the equalities; ``determined_free=False``
    keeps the random pattern alone (the same random stream up to that point), whose free block
    may be structurally rank deficient."""
    rng = np.random.default_rng(seed)
    alphas = rng.uniform(0.2, 0.8, npow)
    kinds, sizes, params, x0, s0 = [], [], [], [], []
    for _ in range(nexp):
        kinds.append(CONE_EXP); sizes.append(3); params.append(0.0)
        x0 += _exp_interior(rng); s0 += _exp_dual_interior(rng)
    for a in alphas:
        kinds.append(CONE_POW); sizes.append(3); params.append(float(a))
        x0 += _pow_interior(rng, a); s0 += _pow_dual_interior(rng, a)
    if nfree:
        kinds.append(CONE_FREE); sizes.append(nfree); params.append(0.0)
        x0 += list(rng.uniform(-1, 1, nfree)); s0 += [0.0] * nfree
    if npos:
        kinds.append(CONE_POS); sizes.append(npos); params.append(0.0)
        x0 += list(rng.uniform(0.5, 2.0, npos)); s0 += list(rng.uniform(0.5, 2.0, npos))
    n = len(x0)
    A = sp.random(m, n, density=density, format="csc", random_state=rng, data_rvs=lambda s: rng.standard_normal(s))
    # every column carries at least one entry so that no variable is unconstrained
    A = sp.lil_matrix(A)
    empty = np.where(np.diff(sp.csc_matrix(A).indptr) == 0)[0]
    for j in empty:
        A[int(rng.integers(m)), j] = rng.standard_normal()
    # each free column also gets an entry in a row of its own (a random injection of the free
    # columns into the rows), so the free block has full structural column rank.  A free column has
    # a zero Hessian block, so only BᵀB can make δH + BᵀB definite on it; with the random pattern
    # alone, seed 0 at n = 20000 has free columns with a single entry in the same row (structural
    # rank 3995 of 4000), δH + BᵀB is singular and every factorization needs the ρ retry.
    if determined_free and nfree and nfree <= m:
        f0 = 3 * (nexp + npow)
        rows = rng.permutation(m)[:nfree]
        for j in range(nfree):
            A[int(rows[j]), f0 + j] = rng.standard_normal()
    A = sp.csc_matrix(A)
    x0 = np.array(x0); s0 = np.array(s0)
    y0 = rng.uniform(-1, 1, m)
    b = A @ x0
    c = A.T @ y0 + s0
    return dict(Q=sp.csc_matrix((n, n)), B=A, f=-c, g=b, mu=0.0, kinds=kinds, sizes=sizes, params=params,
                name=f"exppow nexp={nexp} npow={npow} n={n} m={m} density={density} seed={seed}")


def _svec(M):
    d = M.shape[0]
    r2 = np.sqrt(2.0)
    return np.concatenate([[M[j, j]] + [r2 * M[i, j] for i in range(j + 1, d)] for j in range(d)])


def _spd(rng, d):
    A = rng.standard_normal((d, d))
    return A @ A.T / d + np.eye(d)


def sdp(nblocks=3, d=4, m=10, density=0.3, npos=0, seed=0):
    """Random SDP with ``nblocks`` PSD blocks of order ``d`` (svec coordinates: column-major lower
    triangle, off-diagonals scaled by √2, as SemidefiniteCone stores them) and ``npos`` nonnegative
    columns; A sparse N(0,1) at the given density with every column covered.  Feasible by
    construction: x0, s0 positive definite (A Aᵀ/d + I), y0 ~ N(0,1), b = A x0, c = Aᵀ y0 + s0."""
    rng = np.random.default_rng(seed)
    k = d * (d + 1) // 2
    x0, s0, kinds, sizes = [], [], [], []
    for _ in range(nblocks):
        x0.append(_svec(_spd(rng, d))); s0.append(_svec(_spd(rng, d)))
        kinds.append(CONE_SDP); sizes.append(k)
    if npos:
        x0.append(rng.uniform(0.5, 2.0, npos)); s0.append(rng.uniform(0.5, 2.0, npos))
        kinds.append(CONE_POS); sizes.append(npos)
    x0 = np.concatenate(x0); s0 = np.concatenate(s0)
    n = len(x0)
    A = sp.lil_matrix(sp.random(m, n, density=density, format="csc", random_state=rng,
                                data_rvs=lambda s: rng.standard_normal(s)))
    for j in np.where(np.diff(sp.csc_matrix(A).indptr) == 0)[0]:
        A[int(rng.integers(m)), j] = rng.standard_normal()
    A = sp.csc_matrix(A)
    y0 = rng.standard_normal(m)
    b = A @ x0
    c = A.T @ y0 + s0
    return dict(Q=sp.csc_matrix((n, n)), B=A, f=-c, g=b, mu=0.0, kinds=kinds, sizes=sizes,
                params=[0.0] * len(kinds), name=f"sdp {nblocks}x PSD({d}) npos={npos} m={m} seed={seed}")


def sdp_eigmin(d=5, seed=0):
    """min ⟨C, X⟩ s.t. tr X = 1, X ⪰ 0: the optimum is λmin(C) (C symmetric N(0,1)); returns the
    problem and that value."""
    rng = np.random.default_rng(seed)
    Cm = rng.standard_normal((d, d)); Cm = (Cm + Cm.T) / 2
    k = d * (d + 1) // 2
    B = sp.csc_matrix(_svec(np.eye(d)).reshape(1, k))
    pb = dict(Q=sp.csc_matrix((k, k)), B=B, f=-_svec(Cm), g=np.array([1.0]), mu=0.0, kinds=[CONE_SDP], sizes=[k],
              params=[0.0], name=f"sdp eigmin d={d} seed={seed}")
    return pb, float(np.linalg.eigvalsh(Cm).min())


def maxcut(nodes=12, extra=6, band=2, seed=0):
    """Max-cut relaxation on a band graph (bandwidth ``band``) plus ``extra`` random edges, weights
    U(0,1): max ¼⟨L, X⟩ s.t. diag(X) = 1, X ⪰ 0, written as min ⟨−L/4, X⟩ with one PSD block."""
    rng = np.random.default_rng(seed)
    W = np.zeros((nodes, nodes))
    for i in range(nodes):
        for j in range(i + 1, min(nodes, i + band + 1)):
            W[i, j] = W[j, i] = rng.uniform()
    for _ in range(extra):
        i, j = rng.choice(nodes, 2, replace=False)
        W[i, j] = W[j, i] = rng.uniform()
    L = np.diag(W.sum(1)) - W
    k = nodes * (nodes + 1) // 2
    rows = []
    for i in range(nodes):
        E = np.zeros((nodes, nodes)); E[i, i] = 1.0
        rows.append(_svec(E))
    B = sp.csc_matrix(np.array(rows))
    return dict(Q=sp.csc_matrix((k, k)), B=B, f=_svec(L / 4), g=np.ones(nodes), mu=0.0, kinds=[CONE_SDP],
                sizes=[k], params=[0.0], name=f"maxcut nodes={nodes} band={band} extra={extra} seed={seed}")


def serving_mix(count, seed=0, nmin=100, nmax=2000):
    """Request stream of the serving workload: ``count`` problems, in equal shares SOCP (``socp``,
    SOC(20) blocks, m = 0.4 n, about 25 nonzeros per row), portfolio QP (``portfolio``) and max-cut
    SDP (``maxcut``, one PSD block), each with a target size n log-uniform in [nmin, nmax]; every
    request is a distinct seeded instance.  Returns (kind, problem) pairs."""
    rng = np.random.default_rng(seed)
    out = []
    for i in range(count):
        n = float(np.exp(rng.uniform(np.log(nmin), np.log(nmax))))
        kind = ("socp", "qp", "sdp")[i % 3]
        s = int(rng.integers(1 << 31))
        if kind == "socp":
            ncone = max(1, int(round(n / 20)))
            nn = 20 * ncone
            m = max(4, int(0.4 * nn))
            pb = socp(nn, m, ncone, density=min(0.5, 25.0 / nn), seed=s)
        elif kind == "qp":
            pb = portfolio(max(10, int(round((n - 21) / 2))), seed=s)
        else:
            nodes = max(4, int(round((np.sqrt(1 + 8 * n) - 1) / 2)))
            pb = maxcut(nodes, extra=nodes // 2, band=2, seed=s)
        out.append((kind, pb))
    return out


def socp_infeasible(which="primal", n=200, m=80, ncone=10, density=0.1, seed=0):
    """SOCP from ``socp`` with a planted infeasibility certificate.

    ``which="primal"``: row r of A is replaced so that Aᵀy_c = −s_c for y_c ~ N(0,1) and s_c in
    the cone interior, and b = A x0 + δ y_c with δ = (x0ᵀs_c + 1)/‖y_c‖², so bᵀy_c = 1 > 0.
    y_c is then a Farkas certificate: no x ∈ K has Ax = b.

    ``which="dual"``: column j of A is replaced so that A r = 0 for r in the cone interior, and
    c = Aᵀy0 + s0 − α r with α = (s0ᵀr + 1)/‖r‖², so cᵀr = −1 < 0. With the feasible b = A x0,
    x0 + t r stays feasible and cᵀx → −∞ as t grows: the problem is unbounded."""
    rng = np.random.default_rng(seed)
    k = n // ncone
    assert k * ncone == n
    A = sp.random(m, n, density=density, format="csc", random_state=rng,
                  data_rvs=lambda s: rng.standard_normal(s)).toarray()
    x0 = np.concatenate([_soc_interior(rng, k) for _ in range(ncone)])
    s0 = np.concatenate([_soc_interior(rng, k) for _ in range(ncone)])
    y0 = rng.standard_normal(m)
    if which == "primal":
        yc = rng.standard_normal(m)
        sc = np.concatenate([_soc_interior(rng, k) for _ in range(ncone)])
        r = int(np.argmax(np.abs(yc)))
        rest = np.delete(np.arange(m), r)
        A[r, :] = (-sc - A[rest, :].T @ yc[rest]) / yc[r]
        b = A @ x0 + (x0 @ sc + 1.0) / (yc @ yc) * yc
        c = A.T @ y0 + s0
    elif which == "dual":
        rr = np.concatenate([_soc_interior(rng, k) for _ in range(ncone)])
        j = int(np.argmax(rr))
        rest = np.delete(np.arange(n), j)
        A[:, j] = -(A[:, rest] @ rr[rest]) / rr[j]
        b = A @ x0
        c = A.T @ y0 + s0 - (s0 @ rr + 1.0) / (rr @ rr) * rr
    else:
        raise ValueError(which)
    return dict(Q=sp.csc_matrix((n, n)), B=sp.csc_matrix(A), f=-c, g=b, mu=0.0,
                kinds=[CONE_SOC] * ncone, sizes=[k] * ncone, params=[0.0] * ncone,
                name=f"socp-{which}-infeasible n={n} m={m} {ncone}xSOC({k}) seed={seed}")
