"""Compensated block-sparse products, extmul! / twomul! of BlockSparseArrays (src/comp/comp.jl,
src/comp/twogemv.jl).

The oracle restates the reference's block loops literally.  The reference has no tests for these
routines, so the oracle is pinned against exact rational arithmetic.  The property checked is the
published guarantee of compensated dot products (Ogita, Rump and Oishi, "Accurate sum and dot
product", SISC 26(6), 2005, Prop. 5.5): |res − xᵀy| ≤ u|xᵀy| + γ_n² |x|ᵀ|y|, with u = 2⁻⁵³ and
γ_n = nu/(1 − nu).  It is checked on dot products whose condition numbers reach 1e20, made by
their generator (GenDot, Algorithm 6.1), through both the A b and the Aᵀ b loops.  On those
inputs a plain FP64 sum has no correct digit.

The device is held to the oracle bitwise, for every α/β branch of the epilogue, both orientations,
1 x 1 and zero blocks, explicit zeros and NaN propagation.  Every output entry takes its terms in
the reference's order, so there is no rounding difference to allow for."""
from fractions import Fraction

import numpy as np
import pytest

import oracle
from mumblebee_b200.comp import blocksparse

U = 2.0 ** -53


def _gendot(n, cond, rng):
    """x, y with condition ≈ cond of xᵀy (GenDot, Ogita-Rump-Oishi 2005, Algorithm 6.1; the
    running dot of the second half computed exactly)."""
    n2 = n // 2
    b = np.log2(cond)
    e = np.rint(rng.random(n2) * b / 2).astype(int)
    e[0] = int(np.rint(b / 2)) + 1
    e[-1] = 0
    x = np.zeros(n)
    y = np.zeros(n)
    x[:n2] = (2 * rng.random(n2) - 1) * np.exp2(e)
    y[:n2] = (2 * rng.random(n2) - 1) * np.exp2(e)
    acc = sum(Fraction(float(p)) * Fraction(float(q)) for p, q in zip(x[:n2], y[:n2]))
    for i, ei in zip(range(n2, n), np.rint(np.linspace(b / 2, 0, n - n2)).astype(int)):
        x[i] = (2 * rng.random() - 1) * 2.0 ** ei
        y[i] = float(((2 * rng.random() - 1) * 2.0 ** ei - acc) / Fraction(x[i]))
        acc += Fraction(x[i]) * Fraction(y[i])
    p = rng.permutation(n)
    return x[p], y[p]


def _exact(x, y):
    return sum(Fraction(float(p)) * Fraction(float(q)) for p, q in zip(x, y))


def _bound(x, y, exact):
    n = len(x)
    g = n * U / (1 - n * U)
    return U * abs(float(exact)) + g * g * float(np.abs(x) @ np.abs(y))


def _sizes(n, rng, maxb=4):
    s = []
    while sum(s) < n:
        s.append(int(min(rng.integers(1, maxb + 1), n - sum(s))))
    return s


@pytest.mark.parametrize("cond", [1e4, 1e8, 1e12, 1e16, 1e20])
@pytest.mark.parametrize("trans", [False, True])
def test_oracle_dot_within_compensated_bound(cond, trans):
    rng = np.random.default_rng(int(np.log10(cond)) + 7 * trans)
    n = 64
    x, y = _gendot(n, cond, rng)
    ex = _exact(x, y)
    cs_ = _sizes(n, rng)
    # one row of blocks (A b) or one column of blocks (Aᵀ b): the dot through each loop
    A = blocksparse(x[None, :], cs_, [1]) if not trans else blocksparse(x[:, None], [1], cs_)
    c, _, s, cs = oracle.twomul(A, trans, y, 1.0, 0.0, np.zeros(1), False)
    assert abs(Fraction(float(c[0])) - ex) <= Fraction(_bound(x, y, ex))
    # the pair of twomul!: same hi part bitwise, and hi + lo carries the doubled-precision value
    c2, cc2, _, _ = oracle.twomul(A, trans, y, 1.0, 0.0, np.zeros(1), True)
    assert c2[0] == c[0]
    assert abs(Fraction(float(c2[0])) + Fraction(float(cc2[0])) - ex) <= Fraction(2 * _bound(x, y, ex) - U * abs(float(ex)))
    if cond >= 1e16:   # a plain sum loses every digit here
        naive = float(np.dot(x, y))
        assert abs(Fraction(naive) - ex) > 100 * Fraction(_bound(x, y, ex))


def test_oracle_single_term_is_exact():
    """One 1 x 1 block: (s, cs) is twomul's error-free pair, s + cs = a b exactly."""
    rng = np.random.default_rng(3)
    for _ in range(50):
        a, b = rng.standard_normal(2) * np.exp2(rng.integers(-30, 30, 2))
        A = blocksparse([[a]], [1], [1])
        _, _, s, cs = oracle.twomul(A, False, [b], 1.0, 0.0, np.zeros(1), False)
        assert Fraction(float(s[0])) + Fraction(float(cs[0])) == Fraction(float(a)) * Fraction(float(b))


@pytest.mark.parametrize("alpha,beta", [(1.0, 0.0), (2.5, 0.0), (1.0, 1.0), (-1.0, 1.0), (0.3, 1.0),
                                        (1.0, -1.0), (-1.0, -1.0), (0.3, -1.0), (0.7, 1.9)])
def test_oracle_epilogue_within_bound(alpha, beta):
    """c ← α(s + cs) + β c for each branch of extaxpby!: within a few u of the exact value,
    relative to |α xᵀy| + |β c| (the result is rounded once from doubled precision)."""
    rng = np.random.default_rng(11)
    x, y = _gendot(40, 1e12, rng)
    c0 = float(rng.standard_normal())
    A = blocksparse(x[None, :], _sizes(40, rng), [1])
    ex = Fraction(alpha) * _exact(x, y) + Fraction(beta) * Fraction(c0)
    c, _, _, _ = oracle.twomul(A, False, y, alpha, beta, np.array([c0]), False)
    scale = abs(alpha) * _bound(x, y, _exact(x, y)) / U + abs(beta * c0) + abs(float(ex))
    assert abs(Fraction(float(c[0])) - ex) <= Fraction(4 * U * scale)


def _random_block_matrix(rng, nrow, ncol, density=0.5):
    rs, cs_ = _sizes(nrow, rng, 5), _sizes(ncol, rng, 5)
    M = rng.standard_normal((nrow, ncol))
    xr = np.concatenate([[0], np.cumsum(rs)])
    xc = np.concatenate([[0], np.cumsum(cs_)])
    for u in range(len(rs)):
        for v in range(len(cs_)):
            if rng.random() > density:
                M[xr[u]:xr[u + 1], xc[v]:xc[v + 1]] = 0.0
    M[rng.random(M.shape) < 0.1] = 0.0   # explicit zeros inside stored blocks
    if len(rs) > 1 and len(cs_) > 1:      # one stored block that is entirely zero
        M[xr[0]:xr[1], xc[0]:xc[1]] = 0.0
    A = blocksparse(M, cs_, rs)
    Az = blocksparse(M, cs_, rs, keep_zero_blocks=True)
    return M, A, Az


def test_blocksparse_layout():
    rng = np.random.default_rng(5)
    M, A, Az = _random_block_matrix(rng, 13, 17)
    for d in (A, Az):
        D = np.zeros(M.shape)
        for v in range(d["nvtx"]):
            c0, c1 = d["xcol"][v] - 1, d["xcol"][v + 1] - 1
            for e in range(d["xsrc"][v] - 1, d["xsrc"][v + 1] - 1):
                u = d["tgt"][e] - 1
                r0, r1 = d["xrow"][u] - 1, d["xrow"][u + 1] - 1
                D[r0:r1, c0:c1] = d["val"][d["xblk"][e] - 1:d["xblk"][e + 1] - 1].reshape((r1 - r0, c1 - c0), order="F")
            assert np.all(np.diff(d["tgt"][d["xsrc"][v] - 1:d["xsrc"][v + 1] - 1]) > 0)
        np.testing.assert_array_equal(D, M)
    assert Az["nbnz"] == M.size and A["nbnz"] < M.size


# ---- device (C ABI) against the oracle, bitwise -------------------------------------------------

BRANCHES = [(1.0, 0.0), (-2.0, 0.0), (1.0, 1.0), (-1.0, 1.0), (0.3, 1.0), (1.0, -1.0), (-1.0, -1.0),
            (0.3, -1.0), (0.7, 1.9), (1.0, 0.5)]


@pytest.mark.gpu
@pytest.mark.parametrize("keep", [False, True])
@pytest.mark.parametrize("trans", [False, True])
def test_device_equals_oracle_bitwise(trans, keep):
    from mumblebee_b200.comp import BlockSparseMatrix, extmul, twomul
    rng = np.random.default_rng(17 + trans + 2 * keep)
    M, A, Az = _random_block_matrix(rng, 300, 211)
    d = Az if keep else A
    D = BlockSparseMatrix(d)
    op = D.T if trans else D
    nout, nin = (M.shape[1], M.shape[0]) if trans else M.shape
    b = rng.standard_normal(nin) * np.exp2(rng.integers(-20, 20, nin))
    c0 = rng.standard_normal(nout)
    for alpha, beta in BRANCHES:
        oc, _, os_, ocs = oracle.twomul(d, trans, b, alpha, beta, c0, False)
        c = c0.copy(); s = np.zeros(nout); cs = np.zeros(nout)
        extmul(c, op, b, alpha, beta, s, cs)
        np.testing.assert_array_equal(c, oc)
        np.testing.assert_array_equal(s, os_)
        np.testing.assert_array_equal(cs, ocs)
        pc, pcc, _, _ = oracle.twomul(d, trans, b, alpha, beta, c0, True)
        c2 = c0.copy(); cc2 = np.zeros(nout)
        twomul(c2, cc2, op, b, alpha, beta)
        np.testing.assert_array_equal(c2, pc)
        np.testing.assert_array_equal(cc2, pcc)
        np.testing.assert_array_equal(c2, c)   # the pair's hi part is extmul's result


@pytest.mark.gpu
@pytest.mark.parametrize("trans", [False, True])
def test_device_ill_conditioned_dot(trans):
    from mumblebee_b200.comp import BlockSparseMatrix, extmul
    rng = np.random.default_rng(23)
    n = 200
    x, y = _gendot(n, 1e18, rng)
    sz = _sizes(n, rng)
    d = blocksparse(x[None, :], sz, [1]) if not trans else blocksparse(x[:, None], [1], sz)
    D = BlockSparseMatrix(d)
    c = np.zeros(1)
    extmul(c, D.T if trans else D, y, 1.0, 0.0)
    oc = oracle.twomul(d, trans, y, 1.0, 0.0, np.zeros(1), False)[0]
    assert c[0] == oc[0]
    ex = _exact(x, y)
    assert abs(Fraction(float(c[0])) - ex) <= Fraction(_bound(x, y, ex))


@pytest.mark.gpu
def test_device_nan_and_edge_shapes():
    """An infinite entry of b makes every output it reaches NaN, as in the reference: an explicit
    zero times it is NaN, and a finite nonzero times it gives twomul's error term fma(a, b, -ab)
    = inf - inf = NaN.  An empty matrix leaves α·0 + β c; a matrix with no stored block gives β c."""
    from mumblebee_b200.comp import BlockSparseMatrix, extmul
    M = np.array([[0.0, 2.0], [1.0, 3.0]])
    d = blocksparse(M, [2], [2], keep_zero_blocks=True)
    b = np.array([np.inf, 1.0])
    c = np.zeros(2)
    extmul(c, BlockSparseMatrix(d), b, 1.0, 0.0)
    oc = oracle.twomul(d, False, b, 1.0, 0.0, np.zeros(2), False)[0]
    np.testing.assert_array_equal(c, oc)
    assert np.isnan(c).all()
    Z = blocksparse(np.zeros((3, 4)), [2, 2], [1, 2])
    assert Z["narc"] == 0
    c = np.array([1.0, -2.0, 3.0])
    extmul(c, BlockSparseMatrix(Z), np.ones(4), 2.0, 0.5)
    np.testing.assert_array_equal(c, [0.5, -1.0, 1.5])
    E = blocksparse(np.zeros((0, 3)), [3], [])
    c = np.zeros(3)
    extmul(c, BlockSparseMatrix(E).T, np.zeros(0), 1.0, 0.0)
    np.testing.assert_array_equal(c, np.zeros(3))
