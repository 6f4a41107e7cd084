"""CPU: the oracle's exponential / power cone restatement against the mathematics it encodes
(the reference ships no fixtures for these cones): barrier derivatives by finite differences, the
shadow round trip -f'(p*) = d, the double-double logarithm against decimal arithmetic, the secant
conditions of the Tunçel scaling M p = d and M p* = d*, and the certified step against a brute-force
boundary search."""
import ctypes as C
from decimal import Decimal, getcontext

import numpy as np
import pytest

import oracle
from mumblebee_b200 import generators as G

P = C.POINTER(C.c_double)


@pytest.fixture(scope="module")
def L():
    lib = oracle.lib()
    lib.oracle_tdc_eval.argtypes = [C.c_int, C.c_double, P, P, P]
    lib.oracle_tdc_scale_step.argtypes = [C.c_int, C.c_double, P, P, P, P, P]
    return lib


def _eval(L, kind, a, x, u=(0.3, -0.2, 0.5)):
    x = np.array(x, float); u = np.array(u, float); out = np.zeros(33)
    ok = L.oracle_tdc_eval(kind, a, x.ctypes.data_as(P), u.ctypes.data_as(P), out.ctypes.data_as(P))
    return ok, out


def _f(kind, a):
    if kind == 4:   # exp.jl:29-39: f = -log(x2 log(x1/x2) - x3) - log x1 - log x2
        return lambda x: -np.log(x[1] * np.log(x[0] / x[1]) - x[2]) - np.log(x[0]) - np.log(x[1])
    # pow.jl:41-49: f = -log(x1^2a x2^(2-2a) - x3^2) - (1-a) log x1 - a log x2
    return lambda x: -np.log(x[0] ** (2 * a) * x[1] ** (2 - 2 * a) - x[2] ** 2) - (1 - a) * np.log(x[0]) - a * np.log(x[1])


def _grad(f, x, h=1e-6):
    g = np.zeros(3)
    for i in range(3):
        e = np.zeros(3); e[i] = h
        g[i] = (f(x + e) - f(x - e)) / (2 * h)
    return g


POINTS = [(4, 0.0, [1.5, 0.7, -0.3]), (4, 0.0, [0.6, 1.8, -2.5]), (5, 0.3, [1.1, 0.9, 0.4]),
          (5, 0.7, [0.8, 1.6, -0.5]), (5, 0.5, [2.0, 0.5, 0.9])]


@pytest.mark.parametrize("kind,a,x", POINTS)
def test_barrier_derivatives(L, kind, a, x):
    ok, o = _eval(L, kind, a, x)
    assert ok == 1
    x = np.array(x); f = _f(kind, a); u = np.array([0.3, -0.2, 0.5])
    g = o[:3]; H = o[3:12].reshape(3, 3, order="F"); D = o[12:21].reshape(3, 3, order="F")
    np.testing.assert_allclose(g, _grad(f, x), rtol=1e-7, atol=1e-8)
    Hn = np.array([_grad(lambda z: _grad(f, z, 1e-5)[i], x, 1e-5) for i in range(3)])
    np.testing.assert_allclose(H, Hn, rtol=1e-4, atol=1e-5)
    hess = lambda z: np.array([_grad(lambda w: _grad(f, w, 1e-4)[i], z, 1e-4) for i in range(3)])
    Dn = (hess(x + 1e-5 * u) - hess(x - 1e-5 * u)) / 2e-5
    np.testing.assert_allclose(D, Dn, rtol=2e-3, atol=2e-3 * np.abs(D).max())


@pytest.mark.parametrize("kind,a,x", POINTS)
def test_shadow_roundtrip(L, kind, a, x):
    """d* = -f'(p) and the primal shadow of d* recovers p (tdc.jl:486-501)."""
    ok, o = _eval(L, kind, a, x)
    np.testing.assert_allclose(o[21:24], -o[:3], rtol=1e-15)
    np.testing.assert_allclose(o[24:27], x, rtol=1e-12, atol=1e-13)


def test_identity_points(L):
    """-f'(e) ≈ e at the identity points (exp.jl:15-20, pow.jl:27-33)."""
    ok, o = _eval(L, 4, 0.0, [1.2909282315382298, 0.8051015526498357, -0.8278379086082098])
    np.testing.assert_allclose(-o[:3], [1.2909282315382298, 0.8051015526498357, -0.8278379086082098], rtol=1e-5)
    for a in (0.2, 0.5, 0.8):
        e = [np.sqrt(1 + a), np.sqrt(2 - a), 0.0]
        ok, o = _eval(L, 5, a, e)
        np.testing.assert_allclose(-o[:3], e, rtol=1e-14, atol=1e-15)


def test_double_double_log(L):
    getcontext().prec = 60
    for x1, x2 in [(1.5, 0.7), (1.0 + 2 ** -40, 1.0), (3e-200, 7e-190), (1e150, 2.5e-150), (0.9999999999, 1.0)]:
        ok, o = _eval(L, 4, 0.0, [x1, x2, -1e300])
        ref = (Decimal(x1) / Decimal(x2)).ln()
        got = Decimal(o[31]) + Decimal(o[32])
        assert abs(got - ref) <= Decimal("1e-30") * max(Decimal(1), abs(ref)), (x1, x2, got - ref)


def _member(kind, a, x, dual):
    if kind == 4:
        if dual:
            return x[0] > 0 and x[2] < 0 and 1 + np.log(x[0]) - x[1] / x[2] - np.log(-x[2]) > 0
        return x[0] > 0 and x[1] > 0 and x[1] * np.log(x[0] / x[1]) - x[2] > 0
    if dual:
        return x[0] > 0 and x[1] > 0 and (x[0] / a) ** a * (x[1] / (1 - a)) ** (1 - a) - abs(x[2]) > 0
    return x[0] > 0 and x[1] > 0 and x[0] ** a * x[1] ** (1 - a) - abs(x[2]) > 0


def _brute(kind, a, x, dx, dual):
    if _member(kind, a, x + dx, dual):
        return 1.0
    lo, hi = 0.0, 1.0
    for _ in range(80):
        m = (lo + hi) / 2
        lo, hi = (m, hi) if _member(kind, a, x + m * dx, dual) else (lo, m)
    return lo


@pytest.mark.parametrize("trial", range(10))
def test_tuncel_scaling_and_certified_steps(L, trial):
    rng = np.random.default_rng(100 + trial)
    kind = 4 if trial % 2 == 0 else 5
    a = float(rng.uniform(0.2, 0.8)) if kind == 5 else 0.0
    p = np.array(G._exp_interior(rng) if kind == 4 else G._pow_interior(rng, a))
    d = np.array(G._exp_dual_interior(rng) if kind == 4 else G._pow_dual_interior(rng, a))
    Dp = rng.standard_normal(3) * 2; Dd = rng.standard_normal(3) * 2
    out = np.zeros(17)
    ok = L.oracle_tdc_scale_step(kind, a, *[v.ctypes.data_as(P) for v in (p, d, Dp, Dd, out)])
    assert ok == 1
    M = out[:9].reshape(3, 3, order="F"); sp = out[9:12]; sd = out[12:15]
    np.testing.assert_allclose(M @ p, d, rtol=1e-12, atol=1e-12)
    np.testing.assert_allclose(M @ sp, sd, rtol=1e-10, atol=1e-10)
    assert np.linalg.eigvalsh((M + M.T) / 2).min() > 0
    tp, td = out[15], out[16]
    assert abs(tp - _brute(kind, a, p, Dp, False)) <= 1e-9
    assert abs(td - _brute(kind, a, d, Dd, True)) <= 1e-9


def test_oracle_reinit_reproduces_the_first_solve_before_a_step():
    """reinit! on a solver that has not stepped (H is still Q) starts over exactly as init did."""
    from helpers import SMALL, block_problem, oracle_solve
    import oracle
    ref = block_problem(SMALL["port_small"]())
    _, r1 = oracle_solve(ref)
    s = oracle.OracleSolver(ref, oracle.default_settings())
    s.reinit()
    r2 = s.solve()
    assert r2["status"] == r1["status"] and r2["niter"] == r1["niter"]
    assert np.array_equal(r2["p"], r1["p"])
