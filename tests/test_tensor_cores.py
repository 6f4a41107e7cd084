"""The FP32 factor's trailing-update tiles on the tensor cores (tcgen05.mma kind::tf32 with a
3xTF32 split, per-step FP32 read-out; settings.fp32_tiles = 2, the tensor-core build of the solver
kernels) against the FFMA tiles (fp32_tiles = 1) and the FP64 oracle.  Fronts of order 128 and more take the
tensor-core tiles; the portfolio instances here have one front of order 2 n_assets + 11."""
import numpy as np
import pytest

from helpers import block_problem, oracle_solve
from mumblebee_b200 import generators as G
from mumblebee_b200.ipm import Context, IPMProblem, IPMSettings, IPMStatus, batch_solve, solve

pytestmark = pytest.mark.gpu


def _rel(a, b):
    return abs(a - b) / max(1.0, abs(b))


@pytest.mark.parametrize("n_assets,seed", [(80, 7), (300, 11)])
def test_mixed_tensor_core_tiles_match_oracle(n_assets, seed):
    """Mixed precision reaches the FP64 oracle's optimum within the stopping tolerance with either
    tile engine; with the tensor cores some iterations are accepted on the FP32 factor, and the two
    engines' iterates differ (different arithmetic ran) while both meet the tolerance.  (On some
    instances the first FP32 iteration already misses the KKT tolerance with either engine, and the
    solve goes on in FP64; these two accept FP32 iterations.)"""
    ref = block_problem(G.portfolio(n_assets, seed=seed))
    prob = IPMProblem.from_dict(ref, ctx=Context.default())
    _, o = oracle_solve(ref, vperm=prob.symbolic()["vperm"])
    tc = solve(prob, IPMSettings(precision="mixed", fp32_tiles=2))
    ff = solve(prob, IPMSettings(precision="mixed", fp32_tiles=1))
    for r in (tc, ff):
        assert r.status == IPMStatus.OPTIMAL
        assert r.pres < 1e-8 and r.dres < 1e-8
        assert _rel(r.pobj, o["pobj"]) < 1e-7 and _rel(r.dobj, o["dobj"]) < 1e-7
    assert tc.nfp32 >= 1
    assert not np.array_equal(tc.p, ff.p)


def test_fp32_factor_accuracy_is_fp32_grade():
    """The 3xTF32 split keeps the FP32 factor's accuracy: an FP32 iteration on the tensor-core
    factor needs about as many KKT solves (refinement passes + CG steps) as on the FFMA factor.
    A plain TF32 factor (10-bit mantissa) would need several times more."""
    ref = block_problem(G.portfolio(300, seed=12))
    prob = IPMProblem.from_dict(ref, ctx=Context.default())
    tc = solve(prob, IPMSettings(precision="mixed", fp32_tiles=2))
    ff = solve(prob, IPMSettings(precision="mixed", fp32_tiles=1))
    assert tc.status == ff.status == IPMStatus.OPTIMAL
    assert tc.nsolve <= 1.5 * ff.nsolve + 4, (tc.nsolve, ff.nsolve)


def test_mixed_tensor_core_batch_equals_alone():
    """The tensor-core tiles are deterministic: each mixed-precision instance gives its lone result
    bit for bit inside a batch of several sizes."""
    probs = [IPMProblem.from_dict(block_problem(G.portfolio(n, seed=20 + i)), ctx=Context.default())
             for i, n in enumerate([70, 130, 260, 45])]
    st = IPMSettings(precision="mixed", fp32_tiles=2)
    mix = batch_solve(probs, st, grid=3)
    for p, rm in zip(probs, mix):
        ra = batch_solve([p], st)[0]
        assert ra.status == rm.status and ra.niter == rm.niter and ra.nfp32 == rm.nfp32
        np.testing.assert_array_equal(ra.p, rm.p)
        np.testing.assert_array_equal(ra.y, rm.y)
