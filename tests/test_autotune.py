"""The launch-configuration autotuner (mumblebee_b200.autotune): the stratified sample on the host,
and the choice by timed trial launches on the device."""
import numpy as np
import pytest

from helpers import product_problem
from mumblebee_b200 import generators as G
from mumblebee_b200.autotune import CANDIDATES, _sample, largest_front


def _portfolios(sizes, ctx=None):
    return [product_problem(G.portfolio(int(n), seed=100 + i), ctx=ctx) for i, n in enumerate(sizes)]


def test_sample_is_stratified_by_largest_front():
    """The sample spans the workload's fronts from the smallest to the largest, has no repeats, and
    is the whole list when the list is short."""
    sizes = np.random.default_rng(0).integers(20, 120, size=60)
    probs = _portfolios(sizes)
    fronts = sorted(largest_front(p) for p in probs)
    sub = _sample(probs, 12, seed=0)
    assert 10 <= len(sub) <= 12 and len({id(p) for p in sub}) == len(sub)
    f = sorted(largest_front(p) for p in sub)
    assert f[0] <= fronts[2] and f[-1] >= fronts[-3]
    assert _sample(probs[:5], 12, seed=0) == probs[:5]


@pytest.mark.gpu
@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_tune_times_every_candidate(precision):
    """Every candidate that applies is timed (the tensor-core build only where an FP32 factor runs),
    the choice is the fastest, and its settings solve the workload like the default ones."""
    from mumblebee_b200.autotune import tune
    from mumblebee_b200.ipm import Context, IPMSettings, IPMStatus, batch_solve
    probs = _portfolios(np.random.default_rng(1).integers(40, 200, size=48), ctx=Context.default())
    c = tune(probs, IPMSettings(precision=precision), nsm=4, repeats=1)
    names = {n for n, tiles, _ in CANDIDATES if precision != "fp64" or tiles != 2}
    assert set(c.trials) == names
    assert c.trials[c.name] == min(c.trials.values())
    assert c.settings.precision == precision and c.grid >= 1
    res = batch_solve(probs, c.settings, grid=c.grid)
    assert all(r.status == IPMStatus.OPTIMAL for r in res)
