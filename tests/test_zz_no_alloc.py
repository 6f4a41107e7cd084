"""mb_batch_solve_static (the batched solve from the library's fixed device scratch, no device
allocation) against mb_batch_solve on the same problems.  Both run the same planning, the same
instance order and the same kernel over the same data; only the base addresses differ, so the
results must be bitwise equal, on two static calls in a row, with the device's free memory
unchanged by them.  Collected last so it also runs after every other GPU test in the same
process."""
import numpy as np
import pytest

from helpers import SMALL, TDC, TDC_TOL, product_problem
from mumblebee_b200 import _lib
from mumblebee_b200 import generators as G
from mumblebee_b200.ipm import Context, IPMSettings, batch_solve, batch_solve_static

pytestmark = pytest.mark.gpu


def _same(a, b):
    assert a.status == b.status and a.niter == b.niter and a.nsolve == b.nsolve
    assert a.nfactor == b.nfactor and a.nfactor_retry == b.nfactor_retry
    assert a.nfp32 == b.nfp32 and a.nfallback == b.nfallback
    for x, y in ((a.pobj, b.pobj), (a.dobj, b.dobj), (a.pres, b.pres), (a.dres, b.dres), (a.mu, b.mu)):
        assert x == y or (np.isnan(x) and np.isnan(y))
    for x, y in ((a.p, b.p), (a.d, b.d), (a.y, b.y)):
        np.testing.assert_array_equal(x, y)


def _free():
    import torch
    torch.cuda.synchronize(0)
    return torch.cuda.mem_get_info(0)[0]


@pytest.mark.parametrize("which,settings", [
    ("soc_pos", IPMSettings()),
    ("exp_pow", IPMSettings(**TDC_TOL)),
    ("mixed", IPMSettings(precision="mixed")),
])
def test_static_matches_allocating_path(which, settings):
    ctx = Context.default(0)
    pbs = [f() for f in (TDC if which == "exp_pow" else SMALL).values()]
    probs = [product_problem(pb, ctx=ctx) for pb in pbs]
    ref = batch_solve(probs, settings)
    free0 = _free()
    first = batch_solve_static(probs, settings)
    second = batch_solve_static(probs, settings)
    assert _free() == free0
    for r, a, b in zip(ref, first, second):
        _same(a, r)
        _same(b, r)


def test_static_grid_cooperative_single_instance():
    """settings.large = 1 sends a lone instance to the grid-cooperative launch in both paths."""
    ctx = Context.default(0)
    probs = [product_problem(G.portfolio(120, seed=11), ctx=ctx)]
    s = IPMSettings(large=1)
    ref = batch_solve(probs, s)[0]
    free0 = _free()
    a = batch_solve_static(probs, s)[0]
    b = batch_solve_static(probs, s)[0]
    assert _free() == free0
    _same(a, ref)
    _same(b, ref)


def test_static_rejects_oversize_batch():
    ctx = Context.default(0)
    probs = [product_problem(G.portfolio(400, seed=s), ctx=ctx) for s in range(3)]
    need = sum(p.footprint() for p in probs)
    assert need > _lib.MB_STATIC_SCRATCH_BYTES
    free0 = _free()
    with pytest.raises(_lib.MBError, match="MB_STATIC_SCRATCH_BYTES"):
        batch_solve_static(probs)
    assert _free() == free0
    assert batch_solve_static([]) == []
    # one of them fits, and the scratch is still usable after the rejection
    r = batch_solve_static(probs[:1])[0]
    ref = batch_solve(probs[:1])[0]
    _same(r, ref)
