"""mb_batch_solve_static (the batched solve from the library's fixed device scratch, no device
allocation) against mb_batch_solve on the same problems: two static calls in a row, each within
the parity tolerance of the allocating path, and the device's free memory unchanged by them.
Collected last so it also runs after every other GPU test in the same process."""
import numpy as np
import pytest

from helpers import SMALL, TDC, TDC_TOL, product_problem
from mumblebee_b200 import _lib
from mumblebee_b200 import generators as G
from mumblebee_b200.ipm import Context, IPMSettings, batch_solve, batch_solve_static

pytestmark = pytest.mark.gpu


def _close(a, b):
    assert a.status == b.status and a.niter == b.niter
    assert a.nfactor == b.nfactor and a.nfactor_retry == b.nfactor_retry
    for x, y in ((a.pobj, b.pobj), (a.dobj, b.dobj)):
        assert abs(x - y) <= 1e-9 * max(1.0, abs(y))
    for x, y in ((a.p, b.p), (a.d, b.d), (a.y, b.y)):
        np.testing.assert_allclose(x, y, rtol=1e-9, atol=1e-9)


@pytest.mark.parametrize("which,settings", [
    ("soc_pos", IPMSettings()),
    ("exp_pow", IPMSettings(**TDC_TOL)),
    ("mixed", IPMSettings(precision="mixed")),
])
def test_static_matches_allocating_path(which, settings):
    import torch
    ctx = Context.default(0)
    if which == "exp_pow":
        pbs = [f() for f in TDC.values()]
    else:
        pbs = [f() for f in SMALL.values()]
    probs = [product_problem(pb, ctx=ctx) for pb in pbs]
    ref = batch_solve(probs, settings)
    torch.cuda.synchronize(0)
    free0, _ = torch.cuda.mem_get_info(0)
    first = batch_solve_static(probs, settings)
    second = batch_solve_static(probs, settings)
    free1, _ = torch.cuda.mem_get_info(0)
    assert free1 == free0
    for r, a, b in zip(ref, first, second):
        _close(a, r)
        _close(b, r)


def test_static_rejects_oversize_batch():
    ctx = Context.default(0)
    probs = [product_problem(G.portfolio(400, seed=s), ctx=ctx) for s in range(3)]
    need = sum(p.footprint() for p in probs)
    assert need > _lib.MB_STATIC_SCRATCH_BYTES
    with pytest.raises(_lib.MBError, match="MB_STATIC_SCRATCH_BYTES"):
        batch_solve_static(probs)
    # one of them fits, and the scratch is still usable after the rejection
    r = batch_solve_static(probs[:1])[0]
    ref = batch_solve(probs[:1])[0]
    _close(r, ref)
