"""Grid-cooperative mode for one large instance (settings `large`): the leader CTA runs the solve and
the helper CTAs take update tiles, panel rows, extend-adds and the assembly copy of its large
fronts.  Each of those elements is still computed by exactly one CTA in the same order, so the
result must equal the one-CTA path bit for bit.  That holds for the right-looking factor of fronts
of order 1024 and more too: an entry's accumulator starts from the front's value and takes the
products in increasing k with the same chunk boundaries, and storing it between the 64-column
steps is exact."""
import numpy as np
import pytest

from helpers import SDP, block_problem
from mumblebee_b200 import generators as G
from mumblebee_b200.ipm import Context, IPMProblem, IPMSettings, IPMStatus, solve

pytestmark = pytest.mark.gpu

CASES = {
    "socp500": lambda: G.socp(500, 200, 25, 0.05, 0),                       # one front of 500
    "port300": lambda: G.portfolio(300, seed=4),                            # one front of 621
    "maxcut30": lambda: G.maxcut(30, 15, 2, 1),                             # SDP, one front of 465
    "exppow_multi": lambda: G.exppow(nexp=150, npow=60, nfree=200, npos=200, m=400, density=0.01, seed=2),
    "socp2100": lambda: G.socp(2100, 840, 105, 0.012, 5),                   # front >= 2048: shared solves too
}


@pytest.mark.parametrize("name", list(CASES))
def test_large_mode_equals_one_cta(name):
    prob = IPMProblem.from_dict(block_problem(CASES[name]()), ctx=Context.default())
    tol = dict(feas_tol=1e-7, gap_tol=1e-7) if name.startswith("exppow") else {}
    a = solve(prob, IPMSettings(large=-1, **tol))
    b = solve(prob, IPMSettings(large=1, **tol))
    assert a.status == b.status and a.status in (IPMStatus.OPTIMAL, IPMStatus.NEAR_OPTIMAL)
    assert a.niter == b.niter and a.nfactor == b.nfactor
    assert a.pobj == b.pobj and a.dobj == b.dobj
    for x, y in ((a.p, b.p), (a.d, b.d), (a.y, b.y)):
        assert np.array_equal(x, y)


@pytest.mark.parametrize("tiles", [1, 2])
def test_right_looking_mixed_precision_matches_one_cta(tiles):
    """A portfolio front of order 1211 in the grid-cooperative mode, mixed precision: the
    right-looking FP32 and FP64 factors (FFMA or tensor-core tiles) give the one-CTA result bit
    for bit."""
    prob = IPMProblem.from_dict(block_problem(G.portfolio(600, seed=8)), ctx=Context.default())
    a = solve(prob, IPMSettings(large=-1, precision="mixed", fp32_tiles=tiles))
    b = solve(prob, IPMSettings(large=1, precision="mixed", fp32_tiles=tiles))
    assert a.status == b.status == IPMStatus.OPTIMAL
    assert a.niter == b.niter and a.nfp32 == b.nfp32
    assert a.pobj == b.pobj and np.array_equal(a.p, b.p)


@pytest.mark.parametrize("tiles", [1, 2])
def test_large_mode_mixed_precision_equals_one_cta(tiles):
    """The FP32 tiles, panel rows and solves of the mixed path, shared with the helpers: FFMA tiles
    (fp32_tiles = 1) and the tensor-core build (2), each against one CTA of the same build."""
    prob = IPMProblem.from_dict(block_problem(CASES["port300"]()), ctx=Context.default())
    a = solve(prob, IPMSettings(large=-1, precision="mixed", fp32_tiles=tiles))
    b = solve(prob, IPMSettings(large=1, precision="mixed", fp32_tiles=tiles))
    assert a.status == b.status and a.niter == b.niter and a.nfp32 == b.nfp32
    assert a.pobj == b.pobj and np.array_equal(a.p, b.p)


def test_grid_barrier_wait_runs_out():
    """settings.coop_wait bounds every wait at a grid barrier.  With a limit far shorter than the
    leader's serial work before its first command, a helper's wait runs out: every CTA returns, the
    call fails with MB_E_TIMEOUT, and the same context then solves normally."""
    from mumblebee_b200._lib import MBError
    prob = IPMProblem.from_dict(block_problem(CASES["port300"]()), ctx=Context.default())
    with pytest.raises(MBError, match="code -6.*coop_wait"):
        solve(prob, IPMSettings(large=1, coop_wait=1e-6))
    a = solve(prob, IPMSettings(large=-1))
    b = solve(prob, IPMSettings(large=1))
    assert a.status == b.status == IPMStatus.OPTIMAL
    assert a.niter == b.niter and a.pobj == b.pobj and np.array_equal(a.p, b.p)


def test_large_mode_sdp_and_step_api():
    from mumblebee_b200.ipm import init
    prob = IPMProblem.from_dict(block_problem(SDP["sdp1x10"]()), ctx=Context.default())
    a = solve(prob, IPMSettings(large=-1))
    s = init(prob, IPMSettings(large=1))
    while s.step() == IPMStatus.CONTINUE:
        pass
    b = s.result()
    assert a.niter == b.niter and a.pobj == b.pobj
