"""reinit! (src/IPM/src/ipm/solver/ipm.jl:371-429) and the solver's timers.

reinit! keeps init's equilibration, Q, B, BᵀB and the Hessian blocks H of the last step.  The
first step after it sizes δ from norm(H) (getaug, solver/solver.jl:40-52) before scale! refreshes
H, so after a finished solve that δ comes from the last iteration's scaling; when BᵀB is singular
the first factorization then fails, in the reference as in the oracle and on the device.  The
device is held to the oracle's reinit! on the same problem: same status and iteration count, and
objectives to 1e-9.  Before any step H is still Q, so a reinit there equals a fresh solver on the
new data, bitwise."""
import numpy as np
import pytest

from helpers import SMALL, block_problem, oracle_solve, product_problem
from mumblebee_b200 import generators as G
from mumblebee_b200.ipm import Context, IPMProblem, IPMSettings, IPMStatus, init, print_timers

pytestmark = pytest.mark.gpu


def _rel(a, b):
    return abs(a - b) / max(1.0, abs(b))


def _like_oracle(r, o):
    assert r.status.name == o["status"] and r.niter == o["niter"]
    if o["status"] == "OPTIMAL":
        assert _rel(r.pobj, o["pobj"]) < 1e-9 and _rel(r.dobj, o["dobj"]) < 1e-9


def _pair(pb):
    ref = block_problem(pb)
    prob = IPMProblem.from_dict(ref, ctx=Context.default())
    o, ro = oracle_solve(ref, vperm=prob.symbolic()["vperm"])
    s = init(prob, IPMSettings())
    r = s.solve()
    _like_oracle(r, ro)
    return ref, prob, s, o


@pytest.mark.parametrize("name", ["socp_small", "port_small"])
def test_reinit_after_solve_like_oracle(name):
    pb = SMALL[name]()
    _, _, s, o = _pair(pb)
    _like_oracle(s.reinit().solve(), o.reinit().solve())


@pytest.mark.parametrize("which", ["f", "g", "fg"])
def test_reinit_new_data_like_oracle(which):
    pb = SMALL["port_small"]()
    rng = np.random.default_rng(3)
    f = pb["f"] + 0.01 * rng.standard_normal(pb["f"].shape) if "f" in which else None
    g = pb["g"] * 1.01 if "g" in which else None
    _, _, s, o = _pair(pb)
    _like_oracle(s.reinit(f=f, g=g).solve(), o.reinit(f=f, g=g).solve())


def test_reinit_warm_start_like_oracle():
    pb = SMALL["port_small"]()
    ref, prob, s, o = _pair(pb)
    loose = init(prob, IPMSettings(gap_tol=1e-2, feas_tol=1e-2)).solve()   # an interior iterate
    for k, kw in enumerate((dict(p0=loose.p, d0=loose.d, y0=loose.y), dict(p0=loose.p), dict(d0=loose.d, y0=loose.y))):
        r = s.reinit(**kw).solve()
        ro = o.reinit(**kw).solve()
        _like_oracle(r, ro)
        if k == 0:   # the full warm start re-solves; the partial ones meet the stale-H first step too
            assert r.status == IPMStatus.OPTIMAL


@pytest.mark.parametrize("which", ["f", "g"])
def test_reinit_before_a_step_equals_fresh_solver(which):
    ctx = Context.default()
    pb = G.socp(n=100, m=40, ncone=5, density=0.1, seed=0)
    pb2 = dict(pb)
    rng = np.random.default_rng(7)
    if which == "f":
        pb2["f"] = pb["f"] + 0.05 * rng.standard_normal(pb["f"].shape)
    else:
        pb2["g"] = pb["g"] * (1 + 0.05 * rng.standard_normal(pb["g"].shape))
    s = init(product_problem(pb, ctx=ctx), IPMSettings())
    r = s.reinit(**{which: pb2[which]}).solve()
    fresh = init(product_problem(pb2, ctx=ctx), IPMSettings()).solve()
    assert fresh.status == IPMStatus.OPTIMAL
    assert r.status == fresh.status and r.niter == fresh.niter
    np.testing.assert_array_equal(r.p, fresh.p)
    np.testing.assert_array_equal(r.y, fresh.y)


def test_solver_timers_and_print_timers(capsys):
    prob = product_problem(SMALL["port_small"](), ctx=Context.default())
    s = init(prob, IPMSettings())
    s.solve()
    t = s.timers()
    assert t["initkkt"] > 0 and t["predictor"] > 0 and t["ntrsv"] > 0
    assert t["factor_update"] + t["factor_diag"] + t["factor_panel"] <= t["initkkt"]
    print_timers(s)
    out = capsys.readouterr().out
    assert "initkkt" in out and "%" in out
