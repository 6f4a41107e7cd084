"""settings.stable (the StableUzawaSolver, kkt/uzawa.jl:32-67,117-163): F Fᵀ = δH + BᵀB from the
block-diagonal Cholesky of H updated by the rows of B, without forming BᵀB and without the ρ retry.

The oracle restates it as multifrontal Householder QR of [√δ chol(H_vv)ᵀ; rows of B; children's
triangles] (the reference's update routine, CliqueTrees lowrankupdate!, is not available here; in
exact arithmetic both give the unique Cholesky factor).  Tolerances:
- stable vs the default factor (oracle): the same mathematics with different rounding.  The KKT
  solves stop at their forcing tolerance, so the history rows move apart at about that level.
  The first four rows are held to 1e-5 relative, the final objective to 1e-7.
- device vs oracle (both stable): the same algorithm with different reduction orders and FMA
  contraction.  The portfolio cases and sdp4x3 meet the bar of the default path: the first four
  history rows to 1e-6 relative, same status and iteration count, objectives within 1e-9 relative,
  iterates within 1e-6 relative.  socp_small and sdp1x10 track their first four rows to 1e-6, then
  end optimal or near-optimal with objectives within 1e-6.  Their endgames are decided by rounding:
  the per-vertex Cholesky of an SOC Hessian or of an SDP block's W ⊗ₛ W at μ ≈ 1e-7 (condition
  ≈ 1/μ² ≈ 1e14), as cholblockdiag! runs it in the reference, passes on one side and fails on the
  other, and which side depends on the reduction order.  The exponential and power cases get the
  default path's bar for those cones: the certified step (nflog3 bands) moves with the rounding of
  the direction from the first iteration on, so iteration counts within 2, and objectives within
  1e-6 at an optimal or near-optimal end.
- failures: a free column that no row of B touches gives a zero pivot.  The default path recovers
  through ρ = eps‖F‖; the stable one reports NUMERICAL_FAILURE on its first iteration, as the
  reference does, since it has no retry."""
import numpy as np
import pytest

from helpers import SDP, SMALL, TDC, TDC_TOL, _edge, block_problem, oracle_solve
from mumblebee_b200 import _lib
from mumblebee_b200 import generators as G
from mumblebee_b200.ipm import Context, IPMProblem, IPMSettings, batch_solve, init, solve

CASES = {
    "socp_small": SMALL["socp_small"],
    "port_small": SMALL["port_small"],
    "port_mid": SMALL["port_mid"],
    "sdp4x3": SDP["sdp4x3"],
    "sdp1x10": SDP["sdp1x10"],
    "exp_small": TDC["exp_small"],
    "pow_small": TDC["pow_small"],
}


def _tol(name):
    return TDC_TOL if name in TDC else {}


def _rel(a, b):
    return abs(a - b) / max(1.0, abs(b))


def _zero_column_lp():
    """A standard-form LP plus one free column that no row of B touches (Q = 0, f = 0 there)."""
    rng = np.random.default_rng(0)
    B = np.hstack([np.eye(3), rng.uniform(0.1, 1, (3, 3)), np.zeros((3, 1))])
    return _edge(np.zeros((7, 7)), B, np.r_[-rng.uniform(0.5, 1.5, 6), 0.0], rng.uniform(0.5, 1, 3), [1, 0], [6, 1])


@pytest.mark.parametrize("name", list(CASES))
def test_oracle_stable_tracks_default(name):
    ref = block_problem(CASES[name]())
    _, o0 = oracle_solve(ref, **_tol(name))
    _, o1 = oracle_solve(ref, stable=1, **_tol(name))
    assert o0["status"] == "OPTIMAL" and o1["status"] == "OPTIMAL"
    assert _rel(o1["pobj"], o0["pobj"]) < 1e-7 and _rel(o1["dobj"], o0["dobj"]) < 1e-7
    h0, h1 = o0["history"], o1["history"]
    for i in range(4):
        assert h1[i]["rho"] == 0.0
        for f in ("mu", "pres", "dres", "pobj", "dobj", "step"):
            assert _rel(h1[i][f], h0[i][f]) < 1e-5, (i, f, h1[i][f], h0[i][f])


def test_oracle_stable_zero_pivot_fails():
    ref = block_problem(_zero_column_lp())
    _, o0 = oracle_solve(ref)
    _, o1 = oracle_solve(ref, stable=1)
    assert o0["status"] == "OPTIMAL" and o0["history"][0]["rho"] > 0
    assert o1["status"] == "NUMERICAL_FAILURE" and o1["niter"] == 1


ENDGAME = ("socp_small", "sdp1x10")


@pytest.mark.gpu
@pytest.mark.parametrize("name", list(CASES))
def test_stable_matches_oracle(name):
    ref = block_problem(CASES[name]())
    prob = IPMProblem.from_dict(ref, ctx=Context.default())
    _, o = oracle_solve(ref, vperm=prob.symbolic()["vperm"], stable=1, **_tol(name))
    s = init(prob, IPMSettings(stable=True, **_tol(name)))
    r = s.solve()
    h, oh = s.history(), o["history"]
    assert r.nfactor_retry == 0 and o["status"] == "OPTIMAL"
    if name in TDC:
        assert r.status.name in ("OPTIMAL", "NEAR_OPTIMAL") and abs(r.niter - o["niter"]) <= 2
        assert _rel(r.pobj, o["pobj"]) < 1e-6 and _rel(r.dobj, o["dobj"]) < 1e-6
        return
    for i in range(4):
        for f in ("mu", "pres", "dres", "pobj", "dobj", "step"):
            assert _rel(h[i][f], oh[i][f]) < 1e-6, (i, f, h[i][f], oh[i][f])
    if name in ENDGAME:
        assert r.status.name in ("OPTIMAL", "NEAR_OPTIMAL")
        assert _rel(r.pobj, o["pobj"]) < 1e-6 and _rel(r.dobj, o["dobj"]) < 1e-6
        return
    assert r.status.name == o["status"] and r.niter == o["niter"]
    assert _rel(r.pobj, o["pobj"]) < 1e-9 and _rel(r.dobj, o["dobj"]) < 1e-9
    for k in ("p", "d", "y"):
        a, b = getattr(r, k), o[k]
        assert np.linalg.norm(a - b) <= 1e-6 * max(1.0, np.linalg.norm(b)), k


@pytest.mark.gpu
@pytest.mark.parametrize("which", ["zero_column", "exppow_mix"])
def test_stable_failure_matches_oracle(which):
    pb = _zero_column_lp() if which == "zero_column" else TDC["exppow_mix"]()
    ref = block_problem(pb)
    prob = IPMProblem.from_dict(ref, ctx=Context.default())
    _, o = oracle_solve(ref, vperm=prob.symbolic()["vperm"], stable=1, **TDC_TOL)
    r = solve(prob, IPMSettings(stable=True, **TDC_TOL))
    assert o["status"] == "NUMERICAL_FAILURE"
    assert r.status.name == o["status"] and r.niter == o["niter"]


@pytest.mark.gpu
def test_stable_batch_equals_alone():
    """A stable batch of mixed sizes gives each instance's lone result bit for bit."""
    pbs = [CASES[k]() for k in ("socp_small", "port_small", "sdp4x3")] + [G.portfolio(60, seed=5)]
    probs = [IPMProblem.from_dict(block_problem(p), ctx=Context.default()) for p in pbs]
    st = IPMSettings(stable=True)
    mix = batch_solve(probs, st, grid=2)
    for p, r in zip(probs, mix):
        a = solve(p, st)
        assert a.status == r.status and a.niter == r.niter
        np.testing.assert_array_equal(a.p, r.p)


@pytest.mark.gpu
def test_stable_rejections():
    ctx = Context.default()
    prob = IPMProblem.from_dict(block_problem(SMALL["socp_tiny"]()), ctx=ctx)
    with pytest.raises(_lib.MBError, match="precision must be 0"):
        solve(prob, IPMSettings(stable=True, precision="mixed"))
    # Q coupling two cone vertices: the reference copies H into its block diagonal (uzawa.jl:136)
    pb = SMALL["socp_tiny"]()
    Q = pb["Q"].toarray()
    Q[0, 10] = Q[10, 0] = 0.01
    import scipy.sparse as sp
    pb["Q"] = sp.csc_matrix(Q + np.eye(Q.shape[0]))
    coupled = IPMProblem.from_dict(block_problem(pb), ctx=ctx)
    with pytest.raises(_lib.MBError, match="off-diagonal"):
        solve(coupled, IPMSettings(stable=True))


# Sensitivities under the stable factor: frule! / rrule! / frule2! call initkkt! (differential.jl:7,
# 94, 260), which the stable setting routes to its own factor.  At the barrier points of μ′ = 0.05
# (a well-conditioned KKT matrix) the stable and default factors give the same tangents up to the
# rules' solve tolerance, and the device's stable rules follow the oracle's as the default ones do.
SENS = ("port", "sdp")


def _barrier(name):
    from test_sensitivities import BARRIER, TOLS
    return BARRIER[name](), TOLS[name]


@pytest.mark.parametrize("name", SENS)
def test_oracle_stable_rules_match_default(name):
    from test_sensitivities import _adjoint_gap, _seeds, _seeds2
    pb, tol = _barrier(name)
    ref = block_problem(pb)
    o0, r0 = oracle_solve(ref, **tol)
    o1, r1 = oracle_solve(ref, stable=1, **tol)
    assert r0["status"] == r1["status"] == "OPTIMAL"
    n, m = len(r1["p"]), len(r1["y"])
    assert _adjoint_gap(o1.frule, o1.rrule, n, m) < 1e-4
    (df, dg, dmu), _ = _seeds(n, m, 2)
    for a, b in zip(o1.frule(df, dg, dmu), o0.frule(df, dg, dmu)):
        assert np.linalg.norm(a - b) <= 1e-5 * max(1.0, np.linalg.norm(b))
    seeds = _seeds2(n, m, 1)
    for a, b in zip(o1.frule2(*seeds), o0.frule2(*seeds)):
        assert np.linalg.norm(a - b) <= 1e-5 * max(1.0, np.linalg.norm(b))


@pytest.mark.gpu
@pytest.mark.parametrize("name", SENS)
def test_device_stable_rules_match_oracle(name):
    from test_sensitivities import _adjoint_gap, _seeds, _seeds2
    pb, tol = _barrier(name)
    ref = block_problem(pb)
    prob = IPMProblem.from_dict(ref, ctx=Context.default())
    o, ro = oracle_solve(ref, vperm=prob.symbolic()["vperm"], stable=1, **tol)
    s = init(prob, IPMSettings(stable=True, **tol))
    r = s.solve()
    assert r.status.name == ro["status"] == "OPTIMAL"
    n, m = len(r.p), len(r.y)
    assert _adjoint_gap(s.frule, s.rrule, n, m) < 1e-4
    (df, dg, dmu), (wp, wy, wd) = _seeds(n, m, 2)
    for a, b in zip(s.frule(df, dg, dmu), o.frule(df, dg, dmu)):
        assert np.linalg.norm(a - b) <= 1e-5 * max(1.0, np.linalg.norm(b))
    da, db = s.rrule(wp, wy, wd), o.rrule(wp, wy, wd)
    for a, b in zip(da[:2], db[:2]):
        assert np.linalg.norm(a - b) <= 1e-5 * max(1.0, np.linalg.norm(b))
    seeds = _seeds2(n, m, 1)
    for a, b in zip(s.frule2(*seeds), o.frule2(*seeds)):
        assert np.linalg.norm(a - b) <= 1e-5 * max(1.0, np.linalg.norm(b))
