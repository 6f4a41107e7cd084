"""Sensitivities frule! / rrule! (src/IPM/src/ipm/differential.jl:5-79, 263-334).

frule! maps seeds on (f, g, μ) to tangents of (p, y, d) through one solve with the KKT matrix at the
current iterate; rrule! applies the transposed map.  The oracle's pair is checked for the adjoint
identity ⟨w, J v⟩ = ⟨Jᵀ w, v⟩ and against central finite differences of the solution; the device
pair is held to the same identity and to the oracle's tangents.  Each rule solves its KKT system to
the reference's tolerance, 0.1·μ_last/μ₀ relative to the right-hand side (differential.jl:9-12),
so the identity holds to about that: 1e-8 on the QPs here, 1e-5 on the SOCP, bounded at 1e-4; the
device and oracle tangents, at iterates that agree to 1e-6, are compared to 1e-3 (1e-2 for the
ill-conditioned SOCP)."""
import numpy as np
import pytest

from helpers import SMALL, block_problem, oracle_solve
from mumblebee_b200.ipm import Context, IPMProblem, IPMSettings, IPMStatus, init


def _seeds(n, m, seed):
    rng = np.random.default_rng(seed)
    return (rng.standard_normal(n), rng.standard_normal(m), 0.7), (rng.standard_normal(n), rng.standard_normal(m),
                                                                  rng.standard_normal(n))


def _adjoint_gap(frule, rrule, n, m, seed=1):
    (df, dg, dmu), (wp, wy, wd) = _seeds(n, m, seed)
    dp, dy, dd = frule(df, dg, dmu)
    fb, gb, mb = rrule(wp, wy, wd)
    lhs = wp @ dp + wy @ dy + wd @ dd
    rhs = fb @ df + gb @ dg + mb * dmu
    return abs(lhs - rhs) / max(1.0, abs(lhs))


@pytest.mark.parametrize("name", ["port_small", "port_mid", "socp_small"])
def test_oracle_rules_are_adjoint(name):
    s, r = oracle_solve(block_problem(SMALL[name]()))
    assert r["status"] == "OPTIMAL"
    assert _adjoint_gap(s.frule, s.rrule, len(r["p"]), len(r["y"])) < 1e-4


def test_oracle_frule_matches_finite_differences():
    pb = SMALL["port_small"]()
    s, r = oracle_solve(block_problem(pb))
    rng = np.random.default_rng(4)
    df = rng.standard_normal(len(r["p"]))
    eps = 1e-5
    tight = dict(gap_tol=1e-12, feas_tol=1e-12, max_iter=200)
    _, rp = oracle_solve(block_problem(dict(pb, f=pb["f"] + eps * df)), **tight)
    _, rm = oracle_solve(block_problem(dict(pb, f=pb["f"] - eps * df)), **tight)
    fd = (rp["p"] - rm["p"]) / (2 * eps)
    dp, _, _ = s.frule(df, None, 0.0)
    assert np.linalg.norm(dp - fd) <= 1e-2 * np.linalg.norm(fd)


@pytest.mark.gpu
@pytest.mark.parametrize("name,tol", [("port_small", 1e-3), ("port_mid", 1e-3), ("socp_small", 1e-2)])
def test_device_rules_match_oracle(name, tol):
    """The SOCP's tangents are about 1e4 times its seeds (its final KKT matrix is ill-conditioned), so
    the 1e-6 difference between the device's and the oracle's final iterates moves them by up to a
    few 1e-3; the QPs agree to 1e-3."""
    ref = block_problem(SMALL[name]())
    prob = IPMProblem.from_dict(ref, ctx=Context.default())
    o, ro = oracle_solve(ref, vperm=prob.symbolic()["vperm"])
    s = init(prob, IPMSettings())
    r = s.solve()
    assert r.status == IPMStatus.OPTIMAL and ro["status"] == "OPTIMAL"
    n, m = len(r.p), len(r.y)
    assert _adjoint_gap(s.frule, s.rrule, n, m) < 1e-4
    (df, dg, dmu), (wp, wy, wd) = _seeds(n, m, 2)
    for a, b in zip(s.frule(df, dg, dmu), o.frule(df, dg, dmu)):
        assert np.linalg.norm(a - b) <= tol * max(1.0, np.linalg.norm(b))
    da, db = s.rrule(wp, wy, wd), o.rrule(wp, wy, wd)
    for a, b in zip(da[:2], db[:2]):
        assert np.linalg.norm(a - b) <= tol * max(1.0, np.linalg.norm(b))
    assert abs(da[2] - db[2]) <= tol * max(1.0, abs(db[2]))


# frule2! (differential.jl:82-260) needs a barrier target μ′ > 0 for its third-order term; the
# problems below solve to the central-path point at μ′ = 0.05, which is smooth in the data
BARRIER = {
    "port": lambda: dict(SMALL["port_small"](), mu=0.05),
    "socp": lambda: dict(SMALL["socp_tiny"](), mu=0.05),
    "sdp": lambda: dict(__import__("helpers").SDP["sdp1x10"](), mu=0.05),
    "exp": lambda: dict(__import__("helpers").TDC["exp_small"](), mu=0.05),
    "pow": lambda: dict(__import__("helpers").TDC["pow_small"](), mu=0.05),
}
TIGHT = dict(gap_tol=1e-12, feas_tol=1e-12, max_iter=200)
TOLS = {"port": TIGHT, "socp": TIGHT, "sdp": {}, "exp": dict(gap_tol=1e-7, feas_tol=1e-7),
        "pow": dict(gap_tol=1e-7, feas_tol=1e-7)}


def _seeds2(n, m, seed=0):
    rng = np.random.default_rng(seed)
    return (rng.standard_normal(n), 0.1 * rng.standard_normal(m), 0.01,
            rng.standard_normal(n), 0.1 * rng.standard_normal(m), -0.02)


def test_oracle_frule2_matches_finite_differences():
    pb = BARRIER["port"]()
    s, r = oracle_solve(block_problem(pb), **TIGHT)
    assert r["status"] == "OPTIMAL"
    n, m = len(r["p"]), len(r["y"])
    df1, dg1, dm1, df2, dg2, dm2 = _seeds2(n, m)
    out = s.frule2(df1, dg1, dm1, df2, dg2, dm2)
    for k, x in enumerate(s.frule(df1, dg1, dm1)):   # the same solve; only the RHS's rounding differs
        np.testing.assert_allclose(out[k], x, rtol=1e-12, atol=1e-12)
    eps = 1e-3

    def p_at(e1, e2):
        q = dict(pb, f=pb["f"] + e1 * df1 + e2 * df2, g=pb["g"] + e1 * dg1 + e2 * dg2, mu=pb["mu"] + e1 * dm1 + e2 * dm2)
        _, rr = oracle_solve(block_problem(q), **TIGHT)
        assert rr["status"] == "OPTIMAL"
        return rr["p"]
    fd = (p_at(eps, eps) - p_at(eps, -eps) - p_at(-eps, eps) + p_at(-eps, -eps)) / (4 * eps * eps)
    assert np.linalg.norm(out[6] - fd) <= 1e-3 * np.linalg.norm(fd)


@pytest.mark.gpu
@pytest.mark.parametrize("name", list(BARRIER))
def test_device_frule2_matches_oracle(name):
    pb = BARRIER[name]()
    ref = block_problem(pb)
    prob = IPMProblem.from_dict(ref, ctx=Context.default())
    o, ro = oracle_solve(ref, vperm=prob.symbolic()["vperm"], **TOLS[name])
    s = init(prob, IPMSettings(**TOLS[name]))
    r = s.solve()
    assert r.status.name == ro["status"] == "OPTIMAL"
    n, m = len(r.p), len(r.y)
    seeds = _seeds2(n, m, 1)
    for a, b in zip(s.frule2(*seeds), o.frule2(*seeds)):
        assert np.linalg.norm(a - b) <= 1e-5 * max(1.0, np.linalg.norm(b))
