"""Shared test helpers: seeded problems, the oracle in the product's vertex order, comparisons."""
import numpy as np

import frontend
import oracle
from mumblebee_b200 import generators as G
from mumblebee_b200.ipm import Context, IPMProblem


def block_problem(pb, compress=1.0):
    """The oracle's restated front-end: CSC problem -> block form dict (1-based)."""
    return frontend.ipmproblem_from_csc(pb["Q"], pb["B"], pb["f"], pb["g"], pb["mu"], pb["kinds"], pb["sizes"],
                                        pb["params"], compress)


def product_problem(pb, ctx=None, compress=1.0):
    K = [_cone(k, a) for k, a in zip(pb["kinds"], pb["params"])]
    return IPMProblem(pb["Q"], pb["B"], pb["f"], pb["g"], pb["mu"], K, pb["sizes"], compress=compress,
                      ctx=ctx or Context.host())


def _cone(k, a):
    from mumblebee_b200 import ipm
    if k == 5:
        return ipm.PowerCone(a)
    return {0: ipm.CofreeCone, 1: ipm.PositiveCone, 2: ipm.SecondOrderCone, 3: ipm.SemidefiniteCone,
            4: ipm.ExponentialCone}[k]()


SMALL = {
    "socp_tiny": lambda: G.socp(n=40, m=12, ncone=4, density=0.2, seed=1),
    "socp_small": lambda: G.socp(n=100, m=40, ncone=5, density=0.1, seed=0),
    "port_small": lambda: G.portfolio(30, seed=3),
    "port_mid": lambda: G.portfolio(80, seed=7),
}


def oracle_solve(prob_blocks, vperm=None, threads=1, **settings):
    s = oracle.OracleSolver(prob_blocks, oracle.default_settings(**settings), vperm=vperm, threads=threads)
    return s, s.solve()

TDC = {
    "exp_small": lambda: G.exppow(nexp=30, npow=0, nfree=0, npos=0, m=40, density=0.05, seed=1),
    "pow_small": lambda: G.exppow(nexp=0, npow=30, nfree=0, npos=0, m=40, density=0.05, seed=1),
    "exppow_mix": lambda: G.exppow(nexp=30, npow=15, nfree=10, npos=20, m=60, density=0.05, seed=3,
                                    determined_free=False),
}
# exponential / power cones stall in the certified line-search band just above a 1e-8 gap (the
# reference's own power-cone examples run at 1e-5..1e-6); their parity runs use 1e-7
TDC_TOL = dict(feas_tol=1e-7, gap_tol=1e-7)

SDP = {
    "sdp3x4": lambda: G.sdp(3, 4, 10, 0.3, 0, 0),
    "sdp2x6_pos": lambda: G.sdp(2, 6, 15, 0.3, 5, 1),
    "sdp4x3": lambda: G.sdp(4, 3, 12, 0.2, 0, 2),
    "sdp1x10": lambda: G.sdp(1, 10, 20, 0.2, 0, 3),
    "maxcut12": lambda: G.maxcut(12, 6, 2, 0),
}


def _lp(B, f, g, kinds, sizes):
    import scipy.sparse as sp
    n = np.asarray(B).shape[1]
    return dict(Q=sp.csc_matrix((n, n)), B=sp.csc_matrix(np.asarray(B, float)), f=np.asarray(f, float),
                g=np.asarray(g, float), mu=0.0, kinds=list(kinds), sizes=list(sizes), params=[0.0] * len(kinds))


def _pinf_pos():
    rng = np.random.default_rng(0)
    return _lp(np.vstack([np.ones(20), rng.standard_normal(20)]), -rng.uniform(0.5, 1, 20), [-1.0, 0.3], [1], [20])


# infeasible and unbounded problems with the status the oracle reaches on them: x >= 0 with
# 1ᵀx = -1; ‖u‖ <= t with t = 1, u1 = 2; an unbounded ray along x1 = x2 >= 0; an unbounded t with
# u1 = 0; and SOCPs with a planted Farkas certificate or unbounded ray (generators.socp_infeasible)
INFEAS = {
    "pinf_pos": (_pinf_pos, "PRIMAL_INFEASIBLE"),
    "pinf_soc": (lambda: _lp([[1, 0, 0], [0, 1, 0]], [-1, 0, 0], [1.0, 2.0], [2], [3]), "NEAR_PRIMAL_INFEASIBLE"),
    "dinf_pos": (lambda: _lp([[1.0, -1.0]], [1.0, 0.0], [0.0], [1], [2]), "DUAL_INFEASIBLE"),
    "dinf_soc": (lambda: _lp([[0, 1.0, 0]], [1.0, 0, 0], [0.0], [2], [3]), "DUAL_INFEASIBLE"),
    "pinf_socp40": (lambda: G.socp_infeasible("primal", 40, 12, 4, 0.1, 0), "PRIMAL_INFEASIBLE"),
    "pinf_socp200": (lambda: G.socp_infeasible("primal", 200, 80, 10, 0.1, 2), "PRIMAL_INFEASIBLE"),
    "pinf_socp500": (lambda: G.socp_infeasible("primal", 500, 200, 25, 0.1, 3), "PRIMAL_INFEASIBLE"),
    "dinf_socp40": (lambda: G.socp_infeasible("dual", 40, 12, 4, 0.1, 0), "DUAL_INFEASIBLE"),
    "dinf_socp100": (lambda: G.socp_infeasible("dual", 100, 40, 5, 0.1, 1), "NEAR_DUAL_INFEASIBLE"),
    "dinf_socp200": (lambda: G.socp_infeasible("dual", 200, 80, 10, 0.1, 2), "DUAL_INFEASIBLE"),
}


def cone_violation(x, kinds, sizes):
    """Largest distance outside the cone product (POS, SOC, free; the self-dual ones) of x,
    measured as max(-x_i) on POS and ‖u‖ - t on SOC."""
    v, o = 0.0, 0
    for k, s in zip(kinds, sizes):
        z = x[o:o + s]
        if k == 1:
            v = max(v, float(-z.min()))
        elif k == 2:
            v = max(v, float(np.linalg.norm(z[1:]) - z[0]))
        o += s
    return v


def _edge(Q, B, f, g, kinds, sizes, mu=0.0):
    import scipy.sparse as sp
    return dict(Q=sp.csc_matrix(np.asarray(Q, float)), B=sp.csc_matrix(np.asarray(B, float)), f=np.asarray(f, float),
                g=np.asarray(g, float), mu=mu, kinds=list(kinds), sizes=list(sizes), params=[0.0] * len(kinds))


def _edge_cases():
    rng = np.random.default_rng(0)
    return {
        # no equality rows: min ½‖p‖² − fᵀp over the orthant
        "m0_qp_pos": _edge(np.eye(5), np.zeros((0, 5)), rng.standard_normal(5), [], [1], [5]),
        # no cones (ν = 0: the exact solve of step!): min ½pᵀQp − fᵀp s.t. Bp = g
        "free_eqqp": _edge(np.diag([2.0, 1.0, 3.0, 1.0]), rng.standard_normal((2, 4)), rng.standard_normal(4),
                           rng.standard_normal(2), [0], [4]),
        # a standard-form LP
        "lp": _edge(np.zeros((6, 6)), np.hstack([np.eye(3), rng.uniform(0.1, 1, (3, 3))]), -rng.uniform(0.5, 1.5, 6),
                    rng.uniform(0.5, 1, 3), [1], [6]),
        # one variable: min p s.t. p = 2, p ≥ 0
        "one_var": _edge(np.zeros((1, 1)), np.ones((1, 1)), [-1.0], [2.0], [1], [1]),
    }


EDGE = _edge_cases()
