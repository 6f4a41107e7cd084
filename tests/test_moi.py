"""The MathOptInterface front-end (mumblebee_b200.moi, restating src/IPM/src/moi.jl): the
transcription of a standard-form model into the IPM's primal form on the host, and a solve through
it on the device read back in the model's coordinates."""
import numpy as np
import pytest
import scipy.sparse as sp

from mumblebee_b200 import generators as G
from mumblebee_b200 import ipm
from mumblebee_b200.moi import (MAX_SENSE, MIN_SENSE, ExponentialCone, Model, Nonnegatives, Optimizer, PowerCone,
                                ScaledPSDConeTriangle, SecondOrderCone, TERMINATION, coneperm)


def test_coneperm():
    """MOI coordinates in the IPM cone's order: identity, the reversed exponential triple, and the
    lower-column-major svec read from MOI's upper-column-major PSD triangle (moi.jl:130-165)."""
    assert coneperm(SecondOrderCone(4)) == [1, 2, 3, 4]
    assert coneperm(ExponentialCone()) == [3, 2, 1]
    assert coneperm(PowerCone(0.3)) == [1, 2, 3]
    # side 3: MOI upper col-major (1,1)=1 (1,2)=2 (2,2)=3 (1,3)=4 (2,3)=5 (3,3)=6;
    # IPM svec lower col-major (1,1) (2,1) (3,1) (2,2) (3,2) (3,3)
    assert coneperm(ScaledPSDConeTriangle(3)) == [1, 2, 4, 3, 5, 6]


def test_layout_cones_free_block_and_duplicates():
    """Cone blocks in the order added and in the IPM's coordinate order, the remaining variables as
    a trailing free block, and a variable in a second cone copied to a fresh column pinned by a
    coupling row (moi.jl:201-362)."""
    m = Model()
    x = m.add_variables(7)
    c_soc = m.add_cone(x[0:3], SecondOrderCone(3))
    c_exp = m.add_cone(x[3:6], ExponentialCone())
    c_dup = m.add_cone([x[0]], Nonnegatives(1))          # x1 again: a copied column
    z = m.add_zeros([(1, x[0], 2.0), (1, x[6], -1.0), (2, x[1], 1.0)], [3.0, -4.0])
    jmap, K, s, vmap, vidx, jdup, ncol = Optimizer.layout(m)
    assert [k.kind for k in K] == [2, 4, 1, 0] and s == [3, 3, 1, 1] and ncol == 8
    assert [jmap[v] for v in x] == [1, 2, 3, 6, 5, 4, 8]   # the exponential block reversed, x7 free
    assert list(vidx[vmap[c_exp][0]:vmap[c_exp][1]]) == [6, 5, 4]   # MOI coordinate order
    assert jdup == {7: 1}
    B, g, umap = Optimizer.equalities(m, jmap, ncol, jdup)
    Bd = B.toarray()
    assert B.shape == (3, 8) and umap[z] == (0, 2)
    assert Bd[0, 0] == 2.0 and Bd[0, 7] == -1.0 and Bd[1, 1] == 1.0
    np.testing.assert_array_equal(g, [-3.0, 4.0, 0.0])           # A x + b = 0  =>  A x = -b
    np.testing.assert_array_equal(Bd[2], [-1, 0, 0, 0, 0, 0, 1, 0])   # column 7 copies column 1


@pytest.mark.parametrize("sense", [MIN_SENSE, MAX_SENSE])
def test_objective_signs(sense):
    """The IPM minimizes ½pᵀQp − fᵀp: a MAX objective is negated, a diagonal quadratic term
    (a, a, c) is ½ c x_a², an off-diagonal one sits at (a, b) and (b, a) (moi.jl:364-412)."""
    m = Model()
    x = m.add_variables(3)
    m.add_cone(x, Nonnegatives(3))
    m.set_objective(sense, affine=[(x[0], 1.5), (x[2], -2.0)], quadratic=[(x[1], x[1], 4.0), (x[0], x[2], 0.5)],
                    constant=7.0)
    jmap, K, s, vmap, vidx, jdup, ncol = Optimizer.layout(m)
    Q, f, sen, const = Optimizer.objective(m, jmap, ncol)
    sig = -1.0 if sense == MAX_SENSE else 1.0
    np.testing.assert_array_equal(Q.toarray(), sig * np.array([[0, 0, 0.5], [0, 4.0, 0], [0.5, 0, 0]]))
    np.testing.assert_array_equal(f, -sig * np.array([1.5, 0.0, -2.0]))
    assert sen == sense and const == 7.0


def test_status_map():
    assert TERMINATION[ipm.IPMStatus.OPTIMAL] == "OPTIMAL"
    assert TERMINATION[ipm.IPMStatus.NEAR_OPTIMAL] == "ALMOST_OPTIMAL"
    assert TERMINATION[ipm.IPMStatus.PRIMAL_INFEASIBLE] == "INFEASIBLE"
    assert len(TERMINATION) == 11
    assert Optimizer().termination_status() == "OPTIMIZE_NOT_CALLED"


def _model_of(pb, sense=MIN_SENSE):
    """A generator problem written as a model: one cone constraint per cone block (free blocks are
    left to the trailing free block), Bp = g as one Zeros constraint, the objective ½pᵀQp − fᵀp (its
    negation for MAX)."""
    m = Model()
    n = pb["B"].shape[1]
    x = m.add_variables(n)
    o = 0
    for k, sz, a in zip(pb["kinds"], pb["sizes"], pb["params"]):
        vs = x[o:o + sz]
        if k == 1:
            m.add_cone(vs, Nonnegatives(sz))
        elif k == 2:
            m.add_cone(vs, SecondOrderCone(sz))
        elif k == 4:
            m.add_cone(vs[::-1], ExponentialCone())          # MOI's (x, y, z) is the IPM's (c, b, a)
        elif k == 5:
            m.add_cone(vs, PowerCone(a))
        o += sz
    B = sp.coo_matrix(pb["B"])
    zeros = m.add_zeros([(int(i) + 1, x[int(j)], float(v)) for i, j, v in zip(B.row, B.col, B.data)],
                        -np.asarray(pb["g"]))
    Q = sp.coo_matrix(sp.tril(pb["Q"]))
    sig = -1.0 if sense == MAX_SENSE else 1.0
    m.set_objective(sense, affine=[(x[j], -sig * pb["f"][j]) for j in range(n) if pb["f"][j] != 0],
                    quadratic=[(x[int(i)], x[int(j)], sig * float(v)) for i, j, v in zip(Q.row, Q.col, Q.data)],
                    constant=1.25)
    return m, x, zeros


@pytest.mark.gpu
@pytest.mark.parametrize("name,sense", [("portfolio", MIN_SENSE), ("socp", MAX_SENSE), ("exppow", MIN_SENSE)])
def test_optimizer_matches_direct_solve(name, sense):
    """Through the front-end the device solves the same problem as the direct IPMProblem: the
    objective value (sense and constant applied), every variable's value and the Zeros multipliers
    agree, and the Zeros constraint's primal value is its residual.  The front-end orders the
    columns its own way (cone blocks first, then the free block), so the two solves differ by
    rounding; the exponential/power family, whose path is sensitive to rounding (a 1e-7 stopping
    tolerance, as its other parity tests), is held to 1e-6 in the objective and 1e-4 in the
    vectors."""
    from helpers import product_problem
    from mumblebee_b200.ipm import Context, IPMSettings, solve
    pb = {"portfolio": lambda: G.portfolio(40, seed=2), "socp": lambda: G.socp(n=60, m=20, ncone=3, density=0.2, seed=1),
          "exppow": lambda: G.exppow(nexp=10, npow=5, nfree=4, npos=6, m=20, density=0.1, seed=4)}[name]()
    tol = dict(feas_tol=1e-7, gap_tol=1e-7) if name == "exppow" else {}
    m, x, zeros = _model_of(pb, sense)
    opt = Optimizer(IPMSettings(**tol), ctx=Context.default())
    opt.copy_to(m)
    opt.optimize()
    r = solve(product_problem(pb, ctx=Context.default()), IPMSettings(**tol))
    assert opt.termination_status() in ("OPTIMAL", "ALMOST_OPTIMAL") and opt.primal_status() == "FEASIBLE_POINT"
    sig = -1.0 if sense == MAX_SENSE else 1.0
    ot, vt = (1e-6, 1e-4) if name == "exppow" else (1e-7, 1e-6)
    assert abs(opt.objective_value() - (sig * r.pobj + 1.25)) <= ot * max(1.0, abs(r.pobj))
    p = np.array([opt.variable_primal(v) for v in x])
    assert np.linalg.norm(p - r.p) <= vt * max(1.0, np.linalg.norm(r.p))
    y = opt.constraint_dual(zeros)
    assert np.linalg.norm(y - r.y) <= vt * max(1.0, np.linalg.norm(r.y))
    assert np.abs(opt.constraint_primal(zeros)).max() <= 1e-6 * max(1.0, np.abs(pb["g"]).max())
