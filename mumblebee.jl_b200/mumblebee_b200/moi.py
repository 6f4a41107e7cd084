"""The optimizer front-end of the reference's MathOptInterface wrapper (src/IPM/src/moi.jl), for
Python callers: a model in the IPM's primal form, its transcription into an IPMProblem
(`Optimizer.copy_to`), the solve on the device (`optimize`), and the results read back in the
model's coordinates.  The native form is

    min ½ pᵀQp − fᵀp   s.t.   Bp = g,   p ∈ K

written with the standard-form pieces moi.jl accepts (moi.jl:1-16):

    objective            ScalarQuadraticFunction / ScalarAffineFunction, MIN or MAX sense
    Bp = g               VectorAffineFunction-in-Zeros         (Model.add_zeros)
    p ∈ K                VectorOfVariables-in-{cone}           (Model.add_cone)

with the cones Nonnegatives, SecondOrderCone, ExponentialCone, PowerCone and the scaled PSD
triangle (moi.jl:24-30).  Anything else (affine-in-cone, bounds, scalar constraints) is what MOI's
bridges reduce to these in Julia; a Python caller writes the reduced form directly.  The layout,
the coordinate orders of the cones, the coupling rows for a variable in two cones, the objective's
sign conventions and the status map restate moi.jl's.
"""
from __future__ import annotations

import time
from dataclasses import dataclass, field

import numpy as np
import scipy.sparse as sp

from . import ipm
from .ipm import IPMProblem, IPMSettings, IPMStatus

MIN_SENSE, MAX_SENSE = "min", "max"


# ---------------------------------------------------------------------------------------- sets
@dataclass(frozen=True)
class Nonnegatives:
    dimension: int


@dataclass(frozen=True)
class SecondOrderCone:
    dimension: int        # (t, x) with t ≥ ‖x‖


@dataclass(frozen=True)
class ExponentialCone:   # MOI's (x, y, z): y·exp(x / y) ≤ z
    dimension: int = 3


@dataclass(frozen=True)
class PowerCone:         # MOI's (x, y, z): x^α y^(1−α) ≥ |z|
    exponent: float
    dimension: int = 3


@dataclass(frozen=True)
class ScaledPSDConeTriangle:   # the upper triangle, column-major, off-diagonals scaled by √2
    side_dimension: int

    @property
    def dimension(self):
        return self.side_dimension * (self.side_dimension + 1) // 2


def ipmcone(s):
    """The IPM cone of a set (moi.jl:100-128)."""
    if isinstance(s, Nonnegatives):
        return ipm.PositiveCone()
    if isinstance(s, SecondOrderCone):
        return ipm.SecondOrderCone()
    if isinstance(s, ExponentialCone):
        return ipm.ExponentialCone()
    if isinstance(s, PowerCone):
        return ipm.PowerCone(s.exponent)
    if isinstance(s, ScaledPSDConeTriangle):
        return ipm.SemidefiniteCone()
    raise TypeError(f"unsupported cone {s!r}")


def coneperm(s):
    """1-based MOI coordinates in the order the IPM cone lays them out (moi.jl:130-165): the same
    order where the conventions agree, reversed for the exponential cone ((a, b, c) = (z, y, x)),
    and the lower-column-major svec of the PSD cone read from MOI's upper-column-major triangle
    (entry (i, j), i ≤ j, at j(j − 1)/2 + i)."""
    if isinstance(s, ExponentialCone):
        return [3, 2, 1]
    if isinstance(s, ScaledPSDConeTriangle):
        d = s.side_dimension
        return [(i - 1) * i // 2 + j for j in range(1, d + 1) for i in range(j, d + 1)]
    return list(range(1, s.dimension + 1))


# ---------------------------------------------------------------------------------------- model
@dataclass(frozen=True)
class VariableIndex:
    value: int


@dataclass(frozen=True)
class ConstraintIndex:
    kind: str            # "cone" or "zeros"
    value: int


@dataclass
class Model:
    """A standard-form model: variables, VectorOfVariables-in-cone and VectorAffineFunction-in-Zeros
    constraints in the order they were added, and the objective."""
    nvar: int = 0
    cones: list = field(default_factory=list)     # (ConstraintIndex, [VariableIndex], set)
    zeros: list = field(default_factory=list)     # (ConstraintIndex, [(row, VariableIndex, coef)], constants)
    sense: str = MIN_SENSE
    quadratic: list = field(default_factory=list)  # (VariableIndex, VariableIndex, coef): coef·x_a·x_b
    affine: list = field(default_factory=list)     # (VariableIndex, coef)
    constant: float = 0.0

    def add_variable(self) -> VariableIndex:
        self.nvar += 1
        return VariableIndex(self.nvar)

    def add_variables(self, n: int) -> list:
        return [self.add_variable() for _ in range(n)]

    def add_cone(self, variables, s) -> ConstraintIndex:
        """VectorOfVariables-in-set; the variables in the set's own (MOI) coordinate order."""
        if len(variables) != s.dimension:
            raise ValueError(f"{len(variables)} variables for a set of dimension {s.dimension}")
        ci = ConstraintIndex("cone", len(self.cones) + 1)
        self.cones.append((ci, list(variables), s))
        return ci

    def add_zeros(self, terms, constants) -> ConstraintIndex:
        """VectorAffineFunction-in-Zeros: A x + b = 0, terms (output_index (1-based), variable,
        coefficient), b = constants."""
        ci = ConstraintIndex("zeros", len(self.zeros) + 1)
        self.zeros.append((ci, list(terms), np.asarray(constants, dtype=float)))
        return ci

    def set_objective(self, sense=MIN_SENSE, affine=(), quadratic=(), constant=0.0):
        """A ScalarQuadraticFunction (or, with no quadratic terms, a ScalarAffineFunction) in MOI's
        convention: a diagonal term (a, a, c) is ½·c·x_a², an off-diagonal one (a, b, c) is
        c·x_a·x_b; `affine` holds (variable, coefficient) pairs."""
        if sense not in (MIN_SENSE, MAX_SENSE):
            raise ValueError(sense)
        self.sense = sense
        self.affine = list(affine)
        self.quadratic = list(quadratic)
        self.constant = float(constant)


# ---------------------------------------------------------------------------------------- optimizer
# IPMStatus -> MOI termination status (moi.jl:32-44)
TERMINATION = {
    IPMStatus.OPTIMAL: "OPTIMAL", IPMStatus.NEAR_OPTIMAL: "ALMOST_OPTIMAL", IPMStatus.STALLED: "SLOW_PROGRESS",
    IPMStatus.NUMERICAL_FAILURE: "NUMERICAL_ERROR", IPMStatus.ITERATION_LIMIT: "ITERATION_LIMIT",
    IPMStatus.PRIMAL_INFEASIBLE: "INFEASIBLE", IPMStatus.DUAL_INFEASIBLE: "DUAL_INFEASIBLE",
    IPMStatus.ILL_POSED: "INVALID_MODEL", IPMStatus.NEAR_PRIMAL_INFEASIBLE: "ALMOST_INFEASIBLE",
    IPMStatus.NEAR_DUAL_INFEASIBLE: "ALMOST_DUAL_INFEASIBLE", IPMStatus.NEAR_ILL_POSED: "ALMOST_INFEASIBLE",
}


class Optimizer:
    """The Optimizer of moi.jl:50-80: settings, the column-compression threshold, the assembled
    problem and its result, and the maps from the model's variables and constraints to the IPM's
    columns and rows."""

    def __init__(self, settings: IPMSettings | None = None, compress: float = 1.0, ctx=None):
        self.settings = settings or IPMSettings()
        self.compress = compress
        self.ctx = ctx
        self.empty()

    def empty(self):
        self.problem = None
        self.result = None
        self.jmap, self.vmap, self.umap = {}, {}, {}
        self.vidx = np.zeros(0, dtype=np.int64)
        self.sense, self.objconst, self.solvetime = MIN_SENSE, 0.0, 0.0
        self.data = None

    def is_empty(self):
        return self.result is None and not self.jmap

    def _sign(self):
        return -1.0 if self.sense == MAX_SENSE else 1.0

    # ---- copy_to (moi.jl:199-428)
    @staticmethod
    def layout(model: Model):
        """Columns: each cone block contiguous, in the IPM cone's coordinate order, in the order the
        cone constraints were added; then the variables no cone holds, as one trailing free block.
        A variable already placed by one cone gets a fresh column in a second one, pinned to the
        first by a coupling row (moi.jl:201-276).  Returns (jmap, K, s, vmap, vidx, jdup, ncol);
        columns are 1-based, as in moi.jl."""
        K, s, jmap, vmap, jdup = [], [], {}, {}, {}
        vidx = []
        j = 0
        for ci, vars_, st in model.cones:
            jstrt = j
            d = len(vars_)
            vidx.extend([0] * d)
            for k in coneperm(st):
                j += 1
                jx = vars_[k - 1]
                if jx in jmap:
                    jdup[j] = jmap[jx]
                else:
                    jmap[jx] = j
                vidx[jstrt + k - 1] = j
            K.append(ipmcone(st))
            s.append(d)
            vmap[ci] = (jstrt, j)        # vidx[jstrt:j] (0-based slice)
        jstrt = j
        for v in range(1, model.nvar + 1):
            jx = VariableIndex(v)
            if jx not in jmap:
                j += 1
                jmap[jx] = j
        if jstrt < j:
            K.append(ipm.CofreeCone())
            s.append(j - jstrt)
        return jmap, K, s, vmap, np.asarray(vidx, dtype=np.int64), jdup, j

    @staticmethod
    def equalities(model: Model, jmap, ncol, jdup):
        """B and g from the Zeros constraints (A x + b = 0 gives A x = −b), then one row j − k = 0
        per column j copying column k (moi.jl:322-362)."""
        I, J, V, g, umap = [], [], [], [], {}
        i = 0
        for ci, terms, const in model.zeros:
            d = len(const)
            for (row, var, coef) in terms:
                I.append(i + row - 1); J.append(jmap[var] - 1); V.append(float(coef))
            g.extend((-const).tolist())
            umap[ci] = (i, i + d)
            i += d
        for j, k in jdup.items():
            I += [i, i]; J += [j - 1, k - 1]; V += [1.0, -1.0]
            g.append(0.0)
            i += 1
        B = sp.csc_matrix((V, (I, J)), shape=(i, ncol))
        return B, np.asarray(g, dtype=float), umap

    @staticmethod
    def objective(model: Model, jmap, ncol):
        """½pᵀQp − fᵀp for the objective: the IPM minimizes, so a MAX objective is negated
        (σ = −1); Q takes σ·c at (a, b) and (b, a), f takes −σ·c per affine term
        (moi.jl:364-412)."""
        sig = -1.0 if model.sense == MAX_SENSE else 1.0
        I, J, V = [], [], []
        f = np.zeros(ncol)
        for (va, vb, coef) in model.quadratic:
            a, b = jmap[va] - 1, jmap[vb] - 1
            I.append(a); J.append(b); V.append(sig * coef)
            if a != b:
                I.append(b); J.append(a); V.append(sig * coef)
        for (var, coef) in model.affine:
            f[jmap[var] - 1] -= sig * coef
        Q = sp.csc_matrix((V, (I, J)), shape=(ncol, ncol))
        return Q, f, model.sense, model.constant

    def copy_to(self, model: Model):
        """Read the model into an IPMProblem (moi.jl:414-428).  Returns the identity index map."""
        self.empty()
        jmap, K, s, vmap, vidx, jdup, ncol = self.layout(model)
        B, g, umap = self.equalities(model, jmap, ncol, jdup)
        Q, f, sense, objconst = self.objective(model, jmap, ncol)
        self.jmap, self.vmap, self.vidx, self.umap = jmap, vmap, vidx, umap
        self.sense, self.objconst = sense, objconst
        self.data = dict(Q=Q, B=B, f=f, g=g, K=K, s=s)
        self.problem = IPMProblem(Q, B, f, g, 0.0, K, s, compress=self.compress, ctx=self.ctx)
        return {("var", v.value): ("var", v.value) for v in jmap}

    # ---- optimize! (moi.jl:434-439)
    def optimize(self):
        t0 = time.time()
        self.result = ipm.solve(self.problem, self.settings)
        self.solvetime = time.time() - t0

    # ---- results (moi.jl:445-516)
    def raw_status_string(self):
        return self.result.status.name

    def termination_status(self):
        if self.result is None:
            return "OPTIMIZE_NOT_CALLED"
        return TERMINATION.get(self.result.status, "OTHER_ERROR")

    def primal_status(self):
        ok = self.result is not None and self.result.status in (IPMStatus.OPTIMAL, IPMStatus.NEAR_OPTIMAL)
        return "FEASIBLE_POINT" if ok else "NO_SOLUTION"

    dual_status = primal_status

    def result_count(self):
        return 0 if self.result is None else 1

    def variable_primal(self, v: VariableIndex) -> float:
        return float(self.result.p[self.jmap[v] - 1])

    def constraint_primal(self, c: ConstraintIndex):
        """A cone constraint: its variables' values in the set's coordinate order; a Zeros
        constraint: B p − g on its rows (≈ 0)."""
        if c.kind == "cone":
            a, b = self.vmap[c]
            return self.result.p[self.vidx[a:b] - 1]
        r = self.data["B"] @ self.result.p - self.data["g"]
        a, b = self.umap[c]
        return r[a:b]

    def constraint_dual(self, c: ConstraintIndex):
        """A cone constraint: the conic dual d ∈ K* in the set's coordinate order (its sign does not
        follow the objective sense); a Zeros constraint: the multiplier y on its rows."""
        if c.kind == "cone":
            a, b = self.vmap[c]
            return self.result.d[self.vidx[a:b] - 1]
        a, b = self.umap[c]
        return self.result.y[a:b]

    def objective_value(self) -> float:
        return self._sign() * self.result.pobj + self.objconst

    def dual_objective_value(self) -> float:
        return self._sign() * self.result.dobj + self.objconst

    def solve_time_sec(self) -> float:
        return self.solvetime
