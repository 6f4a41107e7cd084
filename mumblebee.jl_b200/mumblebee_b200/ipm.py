"""Python mirror of Mumblebee.jl's `IPM` solver API over libmbgpu.so.

Same names and argument meaning as the reference (src/IPM/IPM.jl:42-47 exports):

    IPMProblem(Q, B, f, g, μ, K, s; compress)   problem.jl:84-127  (CSC input)
    IPMProblem.from_blocks(Q, B, f, g, μ, K)    problem.jl:49-71   (BlockSparseMatrix input)
    IPMSettings(...)                            settings/ipm.jl:1-18
    init(prob, settings; p0, d0, y0)            solver/ipm.jl:485-491
    step(solver)      — step!(solver)           solver/ipm.jl:577-774
    solve_(solver)    — solve!(solver)          solver/solver.jl:147-150
    solve(prob, settings)                       solver/ipm.jl:798-804
    IPMResult / IPMHistory / IPMStatus          result/ipm.jl, history/ipm.jl, ipm/ipm.jl:1

The numeric work runs on the GPU; there is no CPU path.  `batch_solve` solves many problems in one
persistent launch.
"""
from __future__ import annotations

import ctypes as C
import enum
from dataclasses import dataclass, field, fields

import numpy as np
import scipy.sparse as sp

from . import _lib
from ._lib import check, mb_bsm, mb_csc, mb_history_row, mb_result, mb_settings, ROW_FIELDS


class IPMStatus(enum.IntEnum):
    CONTINUE = 0
    OPTIMAL = 1
    NEAR_OPTIMAL = 2
    STALLED = 3
    NUMERICAL_FAILURE = 4
    ITERATION_LIMIT = 5
    PRIMAL_INFEASIBLE = 6
    DUAL_INFEASIBLE = 7
    ILL_POSED = 8
    NEAR_PRIMAL_INFEASIBLE = 9
    NEAR_DUAL_INFEASIBLE = 10
    NEAR_ILL_POSED = 11


class KKTStatus(enum.IntEnum):
    KKT_CONTINUE = 0
    KKT_SOLVED = 1
    KKT_STAGNATED = 2
    KKT_ITMAX = 3
    KKT_NUMERICAL_FAILURE = 4
    KKT_IRMAX = 5


# ---------------------------------------------------------------------------------------- cones
class AbstractCone:
    kind = -1
    param = 0.0


class CofreeCone(AbstractCone):
    kind = 0


class PositiveCone(AbstractCone):
    kind = 1


class SecondOrderCone(AbstractCone):
    kind = 2


class SemidefiniteCone(AbstractCone):
    kind = 3


class ExponentialCone(AbstractCone):
    kind = 4


class PowerCone(AbstractCone):
    kind = 5

    def __init__(self, alpha: float):
        self.param = float(alpha)


_CONES = {0: CofreeCone, 1: PositiveCone, 2: SecondOrderCone, 3: SemidefiniteCone, 4: ExponentialCone, 5: PowerCone}


# ---------------------------------------------------------------------------------------- settings
@dataclass
class IPMSettings:
    verbose: int = 0
    step_frac: float = 0.99
    feas_tol: float = 1e-8
    gap_tol: float = 1e-8
    max_iter: int = 100
    near_factor: float = 1000.0
    stall_tol: float = 1e-3
    refine_stall_tol: float = 0.5
    scale_max_iter: int = 10
    refine_max_iter: int = 10
    newton_max_iter: int = 100
    aug_tol: float = 1e-7
    stable: bool = False             # StableUzawaSolver factor (FP64 only; Q block-diagonal)
    infeas_abs: float = 1e-8
    infeas_rel: float = 1e-8
    precision: str = "fp64"          # "fp64", "fp32" or "mixed" (factor precision; refinement stays FP64)
    large: int = 0                   # a lone large instance runs grid-cooperatively: 0 auto, 1 always, -1 never
    coop_wait: float = 60.0          # seconds a CTA of that mode waits at a grid barrier (then MB_E_TIMEOUT)
    fp32_tiles: int = 0              # FP32 factor update tiles: 0 auto, 1 FFMA, 2 tensor cores (tcgen05, 3xTF32)

    def to_c(self) -> mb_settings:
        s = mb_settings()
        for f in fields(self):
            if f.name == "precision":
                s.precision = {"fp64": 0, "fp32": 1, "mixed": 2}[self.precision]
            elif f.name == "stable":
                s.stable = int(self.stable)
            else:
                setattr(s, f.name, getattr(self, f.name))
        return s


# ---------------------------------------------------------------------------------------- context
class Context:
    """One device and one stream (mb_ctx).  `Context.host()` is a GPU-less context for problem
    construction and symbolic analysis only."""
    _default: dict = {}
    _host = None

    def __init__(self, device: int = 0):
        self.L = _lib.load()
        h = C.c_void_p()
        rc = self.L.mb_ctx_create(device, C.byref(h))
        if rc != 0:
            raise _lib.MBError(f"mb_ctx_create({device}) failed with code {rc} (no CUDA device?)")
        self.h = h
        self.device = device

    @classmethod
    def host(cls) -> "Context":
        if cls._host is None:
            c = cls.__new__(cls)
            c.L = _lib.load(); c.h = None; c.device = -1
            cls._host = c
        return cls._host

    @classmethod
    def default(cls, device: int = 0) -> "Context":
        if device not in cls._default:
            cls._default[device] = cls(device)
        return cls._default[device]

    def __del__(self):
        if getattr(self, "h", None):
            self.L.mb_ctx_destroy(self.h)
            self.h = None


def _a64(x):
    return np.ascontiguousarray(x, dtype=np.int64)


def _f64(x):
    return np.ascontiguousarray(x, dtype=np.float64)


def _p(a, t):
    return None if a is None else a.ctypes.data_as(C.POINTER(t))


# ---------------------------------------------------------------------------------------- problem
class IPMProblem:
    """A primal-dual pair of conic QPs (problem.jl:1-19):

        (P) min ½pᵀQp − fᵀp  s.t. Bp = g, p ∈ K
        (D) max −½pᵀQp + gᵀy  s.t. Qp − f − Bᵀy = d ∈ K*
    """

    def __init__(self, Q, B, f, g, mu, K, s, compress: float = 1.0, ctx: Context | None = None):
        self.ctx = ctx or Context.default()
        L = self.ctx.L
        Qc = sp.csc_matrix(Q); Bc = sp.csc_matrix(B)
        Qc.sort_indices(); Bc.sort_indices()
        keep = []

        def csc(A):
            cp = _a64(A.indptr + 1); rv = _a64(A.indices + 1); nz = _f64(A.data)
            keep.extend([cp, rv, nz])
            return mb_csc(A.shape[0], A.shape[1], _p(cp, C.c_int64), _p(rv, C.c_int64), _p(nz, C.c_double))

        kinds = np.array([k.kind for k in K], dtype=np.int32)
        params = _f64([k.param for k in K])
        sizes = _a64(s)
        fv, gv = _f64(f), _f64(g)
        q, b = csc(Qc), csc(Bc)
        h = C.c_void_p()
        rc = L.mb_problem_create_csc(self.ctx.h, C.byref(q), C.byref(b), _p(fv, C.c_double), _p(gv, C.c_double),
                                     float(mu), len(K), _p(kinds, C.c_int32), _p(sizes, C.c_int64),
                                     _p(params, C.c_double), float(compress), C.byref(h))
        check(rc, self.ctx.h, "IPMProblem")
        self.h = h
        self.mu = float(mu)

    @classmethod
    def from_blocks(cls, Q: dict, B: dict, f, g, mu, K, P1=None, P2=None, ctx: Context | None = None, params=None):
        """IPMProblem(Q::BlockSparseMatrix, B::BlockSparseMatrix, f, g, μ, K[, P1, P2]); Q/B are dicts
        with the 1-based BlockSparseMatrix fields (nout, nvtx, narc, ncol, nrow, nbnz, xsrc, xcol,
        xrow, xblk, tgt, val)."""
        self = cls.__new__(cls)
        self.ctx = ctx or Context.default()
        L = self.ctx.L
        keep = []

        def bsm(d):
            a = {k: _a64(d[k]) for k in ("xsrc", "xcol", "xrow", "xblk", "tgt")}
            a["val"] = _f64(d["val"])
            keep.extend(a.values())
            return mb_bsm(d["nout"], d["nvtx"], d["narc"], d["ncol"], d["nrow"], d["nbnz"],
                          *[_p(a[k], C.c_int64) for k in ("xsrc", "xcol", "xrow", "xblk", "tgt")],
                          _p(a["val"], C.c_double))

        if len(K) and isinstance(K[0], AbstractCone):
            kinds = np.array([k.kind for k in K], dtype=np.int32)
            params = _f64([k.param for k in K])
        else:
            kinds = np.ascontiguousarray(K, dtype=np.int32)
            params = _f64(np.zeros(len(kinds)) if params is None else params)
        q, b = bsm(Q), bsm(B)
        fv, gv = _f64(f), _f64(g)
        p1 = None if P1 is None else _a64(P1)
        p2 = None if P2 is None else _a64(P2)
        h = C.c_void_p()
        rc = L.mb_problem_create(self.ctx.h, C.byref(q), C.byref(b), _p(fv, C.c_double), _p(gv, C.c_double),
                                 float(mu), _p(kinds, C.c_int32), _p(params, C.c_double), _p(p1, C.c_int64),
                                 _p(p2, C.c_int64), C.byref(h))
        check(rc, self.ctx.h, "IPMProblem")
        self.h = h
        self.mu = float(mu)
        return self

    @classmethod
    def from_dict(cls, d: dict, ctx: Context | None = None):
        return cls.from_blocks(d["Q"], d["B"], d["f"], d["g"], d["mu"], d["kind"], d.get("P1"), d.get("P2"), ctx=ctx,
                               params=d.get("param"))

    def info(self):
        """n, m, vertices, outputs and block counts (read once: a problem's shape never changes)"""
        if getattr(self, "_info", None) is None:
            a = np.zeros(8, dtype=np.int64)
            self.ctx.L.mb_problem_info(self.h, _p(a, C.c_int64))
            self._info = dict(zip(["n", "m", "nvtx", "nout", "narcB", "nbnzB", "narcQ", "nbnzQ"], a.tolist()))
        return dict(self._info)

    def _nm(self):
        if getattr(self, "_info", None) is None:
            self.info()
        return self._info["n"], self._info["m"]

    @property
    def n(self):
        return self.info()["n"]

    @property
    def m(self):
        return self.info()["m"]

    def blocks(self) -> dict:
        """The block form (BlockSparseMatrix fields, 1-based), as the reference stores IPMProblem."""
        i = self.info()
        nv, no, nab, nbb, naq, nbq = i["nvtx"], i["nout"], i["narcB"], i["nbnzB"], i["narcQ"], i["nbnzQ"]
        n, m = i["n"], i["m"]
        Bx = [np.zeros(nv + 1, np.int64), np.zeros(nv + 1, np.int64), np.zeros(no + 1, np.int64),
              np.zeros(nab + 1, np.int64), np.zeros(nab, np.int64), np.zeros(nbb)]
        Qx = [np.zeros(nv + 1, np.int64), np.zeros(naq + 1, np.int64), np.zeros(naq, np.int64), np.zeros(nbq)]
        f = np.zeros(n); g = np.zeros(m); kind = np.zeros(nv, np.int32); par = np.zeros(nv)
        P1 = np.zeros(m, np.int64); P2 = np.zeros(n, np.int64)
        self.ctx.L.mb_problem_export(self.h, *[_p(a, C.c_int64) for a in Bx[:5]], _p(Bx[5], C.c_double),
                                     _p(Qx[0], C.c_int64), _p(Qx[1], C.c_int64), _p(Qx[2], C.c_int64),
                                     _p(Qx[3], C.c_double), _p(f, C.c_double), _p(g, C.c_double),
                                     _p(kind, C.c_int32), _p(par, C.c_double), _p(P1, C.c_int64), _p(P2, C.c_int64))
        B = dict(nout=no, nvtx=nv, narc=nab, ncol=n, nrow=m, nbnz=nbb, xsrc=Bx[0], xcol=Bx[1], xrow=Bx[2],
                 xblk=Bx[3], tgt=Bx[4], val=Bx[5])
        Q = dict(nout=nv, nvtx=nv, narc=naq, ncol=n, nrow=n, nbnz=nbq, xsrc=Qx[0], xcol=Bx[1], xrow=Bx[1],
                 xblk=Qx[1], tgt=Qx[2], val=Qx[3])
        return dict(Q=Q, B=B, f=f, g=g, mu=self.mu, kind=kind, param=par, P1=P1, P2=P2)

    def footprint(self, settings: "IPMSettings | None" = None) -> int:
        """Device bytes of one instance (mb_problem_footprint)."""
        cs = (settings or IPMSettings()).to_c()
        b = C.c_int64()
        check(self.ctx.L.mb_problem_footprint(self.h, C.byref(cs), C.byref(b)), self.ctx.h, "footprint")
        return b.value

    def symbolic(self) -> dict:
        """The host symbolic analysis: solver vertex order (0-based problem vertices) and fronts."""
        i = self.info()
        nv = i["nvtx"]
        vperm = np.zeros(nv, np.int64)
        cap = nv
        arrs = [np.zeros(cap, np.int64) for _ in range(4)]
        nf = C.c_int64()
        self.ctx.L.mb_problem_symbolic(self.h, _p(vperm, C.c_int64), C.byref(nf),
                                       *[_p(a, C.c_int64) for a in arrs], cap)
        k = nf.value
        return dict(vperm=vperm, nfront=k, res0=arrs[0][:k], nres=arrs[1][:k], nsep=arrs[2][:k], parent=arrs[3][:k])

    def __del__(self):
        if getattr(self, "h", None):
            self.ctx.L.mb_problem_destroy(self.h)
            self.h = None


# ---------------------------------------------------------------------------------------- results
@dataclass
class IPMHistory:
    rows: list = field(default_factory=list)

    def __len__(self):
        return len(self.rows)

    def __getitem__(self, i):
        return self.rows[i]

    def column(self, name):
        return np.array([r[name] for r in self.rows])


@dataclass
class IPMResult:
    p: np.ndarray
    d: np.ndarray
    y: np.ndarray
    status: IPMStatus
    niter: int
    nsolve: int
    history: IPMHistory
    mu: float
    pres: float
    dres: float
    pobj: float
    dobj: float
    nfactor_retry: int = 0
    nfactor: int = 0
    factor_flops: float = 0.0
    nfp32: int = 0
    nfallback: int = 0


class IPMSolver:
    """Device-resident solver state (IPMSolver, solver/ipm.jl:1-28)."""

    def __init__(self, prob: IPMProblem, settings: IPMSettings | None = None, p0=None, d0=None, y0=None):
        self.prob = prob
        self.settings = settings or IPMSettings()
        self.L = prob.ctx.L
        self._cs = self.settings.to_c()
        h = C.c_void_p()
        a = [None if x is None else _f64(x) for x in (p0, d0, y0)]
        rc = self.L.mb_solver_create(prob.h, C.byref(self._cs), *[_p(x, C.c_double) for x in a], C.byref(h))
        check(rc, prob.ctx.h, "init")
        self.h = h
        self.status = IPMStatus.CONTINUE

    def step(self) -> IPMStatus:
        st = C.c_int32()
        check(self.L.mb_solver_step(self.h, C.byref(st)), self.prob.ctx.h, "step!")
        self.status = IPMStatus(st.value)
        return self.status

    def solve(self) -> IPMResult:
        st = C.c_int32()
        check(self.L.mb_solver_solve(self.h, C.byref(st)), self.prob.ctx.h, "solve!")
        self.status = IPMStatus(st.value)
        return self.result()

    def reinit(self, p0=None, d0=None, y0=None, f=None, g=None) -> "IPMSolver":
        """reinit!(s; p0, d0, y0, f, g) (solver/ipm.jl:371-429): restart from the cone identity, or from
        the given p0/d0/y0 completed by shadows, with an empty history, on a new f and/or g when
        given (user order).  The equilibration, Q, B and BᵀB of init stay."""
        a = [None if x is None else _f64(x) for x in (p0, d0, y0, f, g)]
        check(self.L.mb_solver_reinit(self.h, *[_p(x, C.c_double) for x in a]), self.prob.ctx.h, "reinit!")
        self.status = IPMStatus.CONTINUE
        return self

    def frule(self, df=None, dg=None, dmu=0.0):
        """frule!(Δp, Δy, Δd, s, Δf, Δg, Δμ) (ipm/differential.jl:5-79): the tangents (Δp, Δy, Δd) of the
        current iterate for seeds Δf (n), Δg (m), Δμ; user order, None = 0."""
        i = self.prob.info()
        dp, dd, dy = np.zeros(i["n"]), np.zeros(i["n"]), np.zeros(i["m"])
        a = [None if x is None else _f64(x) for x in (df, dg)]
        check(self.L.mb_solver_frule(self.h, _p(a[0], C.c_double), _p(a[1], C.c_double), float(dmu),
                                     _p(dp, C.c_double), _p(dy, C.c_double), _p(dd, C.c_double)), self.prob.ctx.h, "frule!")
        return dp, dy, dd

    def frule2(self, df1=None, dg1=None, dmu1=0.0, df2=None, dg2=None, dmu2=0.0):
        """frule2! (ipm/differential.jl:82-260): the first-order tangents for two seed sets and the
        second-order tangent, as (Δp1, Δy1, Δd1, Δp2, Δy2, Δd2, Δp12, Δy12, Δd12); user order."""
        i = self.prob.info()
        outs = [np.zeros(i["m"] if k % 3 == 1 else i["n"]) for k in range(9)]
        arr = (C.POINTER(C.c_double) * 9)(*[_p(x, C.c_double) for x in outs])
        a = [None if x is None else _f64(x) for x in (df1, dg1, df2, dg2)]
        check(self.L.mb_solver_frule2(self.h, _p(a[0], C.c_double), _p(a[1], C.c_double), float(dmu1),
                                      _p(a[2], C.c_double), _p(a[3], C.c_double), float(dmu2), arr),
              self.prob.ctx.h, "frule2!")
        return tuple(outs)

    def rrule(self, dp=None, dy=None, dd=None):
        """rrule!(Δf, Δg, s, Δp, Δy, Δd) (ipm/differential.jl:263-334): the cotangents (Δf, Δg, Δμ) for
        seeds Δp (n), Δy (m), Δd (n); user order, None = 0."""
        i = self.prob.info()
        df, dg, dmu = np.zeros(i["n"]), np.zeros(i["m"]), C.c_double()
        a = [None if x is None else _f64(x) for x in (dp, dy, dd)]
        check(self.L.mb_solver_rrule(self.h, *[_p(x, C.c_double) for x in a], _p(df, C.c_double),
                                     _p(dg, C.c_double), C.byref(dmu)), self.prob.ctx.h, "rrule!")
        return df, dg, dmu.value

    SECTIONS = ["equilibrate", "BtB", "scale", "initkkt", "predictor", "corrector", "maxsteps", "trsv", "gemv",
                "assemble", "residual", "getaug", "factor_update", "factor_diag", "factor_panel", "extend_add",
                "ntrsv", "ngemv"]

    def timers(self) -> dict:
        """The solver's section clocks (SM cycles; TimerOutput sections of the reference plus set-up and
        the factor's parts), and the counts of triangular-solve sweeps and matvecs."""
        a = np.zeros(len(self.SECTIONS))
        check(self.L.mb_solver_timers(self.h, _p(a, C.c_double), a.size), self.prob.ctx.h, "timers")
        return dict(zip(self.SECTIONS, a.tolist()))

    def print_timers(self, file=None):
        """print_timers(s): one line per section, SM cycles and share of the iteration sections."""
        t = self.timers()
        top = ["equilibrate", "BtB", "scale", "initkkt", "predictor", "corrector", "maxsteps", "residual", "getaug"]
        tot = sum(t[k] for k in top) or 1.0
        for k in self.SECTIONS:
            v = t[k]
            share = f"{100 * v / tot:5.1f} %" if k not in ("ntrsv", "ngemv") else ""
            print(f"{k:14s} {v:16.0f} {share}", file=file)

    def history(self) -> IPMHistory:
        cap = self.settings.max_iter + 1
        rows = (mb_history_row * cap)()
        nr = C.c_int32()
        check(self.L.mb_solver_history(self.h, rows, cap, C.byref(nr)), self.prob.ctx.h, "history")
        return IPMHistory([{f: getattr(rows[i], f) for f in ROW_FIELDS} for i in range(nr.value)])

    def result(self) -> IPMResult:
        i = self.prob.info()
        p = np.zeros(i["n"]); d = np.zeros(i["n"]); y = np.zeros(i["m"])
        r = mb_result()
        check(self.L.mb_solver_result(self.h, _p(p, C.c_double), _p(d, C.c_double), _p(y, C.c_double), C.byref(r)),
              self.prob.ctx.h, "result")
        return IPMResult(p, d, y, IPMStatus(r.status), r.niter, r.nsolve, self.history(), r.mu, r.pres, r.dres,
                         r.pobj, r.dobj, r.nfactor_retry, r.nfactor, r.factor_flops, r.nfp32, r.nfallback)

    def __del__(self):
        if getattr(self, "h", None):
            self.L.mb_solver_destroy(self.h)
            self.h = None


def frule(solver: IPMSolver, df=None, dg=None, dmu=0.0):
    """frule!(Δp, Δy, Δd, solver, Δf, Δg, Δμ) → (Δp, Δy, Δd)"""
    return solver.frule(df, dg, dmu)


def frule2(solver: IPMSolver, df1=None, dg1=None, dmu1=0.0, df2=None, dg2=None, dmu2=0.0):
    """frule2!(…, solver, Δf1, Δg1, Δμ1, Δf2, Δg2, Δμ2) → nine tangents"""
    return solver.frule2(df1, dg1, dmu1, df2, dg2, dmu2)


def rrule(solver: IPMSolver, dp=None, dy=None, dd=None):
    """rrule!(Δf, Δg, solver, Δp, Δy, Δd) → (Δf, Δg, Δμ)"""
    return solver.rrule(dp, dy, dd)


def reinit(solver: IPMSolver, p0=None, d0=None, y0=None, f=None, g=None) -> IPMSolver:
    """reinit!(solver; p0, d0, y0, f, g)"""
    return solver.reinit(p0, d0, y0, f, g)


def print_timers(solver: IPMSolver, file=None):
    """print_timers(solver)"""
    solver.print_timers(file)


def init(prob: IPMProblem, settings: IPMSettings | None = None, p0=None, d0=None, y0=None) -> IPMSolver:
    return IPMSolver(prob, settings, p0, d0, y0)


def step(solver: IPMSolver) -> IPMStatus:
    """step!(solver)"""
    return solver.step()


def solve_(solver: IPMSolver) -> IPMResult:
    """solve!(solver)"""
    return solver.solve()


def solve(prob: IPMProblem, settings: IPMSettings | None = None, p0=None, d0=None, y0=None) -> IPMResult:
    return init(prob, settings, p0, d0, y0).solve()


# ---------------------------------------------------------------------------------------- batches
class Batch:
    """Many problems resident on the device, solved by one persistent launch per `run`."""

    def __init__(self, probs, settings: IPMSettings | None = None, ctx: Context | None = None):
        self.ctx = ctx or probs[0].ctx
        self.L = self.ctx.L
        self.probs = list(probs)
        self.settings = settings or IPMSettings()
        self._cs = self.settings.to_c()
        arr = (C.c_void_p * len(self.probs))(*[p.h.value for p in self.probs])
        h = C.c_void_p()
        check(self.L.mb_batch_prepare(self.ctx.h, arr, len(self.probs), C.byref(self._cs), C.byref(h)),
              self.ctx.h, "batch prepare")
        self.h = h
        self.sizes = [p.info() for p in self.probs]

    def run(self, grid: int = 0) -> float:
        ms = C.c_float()
        check(self.L.mb_batch_run(self.h, grid, C.byref(ms)), self.ctx.h, "batch run")
        return ms.value

    def fetch(self, want_vectors: bool = True):
        k = len(self.probs)
        res = (mb_result * k)()
        if want_vectors:
            ps = [np.zeros(s["n"]) for s in self.sizes]
            ds = [np.zeros(s["n"]) for s in self.sizes]
            ys = [np.zeros(s["m"]) for s in self.sizes]
            mk = lambda lst: (C.POINTER(C.c_double) * k)(*[_p(a, C.c_double) for a in lst])
            check(self.L.mb_batch_fetch(self.h, mk(ps), mk(ds), mk(ys), res), self.ctx.h, "batch fetch")
        else:
            ps = ds = ys = [None] * k
            check(self.L.mb_batch_fetch(self.h, None, None, None, res), self.ctx.h, "batch fetch")
        out = []
        for i in range(k):
            r = res[i]
            out.append(IPMResult(ps[i], ds[i], ys[i], IPMStatus(r.status), r.niter, r.nsolve, IPMHistory(), r.mu,
                                 r.pres, r.dres, r.pobj, r.dobj, r.nfactor_retry, r.nfactor, r.factor_flops, r.nfp32, r.nfallback))
        return out

    SECTIONS = ["equilibrate", "BtB", "scale", "initkkt", "predictor", "corrector", "maxsteps", "trsv", "gemv",
                "assemble", "residual", "getaug", "factor_update", "factor_diag", "factor_panel", "extend_add",
                "ntrsv", "ngemv"]

    def timers(self):
        """Per-instance section clocks (after fetch): array (ninst, len(SECTIONS)), columns SECTIONS.  The
        factor_* and extend_add clocks are part of initkkt; trsv and gemv are part of predictor and
        corrector; the last two columns count triangular-solve sweeps and matvecs."""
        W = len(self.SECTIONS)
        a = np.zeros(len(self.probs) * W)
        check(self.L.mb_batch_timers(self.h, _p(a, C.c_double), a.size), self.ctx.h, "timers")
        return a.reshape(len(self.probs), W)

    def times(self):
        """Per-instance GPU global-timer stamps (after fetch), int64 ns, array (ninst, 2): when a CTA
        took the instance and when its solve finished."""
        a = np.zeros(2 * len(self.probs), np.int64)
        check(self.L.mb_batch_times(self.h, _p(a, C.c_int64), a.size), self.ctx.h, "times")
        return a.reshape(len(self.probs), 2)

    def latencies_ms(self):
        """Latency of each instance of the last run, all submitted with the launch: finish time minus
        the launch's earliest take (ms); and its solve time on its CTA (ms)."""
        t = self.times()
        return (t[:, 1] - t[:, 0].min()) / 1e6, (t[:, 1] - t[:, 0]) / 1e6

    def stats(self):
        a = np.zeros(8, np.int64)
        self.L.mb_batch_stats(self.h, _p(a, C.c_int64))
        return dict(input_bytes=int(a[0]), work_bytes=int(a[1]), factor_bytes=int(a[2]), launches=int(a[3]),
                    ninst=int(a[4]), output_bytes=int(a[5]))

    def __del__(self):
        if getattr(self, "h", None):
            self.L.mb_batch_destroy(self.h)
            self.h = None


_RESULT_DTYPE = np.dtype([(f, "<i4") for f in ("status", "niter", "nsolve", "nfactor_retry", "nfactor", "nfp32",
                                                 "nfallback", "reserved")] +
                         [(f, "<f8") for f in ("mu", "pres", "dres", "pobj", "dobj", "factor_flops")])
assert _RESULT_DTYPE.itemsize == C.sizeof(mb_result)
_STATUS = {s.value: s for s in IPMStatus}


def _batch_call(fn, probs, settings, grid, ctx, what):
    """Run a batched C entry point over `probs` with outputs in three contiguous host buffers (one
    allocation each; every problem's p, d and y are views into them) and the results read back
    through a structured view of the mb_result array."""
    probs = list(probs)
    if not probs:
        return []
    ctx = ctx or probs[0].ctx
    settings = settings or IPMSettings()
    cs = settings.to_c()
    k = len(probs)
    nm = np.array([p._nm() for p in probs], dtype=np.int64).reshape(k, 2)
    on = np.zeros(k + 1, np.int64); np.cumsum(nm[:, 0], out=on[1:])
    om = np.zeros(k + 1, np.int64); np.cumsum(nm[:, 1], out=om[1:])
    P, D, Y = np.zeros(max(int(on[-1]), 1)), np.zeros(max(int(on[-1]), 1)), np.zeros(max(int(om[-1]), 1))
    pa = (P.ctypes.data + 8 * on[:-1]).astype(np.uint64)
    da = (D.ctypes.data + 8 * on[:-1]).astype(np.uint64)
    ya = (Y.ctypes.data + 8 * om[:-1]).astype(np.uint64)
    pp = lambda a: C.cast(a.ctypes.data, C.POINTER(C.POINTER(C.c_double)))
    res = (mb_result * k)()
    arr = (C.c_void_p * k)(*[p.h.value for p in probs])
    check(fn(ctx.h, arr, k, C.byref(cs), grid, pp(pa), pp(da), pp(ya), res), ctx.h, what)
    r = np.frombuffer(res, dtype=_RESULT_DTYPE)
    col = {f: r[f].tolist() for f in _RESULT_DTYPE.names}
    on, om = on.tolist(), om.tolist()
    return [IPMResult(P[on[i]:on[i + 1]], D[on[i]:on[i + 1]], Y[om[i]:om[i + 1]], _STATUS[col["status"][i]],
                      col["niter"][i], col["nsolve"][i], IPMHistory(), col["mu"][i], col["pres"][i], col["dres"][i],
                      col["pobj"][i], col["dobj"][i], col["nfactor_retry"][i], col["nfactor"][i],
                      col["factor_flops"][i], col["nfp32"][i], col["nfallback"][i]) for i in range(k)]


def batch_solve(probs, settings: IPMSettings | None = None, grid: int = 0, ctx: Context | None = None):
    """solve over many problems (solver/ipm.jl:798-804) through mb_batch_solve: planning, upload,
    one persistent launch per chunk, results.  With grid = 0 and 1024 or more problems the library
    splits the call into chunks on their own streams, so host planning overlaps device work.  Each
    result's p, d and y are non-overlapping views into three arrays shared by the call's results
    (copy one to keep it apart from the others' memory)."""
    probs = list(probs)
    if not probs:
        return []
    ctx = ctx or probs[0].ctx
    return _batch_call(ctx.L.mb_batch_solve, probs, settings, grid, ctx, "batch solve")


def batch_solve_static(probs, settings: IPMSettings | None = None, grid: int = 0, ctx: Context | None = None):
    """batch_solve from the library's fixed device scratch (mb_batch_solve_static): no device
    allocation, for callers that hold a fixed HBM budget or cannot absorb cudaFree's device-wide
    synchronisation.  All problems together must fit in MB_STATIC_SCRATCH_BYTES (32 MiB), else
    MBError (MB_E_NOMEM).  Calls that overlap in time on one device race on the scratch."""
    probs = list(probs)
    if not probs:
        return []
    ctx = ctx or probs[0].ctx
    return _batch_call(ctx.L.mb_batch_solve_static, probs, settings, grid, ctx, "static batch solve")


# ---------------------------------------------------------------------------------------- serving
class Server:
    """Continuous-batching request loop (mb_server_*): one device arena of ``arena_bytes`` and a ring
    of ``capacity`` request slots feed a persistent solver grid; requests submitted while others are
    on the device are admitted as memory and slots free up.  Keep each problem alive until its
    result has been read."""

    QUEUED, PLANNED, RUNNING, DONE, FAILED = range(5)

    def __init__(self, settings: IPMSettings | None = None, arena_bytes: int = 8 << 30, capacity: int = 4096,
                 planners: int = 0, ctx: Context | None = None):
        self.ctx = ctx or Context.default()
        self.L = self.ctx.L
        self.settings = settings or IPMSettings()
        self._cs = self.settings.to_c()
        h = C.c_void_p()
        check(self.L.mb_server_create(self.ctx.h, C.byref(self._cs), int(arena_bytes), int(capacity), int(planners),
                                      C.byref(h)), self.ctx.h, "server create")
        self.h = h
        self._probs = {}

    def submit(self, prob: IPMProblem) -> int:
        t = C.c_int64()
        check(self.L.mb_server_submit(self.h, prob.h, C.byref(t)), self.ctx.h, "server submit")
        self._probs[t.value] = prob
        return t.value

    def state(self, ticket: int) -> int:
        s = C.c_int32()
        check(self.L.mb_server_poll(self.h, ticket, C.byref(s)), self.ctx.h, "server poll")
        return s.value

    def wait(self, ticket: int, timeout: float = 60.0) -> int:
        s = C.c_int32()
        check(self.L.mb_server_wait(self.h, ticket, float(timeout), C.byref(s)), self.ctx.h, "server wait")
        return s.value

    def result(self, ticket: int):
        """IPMResult of a finished ticket and its times: (result, [submitted, admitted, finished] in
        host seconds, (device start, device end) in ns).  Raises MBError for a failed request."""
        prob = self._probs[ticket]
        info = prob.info()
        p, d, y = np.zeros(info["n"]), np.zeros(info["n"]), np.zeros(info["m"])
        r = mb_result()
        t = np.zeros(5)
        rc = self.L.mb_server_result(self.h, ticket, _p(p, C.c_double), _p(d, C.c_double), _p(y, C.c_double),
                                     C.byref(r), _p(t, C.c_double))
        self._probs.pop(ticket, None)
        check(rc, self.ctx.h, "server result")
        res = IPMResult(p, d, y, IPMStatus(r.status), r.niter, r.nsolve, IPMHistory(), r.mu, r.pres, r.dres, r.pobj,
                        r.dobj, r.nfactor_retry, r.nfactor, r.factor_flops, r.nfp32, r.nfallback)
        return res, t[:3].tolist(), (int(t[3]), int(t[4]))

    def stats(self):
        a = np.zeros(8, np.int64)
        check(self.L.mb_server_stats(self.h, _p(a, C.c_int64)), self.ctx.h, "server stats")
        return dict(queued=int(a[0]), planned=int(a[1]), running=int(a[2]), completed=int(a[3]), failed=int(a[4]),
                    launches=int(a[5]), arena_used=int(a[6]), arena_bytes=int(a[7]))

    def close(self):
        if getattr(self, "h", None):
            self.L.mb_server_destroy(self.h)
            self.h = None

    def __del__(self):
        self.close()
