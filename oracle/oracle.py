"""ORACLE — test infrastructure only.

ctypes binding of the FP64 CPU restatement (oracle/ipm_oracle.cpp) of Mumblebee.jl's IPM hot
path.  Only tests/, the smoke check and bench.py's CPU-baseline leg import this module.

The reference has no test suite, fixtures or golden vectors (and Julia is absent), so parity is
pinned against documented mathematics only — see the header of ipm_oracle.cpp.
"""
from __future__ import annotations

import ctypes as C
import glob
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "_build", "liboracle.so")

STATUS = ["CONTINUE", "OPTIMAL", "NEAR_OPTIMAL", "STALLED", "NUMERICAL_FAILURE", "ITERATION_LIMIT",
          "PRIMAL_INFEASIBLE", "DUAL_INFEASIBLE", "ILL_POSED", "NEAR_PRIMAL_INFEASIBLE",
          "NEAR_DUAL_INFEASIBLE", "NEAR_ILL_POSED"]
ROW_FIELDS = ["pres", "dres", "pobj", "dobj", "step", "piter", "ppass", "pstat", "citer", "cpass",
              "cstat", "dmin", "dmax", "rho", "delta", "mu", "chi"]


class Settings(C.Structure):
    """IPMSettings (settings/ipm.jl:1-18) plus the precision knob; layout shared with mb_settings."""
    _fields_ = [("verbose", C.c_int32), ("max_iter", C.c_int32), ("scale_max_iter", C.c_int32),
                ("refine_max_iter", C.c_int32), ("newton_max_iter", C.c_int32), ("stable", C.c_int32),
                ("precision", C.c_int32), ("large", C.c_int32),
                ("step_frac", C.c_double), ("feas_tol", C.c_double), ("gap_tol", C.c_double),
                ("near_factor", C.c_double), ("stall_tol", C.c_double), ("refine_stall_tol", C.c_double),
                ("aug_tol", C.c_double), ("infeas_abs", C.c_double), ("infeas_rel", C.c_double)]


def default_settings(**kw) -> Settings:
    s = Settings(verbose=0, max_iter=100, scale_max_iter=10, refine_max_iter=10, newton_max_iter=100,
                 stable=0, precision=0, large=0, step_frac=0.99, feas_tol=1e-8, gap_tol=1e-8,
                 near_factor=1000.0, stall_tol=1e-3, refine_stall_tol=0.5, aug_tol=1e-7,
                 infeas_abs=1e-8, infeas_rel=1e-8)
    for k, v in kw.items():
        setattr(s, k, v)
    return s


class BSM(C.Structure):
    _fields_ = [("nout", C.c_int64), ("nvtx", C.c_int64), ("narc", C.c_int64), ("ncol", C.c_int64),
                ("nrow", C.c_int64), ("nbnz", C.c_int64),
                ("xsrc", C.POINTER(C.c_int64)), ("xcol", C.POINTER(C.c_int64)), ("xrow", C.POINTER(C.c_int64)),
                ("xblk", C.POINTER(C.c_int64)), ("tgt", C.POINTER(C.c_int64)), ("val", C.POINTER(C.c_double))]


class Row(C.Structure):
    _fields_ = [(f, C.c_double) for f in ROW_FIELDS]


def _p64(a):
    return a.ctypes.data_as(C.POINTER(C.c_int64))


def _pd(a):
    return None if a is None else a.ctypes.data_as(C.POINTER(C.c_double))


def bsm_struct(d, keep):
    arrs = {k: np.ascontiguousarray(d[k], dtype=np.int64) for k in ("xsrc", "xcol", "xrow", "xblk", "tgt")}
    arrs["val"] = np.ascontiguousarray(d["val"], dtype=np.float64)
    keep.extend(arrs.values())
    return BSM(d["nout"], d["nvtx"], d["narc"], d["ncol"], d["nrow"], d["nbnz"],
               _p64(arrs["xsrc"]), _p64(arrs["xcol"]), _p64(arrs["xrow"]), _p64(arrs["xblk"]),
               _p64(arrs["tgt"]), _pd(arrs["val"]))


_lib = None


def build():
    subprocess.run(["make", "-s", "-C", HERE], check=True)


def find_openblas():
    import scipy
    d = os.path.join(os.path.dirname(os.path.dirname(scipy.__file__)), "scipy.libs")
    c = sorted(glob.glob(os.path.join(d, "libscipy_openblas*.so")))
    return c[0] if c else None


def lib(threads: int = 1):
    global _lib
    if _lib is None:
        if not os.path.exists(LIB):
            build()
        L = C.CDLL(LIB)
        L.oracle_create.restype = C.c_void_p
        L.oracle_create.argtypes = [C.POINTER(BSM), C.POINTER(BSM), C.POINTER(C.c_double), C.POINTER(C.c_double),
                                    C.c_double, C.POINTER(C.c_int32), C.POINTER(C.c_double), C.POINTER(C.c_int64),
                                    C.POINTER(C.c_int64), C.POINTER(C.c_int64), C.POINTER(Settings),
                                    C.POINTER(C.c_double), C.POINTER(C.c_double), C.POINTER(C.c_double)]
        L.oracle_step.argtypes = [C.c_void_p]
        L.oracle_reinit.argtypes = [C.c_void_p] + [C.POINTER(C.c_double)] * 5
        L.oracle_frule.argtypes = [C.c_void_p, C.POINTER(C.c_double), C.POINTER(C.c_double), C.c_double] + \
            [C.POINTER(C.c_double)] * 3
        L.oracle_rrule.argtypes = [C.c_void_p] + [C.POINTER(C.c_double)] * 6
        L.oracle_frule2.argtypes = [C.c_void_p, C.POINTER(C.c_double), C.POINTER(C.c_double), C.c_double,
                                    C.POINTER(C.c_double), C.POINTER(C.c_double), C.c_double,
                                    C.POINTER(C.POINTER(C.c_double))]
        L.oracle_solve.argtypes = [C.c_void_p]
        L.oracle_result.argtypes = [C.c_void_p, C.c_int, C.POINTER(C.c_double), C.POINTER(C.c_double),
                                    C.POINTER(C.c_double), C.POINTER(C.c_double), C.POINTER(C.c_int32),
                                    C.POINTER(C.c_int32)]
        L.oracle_history.argtypes = [C.c_void_p, C.POINTER(Row), C.c_int32]
        L.oracle_timers.argtypes = [C.c_void_p, C.POINTER(C.c_double)]
        L.oracle_symbolic.argtypes = [C.c_void_p] + [C.POINTER(C.c_int64)] * 5 + [C.c_int64]
        L.oracle_nfactor_retry.argtypes = [C.c_void_p]
        L.oracle_nfactor_retry.restype = C.c_int64
        L.oracle_destroy.argtypes = [C.c_void_p]
        for nm in ("oracle_nfallback", "oracle_nfp32"):
            getattr(L, nm).argtypes = [C.c_void_p]
            getattr(L, nm).restype = C.c_int64
        PD = C.POINTER(C.c_double)
        L.oracle_sdp_probe.argtypes = [C.c_int64, PD, PD, PD, PD, C.c_double, PD, PD, PD, PD, PD, PD, PD]
        L.oracle_sdp_probe.restype = C.c_int
        L.oracle_sdp_eig.argtypes = [C.c_int, PD, C.c_double, PD, PD, PD, PD]
        L.oracle_sdp_eig.restype = C.c_int
        L.oracle_twomul.argtypes = [C.POINTER(BSM), C.c_int, PD, C.c_double, C.c_double, PD, PD, PD, PD]
        L.oracle_set_blas.argtypes = [C.c_char_p, C.c_int]
        L.oracle_set_threads.argtypes = [C.c_int]
        path = find_openblas()
        if path:
            L.oracle_set_blas(path.encode(), threads)
        _lib = L
    if threads:
        _lib.oracle_set_threads(threads)
    return _lib


class OracleSolver:
    """IPMSolver on the CPU: init / step! / solve! / result (solver/ipm.jl, solver/solver.jl)."""

    def __init__(self, prob, settings: Settings | None = None, vperm=None, p0=None, d0=None, y0=None,
                 threads: int = 1):
        self.L = lib(threads)
        self.prob = prob
        self.settings = settings or default_settings()
        keep = []
        self._Q = bsm_struct(prob["Q"], keep)
        self._B = bsm_struct(prob["B"], keep)
        f = np.ascontiguousarray(prob["f"], dtype=np.float64)
        g = np.ascontiguousarray(prob["g"], dtype=np.float64)
        kind = np.ascontiguousarray(prob["kind"], dtype=np.int32)
        par = np.ascontiguousarray(prob["param"], dtype=np.float64)
        P1 = np.ascontiguousarray(prob["P1"], dtype=np.int64)
        P2 = np.ascontiguousarray(prob["P2"], dtype=np.int64)
        vp = None if vperm is None else np.ascontiguousarray(vperm, dtype=np.int64)
        arr = [None if a is None else np.ascontiguousarray(a, dtype=np.float64) for a in (p0, d0, y0)]
        keep += [f, g, kind, par, P1, P2, vp] + arr
        self._keep = keep
        self.n = prob["B"]["ncol"]
        self.m = prob["B"]["nrow"]
        self.h = self.L.oracle_create(C.byref(self._Q), C.byref(self._B), _pd(f), _pd(g), float(prob["mu"]),
                                      kind.ctypes.data_as(C.POINTER(C.c_int32)), _pd(par), _p64(P1), _p64(P2),
                                      None if vp is None else _p64(vp), C.byref(self.settings),
                                      _pd(arr[0]), _pd(arr[1]), _pd(arr[2]))
        self.status = 0

    def step(self) -> int:
        self.status = self.L.oracle_step(self.h)
        return self.status

    def frule(self, df=None, dg=None, dmu=0.0):
        """frule!(Δp, Δy, Δd, s, Δf, Δg, Δμ): tangents of (p, y, d) for seeds on (f, g, μ); user order."""
        a = [None if x is None else np.ascontiguousarray(x, dtype=np.float64) for x in (df, dg)]
        dp, dd, dy = np.zeros(self.n), np.zeros(self.n), np.zeros(self.m)
        rc = self.L.oracle_frule(self.h, _pd(a[0]), _pd(a[1]), float(dmu), _pd(dp), _pd(dy), _pd(dd))
        if rc:
            raise RuntimeError("frule!: the factorization failed")
        return dp, dy, dd

    def frule2(self, df1=None, dg1=None, dmu1=0.0, df2=None, dg2=None, dmu2=0.0):
        """frule2!: first-order tangents for two seed sets and the second-order tangent, as nine
        vectors (Δp1, Δy1, Δd1, Δp2, Δy2, Δd2, Δp12, Δy12, Δd12); user order."""
        a = [None if x is None else np.ascontiguousarray(x, dtype=np.float64) for x in (df1, dg1, df2, dg2)]
        outs = [np.zeros(self.m if k % 3 == 1 else self.n) for k in range(9)]
        arr = (C.POINTER(C.c_double) * 9)(*[_pd(x) for x in outs])
        rc = self.L.oracle_frule2(self.h, _pd(a[0]), _pd(a[1]), float(dmu1), _pd(a[2]), _pd(a[3]), float(dmu2), arr)
        if rc:
            raise RuntimeError("frule2!: the factorization failed")
        return tuple(outs)

    def rrule(self, dp=None, dy=None, dd=None):
        """rrule!(Δf, Δg, s, Δp, Δy, Δd): cotangents of (f, g) and μ for seeds on (p, y, d)."""
        a = [None if x is None else np.ascontiguousarray(x, dtype=np.float64) for x in (dp, dy, dd)]
        df, dg, dmu = np.zeros(self.n), np.zeros(self.m), C.c_double()
        rc = self.L.oracle_rrule(self.h, _pd(a[0]), _pd(a[1]), _pd(a[2]), _pd(df), _pd(dg), C.byref(dmu))
        if rc:
            raise RuntimeError("rrule!: the factorization failed")
        return df, dg, dmu.value

    def reinit(self, p0=None, d0=None, y0=None, f=None, g=None):
        """reinit!(s; p0, d0, y0, f, g), every vector in user order."""
        arr = [None if a is None else np.ascontiguousarray(a, dtype=np.float64) for a in (p0, d0, y0, f, g)]
        self._keep_reinit = arr
        self.L.oracle_reinit(self.h, *[_pd(a) for a in arr])
        self.status = 0
        return self

    def solve(self):
        self.status = self.L.oracle_solve(self.h)
        return self.result()

    def result(self):
        p = np.zeros(self.n); d = np.zeros(self.n); y = np.zeros(self.m)
        sc = np.zeros(5); ni = C.c_int32(); ns = C.c_int32()
        self.L.oracle_result(self.h, self.status, _pd(p), _pd(d), _pd(y), _pd(sc), C.byref(ni), C.byref(ns))
        return dict(p=p, d=d, y=y, status=STATUS[self.status], status_code=self.status, niter=ni.value,
                    nsolve=ns.value, mu=sc[0], pres=sc[1], dres=sc[2], pobj=sc[3], dobj=sc[4],
                    history=self.history(), timers=self.timers())

    def history(self):
        cap = 256
        rows = (Row * cap)()
        n = self.L.oracle_history(self.h, rows, cap)
        return [{f: getattr(rows[i], f) for f in ROW_FIELDS} for i in range(min(n, cap))]

    def timers(self):
        t = np.zeros(6)
        self.L.oracle_timers(self.h, _pd(t))
        return dict(zip(["scale", "initkkt", "predictor", "corrector", "maxsteps", "exact"], t.tolist()))

    def symbolic(self):
        cap = 1 << 20
        a = [np.zeros(cap, dtype=np.int64) for _ in range(4)]
        nf = C.c_int64()
        self.L.oracle_symbolic(self.h, C.byref(nf), *[_p64(x) for x in a], cap)
        k = nf.value
        return dict(nfront=k, res0=a[0][:k], nres=a[1][:k], nsep=a[2][:k], parent=a[3][:k])

    def mixed_counts(self):
        return self.L.oracle_nfp32(self.h), self.L.oracle_nfallback(self.h)

    def nfactor_retry(self):
        return self.L.oracle_nfactor_retry(self.h)

    def __del__(self):
        if getattr(self, "h", None):
            self.L.oracle_destroy(self.h)
            self.h = None


def solve(prob, settings=None, vperm=None, **kw):
    s = OracleSolver(prob, settings, vperm, **kw)
    return s.solve()


def twomul(A, trans, b, alpha, beta, c, pair):
    """extmul! (pair False) or twomul! (pair True) on the host: returns (c, cc or None, s, cs); c is
    a copy of the input c, updated."""
    keep = []
    Ab = bsm_struct(A, keep)
    nout = A["ncol"] if trans else A["nrow"]
    b = np.ascontiguousarray(b, dtype=np.float64)
    c = np.array(c, dtype=np.float64, copy=True)
    cc = np.zeros(nout) if pair else None
    s, cs = np.zeros(nout), np.zeros(nout)
    lib(0).oracle_twomul(C.byref(Ab), int(trans), _pd(b), float(alpha), float(beta), _pd(c), _pd(cc), _pd(s), _pd(cs))
    return c, cc, s, cs


def sdp_probe(p, d, Dp, Dd, sm):
    """Semidefinite-cone primitives at svec points (p, d): the added Hessian block H, the cache
    [R | S | s], ⟨p*, d*⟩, corrector along (Δp, Δd), zero corrector, steps (τp, τd), shadow p⁻¹."""
    n = len(p)
    k = int((np.sqrt(1 + 8 * n) - 1) // 2)
    arr = lambda x: np.ascontiguousarray(x, dtype=np.float64)
    p, d, Dp, Dd = arr(p), arr(d), arr(Dp), arr(Dd)
    H = np.zeros(n * n); cache = np.zeros(2 * k * k + k); spsd = np.zeros(1)
    r = np.zeros(n); r0 = np.zeros(n); steps = np.zeros(2); shp = np.zeros(n)
    flags = lib().oracle_sdp_probe(n, _pd(p), _pd(d), _pd(Dp), _pd(Dd), sm, _pd(H), _pd(cache), _pd(spsd), _pd(r),
                                   _pd(r0), _pd(steps), _pd(shp))
    R = cache[:k * k].reshape(k, k, order="F"); S = cache[k * k:2 * k * k].reshape(k, k, order="F")
    return dict(ok=bool(flags & 1), shadow_ok=bool(flags & 2), H=H.reshape(n, n, order="F"), R=R, S=S,
                s=cache[2 * k * k:], spsd=spsd[0], corr=r, corr0=r0, tp=steps[0], td=steps[1], shadow=shp)


def sdp_eig(M, lmax, A):
    """eigmin of M by the Laguerre/Sturm path (capped at lmax) and the analytic path (d ≤ 3), and the
    one-sided Jacobi SVD of A (U, s, converged)."""
    d = M.shape[0]
    Mf = np.asfortranarray(M, dtype=np.float64).ravel(order="F")
    Af = np.asfortranarray(A, dtype=np.float64).ravel(order="F")
    out = np.zeros(2); U = np.zeros(d * d); sv = np.zeros(d)
    ok = lib().oracle_sdp_eig(d, _pd(Mf), lmax, _pd(Af), _pd(out), _pd(U), _pd(sv))
    return out[0], out[1], U.reshape(d, d, order="F"), sv, bool(ok)
