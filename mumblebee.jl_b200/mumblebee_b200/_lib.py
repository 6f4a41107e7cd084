"""ctypes binding of libmbgpu.so (include/mumblebee_gpu.h).

Loading never falls back to anything: if the shared library is missing the import of the solver
API raises, and every GPU entry point reports CUDA errors as exceptions.
"""
from __future__ import annotations

import ctypes as C
import os

HERE = os.path.dirname(os.path.abspath(__file__))
PKG = os.path.dirname(HERE)
LIBPATH = os.path.join(PKG, "lib", "libmbgpu.so")

I32, I64, F64, F32 = C.c_int32, C.c_int64, C.c_double, C.c_float
PI64, PF64, PI32 = C.POINTER(I64), C.POINTER(F64), C.POINTER(I32)


class mb_settings(C.Structure):
    _fields_ = [("verbose", I32), ("max_iter", I32), ("scale_max_iter", I32), ("refine_max_iter", I32),
                ("newton_max_iter", I32), ("stable", I32), ("precision", I32), ("large", I32),
                ("step_frac", F64), ("feas_tol", F64), ("gap_tol", F64), ("near_factor", F64),
                ("stall_tol", F64), ("refine_stall_tol", F64), ("aug_tol", F64), ("infeas_abs", F64),
                ("infeas_rel", F64), ("coop_wait", F64), ("fp32_tiles", I32), ("reserved", I32)]


class mb_bsm(C.Structure):
    _fields_ = [("nout", I64), ("nvtx", I64), ("narc", I64), ("ncol", I64), ("nrow", I64), ("nbnz", I64),
                ("xsrc", PI64), ("xcol", PI64), ("xrow", PI64), ("xblk", PI64), ("tgt", PI64), ("val", PF64)]


class mb_csc(C.Structure):
    _fields_ = [("m", I64), ("n", I64), ("colptr", PI64), ("rowval", PI64), ("nzval", PF64)]


class mb_result(C.Structure):
    _fields_ = [("status", I32), ("niter", I32), ("nsolve", I32), ("nfactor_retry", I32),
                ("nfactor", I32), ("nfp32", I32), ("nfallback", I32), ("reserved", I32),
                ("mu", F64), ("pres", F64), ("dres", F64), ("pobj", F64), ("dobj", F64), ("factor_flops", F64)]


ROW_FIELDS = ["pres", "dres", "pobj", "dobj", "step", "piter", "ppass", "pstat", "citer", "cpass",
              "cstat", "dmin", "dmax", "rho", "delta", "mu", "chi"]


class mb_history_row(C.Structure):
    _fields_ = [(f, F64) for f in ROW_FIELDS]


# every symbol the header declares, with its signature
SIGNATURES = {
    "mb_version": (I32, [PI32, PI32]),
    "mb_settings_default": (None, [C.POINTER(mb_settings)]),
    "mb_ctx_create": (I32, [I32, C.POINTER(C.c_void_p)]),
    "mb_ctx_destroy": (I32, [C.c_void_p]),
    "mb_last_error": (I32, [C.c_void_p, C.c_char_p, I64]),
    "mb_problem_create": (I32, [C.c_void_p, C.POINTER(mb_bsm), C.POINTER(mb_bsm), PF64, PF64, F64, PI32, PF64,
                                PI64, PI64, C.POINTER(C.c_void_p)]),
    "mb_problem_create_csc": (I32, [C.c_void_p, C.POINTER(mb_csc), C.POINTER(mb_csc), PF64, PF64, F64, I64, PI32,
                                    PI64, PF64, F64, C.POINTER(C.c_void_p)]),
    "mb_problem_info": (I32, [C.c_void_p, PI64]),
    "mb_problem_export": (I32, [C.c_void_p, PI64, PI64, PI64, PI64, PI64, PF64, PI64, PI64, PI64, PF64, PF64, PF64,
                                PI32, PF64, PI64, PI64]),
    "mb_problem_destroy": (I32, [C.c_void_p]),
    "mb_problem_symbolic": (I32, [C.c_void_p, PI64, PI64, PI64, PI64, PI64, PI64, I64]),
    "mb_problem_footprint": (I32, [C.c_void_p, C.POINTER(mb_settings), PI64]),
    "mb_solver_create": (I32, [C.c_void_p, C.POINTER(mb_settings), PF64, PF64, PF64, C.POINTER(C.c_void_p)]),
    "mb_solver_step": (I32, [C.c_void_p, PI32]),
    "mb_solver_solve": (I32, [C.c_void_p, PI32]),
    "mb_solver_result": (I32, [C.c_void_p, PF64, PF64, PF64, C.POINTER(mb_result)]),
    "mb_solver_history": (I32, [C.c_void_p, C.POINTER(mb_history_row), I32, PI32]),
    "mb_solver_reinit": (I32, [C.c_void_p, PF64, PF64, PF64, PF64, PF64]),
    "mb_solver_timers": (I32, [C.c_void_p, PF64, I64]),
    "mb_solver_frule": (I32, [C.c_void_p, PF64, PF64, F64, PF64, PF64, PF64]),
    "mb_solver_rrule": (I32, [C.c_void_p, PF64, PF64, PF64, PF64, PF64, PF64]),
    "mb_solver_frule2": (I32, [C.c_void_p, PF64, PF64, F64, PF64, PF64, F64, C.POINTER(PF64)]),
    "mb_solver_destroy": (I32, [C.c_void_p]),
    "mb_batch_solve": (I32, [C.c_void_p, C.POINTER(C.c_void_p), I32, C.POINTER(mb_settings), I32,
                             C.POINTER(PF64), C.POINTER(PF64), C.POINTER(PF64), C.POINTER(mb_result)]),
    "mb_batch_prepare": (I32, [C.c_void_p, C.POINTER(C.c_void_p), I32, C.POINTER(mb_settings),
                               C.POINTER(C.c_void_p)]),
    "mb_batch_run": (I32, [C.c_void_p, I32, C.POINTER(F32)]),
    "mb_batch_fetch": (I32, [C.c_void_p, C.POINTER(PF64), C.POINTER(PF64), C.POINTER(PF64), C.POINTER(mb_result)]),
    "mb_batch_stats": (I32, [C.c_void_p, PI64]),
    "mb_batch_timers": (I32, [C.c_void_p, PF64, I64]),
    "mb_batch_times": (I32, [C.c_void_p, PI64, I64]),
    "mb_batch_destroy": (I32, [C.c_void_p]),
    "mb_server_create": (I32, [C.c_void_p, C.POINTER(mb_settings), I64, I32, I32, C.POINTER(C.c_void_p)]),
    "mb_server_submit": (I32, [C.c_void_p, C.c_void_p, PI64]),
    "mb_server_poll": (I32, [C.c_void_p, I64, PI32]),
    "mb_server_wait": (I32, [C.c_void_p, I64, C.c_double, PI32]),
    "mb_server_result": (I32, [C.c_void_p, I64, PF64, PF64, PF64, C.POINTER(mb_result), PF64]),
    "mb_server_stats": (I32, [C.c_void_p, PI64]),
    "mb_server_destroy": (I32, [C.c_void_p]),
    "mb_matrix_create": (I32, [C.c_void_p, C.POINTER(mb_bsm), C.POINTER(C.c_void_p)]),
    "mb_matrix_destroy": (I32, [C.c_void_p]),
    "mb_extmul": (I32, [C.c_void_p, I32, PF64, F64, F64, PF64, PF64, PF64]),
    "mb_twomul": (I32, [C.c_void_p, I32, PF64, F64, F64, PF64, PF64, PF64, PF64]),
    "mb_batch_solve_static": (I32, [C.c_void_p, C.POINTER(C.c_void_p), I32, C.POINTER(mb_settings), I32,
                                    C.POINTER(PF64), C.POINTER(PF64), C.POINTER(PF64), C.POINTER(mb_result)]),
}

MB_STATIC_SCRATCH_BYTES = 32 << 20   # include/mumblebee_gpu.h

_lib = None


def load(path: str | None = None):
    """Load libmbgpu.so (built in-tree by mumblebee.jl_b200/build.py).  Raises if it is absent."""
    global _lib
    if _lib is not None:
        return _lib
    p = path or LIBPATH
    if not os.path.exists(p):
        raise RuntimeError(f"libmbgpu.so not found at {p}; build it with `python mumblebee.jl_b200/build.py`")
    L = C.CDLL(p)
    for name, (res, args) in SIGNATURES.items():
        fn = getattr(L, name)
        fn.restype = res
        fn.argtypes = args
    _lib = L
    return L


class MBError(RuntimeError):
    pass


def check(rc: int, ctx=None, what: str = ""):
    if rc != 0:
        msg = ""
        if ctx:
            buf = C.create_string_buffer(1024)
            load().mb_last_error(ctx, buf, 1024)
            msg = buf.value.decode(errors="replace")
        raise MBError(f"{what} failed with code {rc}: {msg}")
