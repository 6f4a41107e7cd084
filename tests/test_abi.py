"""The C ABI library loads without a GPU and exports every function include/mumblebee_gpu.h
declares; the ctypes binding covers each of them.  No compute call is made."""
import ctypes
import os
import re

from mumblebee_b200 import _lib

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "mumblebee_gpu.h")


def declared():
    src = open(HEADER).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"^\s*(?:int|void)\s+(mb_\w+)\s*\(", src, flags=re.M)))


def test_header_declares_the_api():
    names = declared()
    for must in ("mb_ctx_create", "mb_problem_create", "mb_problem_create_csc", "mb_solver_create", "mb_solver_step",
                 "mb_solver_solve", "mb_solver_result", "mb_batch_solve", "mb_batch_solve_static"):
        assert must in names


def test_library_exports_every_declared_symbol():
    lib = ctypes.CDLL(_lib.load()._name)
    missing = [n for n in declared() if not hasattr(lib, n)]
    assert not missing, missing


def test_binding_covers_every_declared_symbol():
    missing = [n for n in declared() if n not in _lib.SIGNATURES]
    assert not missing, missing


def test_struct_layouts_match_header():
    # mb_settings: 8 int32, 10 doubles, then 2 int32; mb_result: 8 int32 then 6 doubles; history
    # rows: 17 doubles
    assert ctypes.sizeof(_lib.mb_settings) == 8 * 4 + 10 * 8 + 2 * 4
    assert ctypes.sizeof(_lib.mb_result) == 8 * 4 + 6 * 8
    assert ctypes.sizeof(_lib.mb_history_row) == 17 * 8
