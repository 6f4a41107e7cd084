"""Build libmbgpu.so in-tree (sm_100a only).

    python mumblebee.jl_b200/build.py

Compiles the CUDA solver and the C++ host runtime with nvcc and links a shared library with a
static CUDA runtime, so the artefact needs only the driver at load time.
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
LIBDIR = os.path.join(HERE, "lib")
LIB = os.path.join(LIBDIR, "libmbgpu.so")
NVCC = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
COMMON = ["-O3", "-std=c++17", "-Xcompiler", "-fPIC", "-lineinfo"]

SOURCES_CU = ["mb_solver.cu", "mb_solver_tc.cu", "mb_comp.cu"]
SOURCES_CPP = ["mb_host.cpp"]
# headers each source includes (a change rebuilds only the sources that use it)
_SOLVER_DEPS = ["mb_internal.h", "mb_device.cuh", "mb_cones.cuh", "mb_tdc.cuh", "mb_sdp.cuh"]
DEPS = {
    "mb_solver.cu": _SOLVER_DEPS,
    "mb_solver_tc.cu": _SOLVER_DEPS + ["mb_solver.cu"],   # the tensor-core build of the same source
    "mb_comp.cu": ["mb_internal.h"],
    "mb_host.cpp": ["mb_internal.h", "mb_symbolic.hpp"],
}
HEADERS = sorted({h for v in DEPS.values() for h in v})


def _newer(target, deps):
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def build(verbose: bool = False, force: bool = False) -> str:
    api = os.path.join(HERE, "..", "include", "mumblebee_gpu.h")
    sources = [os.path.join(CSRC, f) for f in SOURCES_CU + SOURCES_CPP + HEADERS] + [api, os.path.abspath(__file__)]
    # a copy of the tree that carries the built library but not the intermediate objects: the
    # library is up to date when it is newer than every source (where the objects exist, each is
    # checked against its own sources below, which also catches a source edited during a build)
    objdir = os.path.join(HERE, "_build")
    if not force and not os.path.isdir(objdir) and not _newer(LIB, sources):
        return LIB
    os.makedirs(LIBDIR, exist_ok=True)
    os.makedirs(objdir, exist_ok=True)
    objs, cmds = [], []
    for src in SOURCES_CU + SOURCES_CPP:
        s = os.path.join(CSRC, src)
        o = os.path.join(objdir, src + ".o")
        objs.append(o)
        hdrs = [os.path.join(CSRC, h) for h in DEPS[src]] + [api]
        if force or _newer(o, [s] + hdrs):
            cmd = [NVCC] + ARCH + COMMON + ["-c", s, "-o", o]
            if src.endswith(".cu"):
                cmd += ["-Xptxas", "-v"] if verbose else []
            if verbose:
                print(" ".join(cmd))
            cmds.append(cmd)
    # the translation units compile in parallel (the two solver builds take minutes each)
    procs = [subprocess.Popen(c) for c in cmds]
    rcs = [p.wait() for p in procs]
    for c, rc in zip(cmds, rcs):
        if rc:
            raise subprocess.CalledProcessError(rc, c)
    if force or _newer(LIB, objs):
        cmd = [NVCC] + ARCH + ["-shared", "-cudart", "static", "-o", LIB] + objs
        if verbose:
            print(" ".join(cmd))
        subprocess.run(cmd, check=True)
    return LIB


if __name__ == "__main__":
    build(verbose="-v" in sys.argv, force="-f" in sys.argv)
    print(LIB)
