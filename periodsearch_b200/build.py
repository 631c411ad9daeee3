"""Build the native library and executable in-tree (no JIT cache).

    python -m periodsearch_b200.build

produces
    periodsearch_b200/libps_b200.so      C ABI (include/period_search_b200.h)
    periodsearch_b200/period_search_b200 drop-in executable

Device code is compiled for sm_100a only; the FP64 kernels are built with
-fmad=false so that products and sums round exactly like the reference's
C source, and host code with -ffp-contract=off for the same reason.
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
OBJ = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "libps_b200.so")
EXE = os.path.join(HERE, "period_search_b200")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
HOST_FLAGS = ["-Xcompiler", "-O3,-fPIC,-ffp-contract=off", "-std=c++17"]

DEVICE_SOURCES = {"ps_fp64.cu": ["-fmad=false"], "ps_fast.cu": [], "ps_mixed.cu": [], "ps_noalloc.cu": [], "ps_peak.cu": [], "ps_adjoint.cu": []}
HOST_SOURCES = ["ps_host.cpp", "ps_api.cpp", "ps_batch.cpp"]


def _nvcc():
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", shutil.which("nvcc")):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def _run(cmd, verbose):
    if verbose:
        print(" ".join(cmd), flush=True)
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        sys.stderr.write(r.stdout + r.stderr)
        raise RuntimeError("build step failed: " + " ".join(cmd[:4]))
    return r.stdout + r.stderr


def _stale(target, deps):
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def build(verbose: bool = False, force: bool = False, ptxas_info: bool = False) -> str:
    nvcc = _nvcc()
    os.makedirs(OBJ, exist_ok=True)
    headers = [os.path.join(CSRC, h) for h in os.listdir(CSRC) if h.endswith((".hpp", ".h", ".cuh"))]
    headers.append(os.path.join(os.path.dirname(HERE), "include", "period_search_b200.h"))
    objs = []
    log = ""
    for src, extra in DEVICE_SOURCES.items():
        s = os.path.join(CSRC, src)
        o = os.path.join(OBJ, src + ".o")
        if force or _stale(o, [s] + headers):
            cmd = [nvcc, "-c", s, "-o", o, "-O3", "-lineinfo", *ARCH, *HOST_FLAGS, *extra]
            if ptxas_info:
                cmd += ["-Xptxas", "-v"]
            log += _run(cmd, verbose)
        objs.append(o)
    for src in HOST_SOURCES:
        s = os.path.join(CSRC, src)
        o = os.path.join(OBJ, src + ".o")
        if force or _stale(o, [s] + headers):
            log += _run([nvcc, "-c", s, "-o", o, *HOST_FLAGS], verbose)
        objs.append(o)
    if force or _stale(LIB, objs):
        _run([nvcc, "-shared", *ARCH, "-o", LIB, *objs, "-Xcompiler", "-fPIC"], verbose)
    app_src = os.path.join(CSRC, "ps_app.cpp")
    app_obj = os.path.join(OBJ, "ps_app.cpp.o")
    if force or _stale(app_obj, [app_src] + headers):
        _run([nvcc, "-c", app_src, "-o", app_obj, *HOST_FLAGS], verbose)
    if force or _stale(EXE, objs + [app_obj]):
        _run([nvcc, *ARCH, "-o", EXE, app_obj, *objs], verbose)
    if ptxas_info and verbose:
        print(log)
    return LIB


if __name__ == "__main__":
    build(verbose=True, force="--force" in sys.argv, ptxas_info="--ptxas" in sys.argv)
