"""Compile the CUDA library in place: multiblockmomentsfv_b200/lib/libmbm_b200.so.

sm_100a only.  -fmad=false keeps every multiply and add of the forward path
separately rounded (the bitwise mode depends on it); double division and sqrt are
IEEE by default.  The adjoint kernels (derivatives, not restatements of the
reference's arithmetic) and the fast-arithmetic stage kernel are compiled with
fused multiply-adds.
"""
from __future__ import annotations

import os
import subprocess
import sys

PKG = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(PKG, "csrc")
LIBDIR = os.path.join(PKG, "lib")
LIB = os.path.join(LIBDIR, "libmbm_b200.so")

SOURCES = ["mbm_host.cu", "mbm_kernels.cu", "mbm_stage_fast.cu", "mbm_noalloc.cu", "mbm_adjoint.cu"]
HEADERS = ["mbm_internal.h", "mbm_math.cuh", "mbm_stage.cuh", "mbm_adjoint_math.cuh", "mbm_newton.cuh"]

NVCC_FLAGS = [
    "-gencode", "arch=compute_100a,code=sm_100a",
    "-lineinfo", "-O3", "-std=c++17",
    "-Xcompiler", "-fPIC",
]
FMAD = {"mbm_adjoint.cu": "true", "mbm_stage_fast.cu": "true"}   # every other source: -fmad=false


def nvcc() -> str:
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", "nvcc"):
        if cand and (os.path.isabs(cand) and os.path.exists(cand) or not os.path.isabs(cand)):
            return cand
    return "nvcc"


def _stale() -> bool:
    if not os.path.exists(LIB):
        return True
    t = os.path.getmtime(LIB)
    deps = [os.path.join(CSRC, f) for f in SOURCES + HEADERS]
    deps.append(os.path.join(os.path.dirname(PKG), "include", "mbm_b200.h"))
    return any(os.path.getmtime(p) > t for p in deps if os.path.exists(p))


def build(force: bool = False, verbose: bool = False, ptxas_info: bool = False) -> str:
    if not force and not _stale():
        return LIB
    os.makedirs(LIBDIR, exist_ok=True)
    objdir = os.path.join(LIBDIR, "obj")
    os.makedirs(objdir, exist_ok=True)
    procs, objs = [], []
    for f in SOURCES:                     # one object per source, compiled in parallel
        obj = os.path.join(objdir, f.replace(".cu", ".o"))
        cmd = [nvcc(), *NVCC_FLAGS, "-fmad=" + FMAD.get(f, "false")]
        if ptxas_info:
            cmd += ["-Xptxas", "-v"]
        cmd += ["-c", os.path.join(CSRC, f), "-o", obj]
        procs.append((f, subprocess.Popen(cmd, stdout=subprocess.PIPE, stderr=subprocess.STDOUT, text=True)))
        objs.append(obj)
    failed = []
    for f, p in procs:
        out = p.communicate()[0]
        if verbose or p.returncode != 0:
            sys.stderr.write(out)
        if p.returncode != 0:
            failed.append(f)
    if failed:
        raise RuntimeError("nvcc failed on " + ", ".join(failed))
    tmp = LIB + ".tmp"
    r = subprocess.run([nvcc(), "-gencode", "arch=compute_100a,code=sm_100a", "-shared", "-o", tmp, *objs],
                       capture_output=True, text=True)
    if verbose or r.returncode != 0:
        sys.stderr.write(r.stdout + r.stderr)
    if r.returncode != 0:
        raise RuntimeError("nvcc failed linking libmbm_b200.so")
    os.replace(tmp, LIB)
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose=True, ptxas_info="-v" in sys.argv)
    print(LIB)
