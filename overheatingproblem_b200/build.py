"""Build libeuler_b200.so in-tree for sm_100a.

    python -m overheatingproblem_b200.build [--force]

Each CUDA translation unit is compiled by nvcc for ``sm_100a`` only; the
bit-parity units (the FP64 stage kernels, the boundary/reduction/granular
kernels and the host runtime) get ``-fmad=false`` so that no multiply-add is
contracted, the mixed-precision unit keeps FMA contraction.  The C control-file
reader is compiled by gcc.  Objects go to ``_build/`` (git-ignored); the shared
library lands next to this file so that it travels with the source tree.
"""
from __future__ import annotations

import concurrent.futures as cf
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
BUILD = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "libeuler_b200.so")
INCLUDE = os.path.join(os.path.dirname(HERE), "include")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVFLAGS = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC", "-Xptxas", "-v",
           "--expt-relaxed-constexpr", "-I", CSRC, "-I", INCLUDE]

# (source, exact): exact units are compiled without FMA contraction.
CUDA_SOURCES = [
    ("eb2_stage_fp64_w5.cu", True),
    ("eb2_stage_fp64_tvd.cu", True),
    ("eb2_stage_fp64_g1.cu", True),
    ("eb2_stage_fp64_w3.cu", True),
    ("eb2_stage_fp64_hc.cu", True),
    ("eb2_stage.cu", True),
    ("eb2_aux.cu", True),
    ("eb2_api.cu", True),
    ("eb2_cases.cu", True),
    ("eb2_noalloc.cu", True),
    ("eb2_batch_fp64.cu", True),
    ("eb2_server.cu", True),
    ("eb2_stage_mixed.cu", False),
    ("eb2_batch_mixed.cu", False),
    ("eb2_batch_mixed_s8.cu", False),
    ("eb2_batch_mixed_s32.cu", False),
]
C_SOURCES = ["eb2_control.c", "rpf_runtime.c"]
HEADERS = ["eb2_common.cuh", "eb2_kernels.h", "eb2_fdiv.cuh", "eb2_point_fp64.cuh", "eb2_stage_fp64.cuh",
           "eb2_point_mixed.cuh", "eb2_stage_mixed.cuh", "eb2_loop.cuh", "eb2_batch.cuh",
           "eb2_batch_mixed.cuh"]


def _nvcc() -> str:
    for cand in (shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found: libeuler_b200 needs the CUDA toolkit to build")


def _newest_header() -> float:
    t = 0.0
    for h in HEADERS:
        p = os.path.join(CSRC, h)
        if os.path.exists(p):
            t = max(t, os.path.getmtime(p))
    for h in ("euler_b200.h", os.path.join("rp_fvm", "rpf_runtime.h")):
        t = max(t, os.path.getmtime(os.path.join(INCLUDE, h)))
    return t


def _stale(src: str, obj: str, hdr_time: float) -> bool:
    if not os.path.exists(obj):
        return True
    t = os.path.getmtime(obj)
    return t < os.path.getmtime(src) or t < hdr_time


def _compile_cuda(src: str, exact: bool, log: list) -> str:
    obj = os.path.join(BUILD, os.path.basename(src) + ".o")
    cmd = [_nvcc()] + ARCH + NVFLAGS + (["-fmad=false"] if exact else []) + ["-c", src, "-o", obj]
    res = subprocess.run(cmd, capture_output=True, text=True)
    log.append((src, res.stdout + res.stderr))
    if res.returncode:
        raise RuntimeError(f"nvcc failed for {src}:\n{res.stderr[-4000:]}")
    return obj


def _compile_c(src: str, log: list) -> str:
    obj = os.path.join(BUILD, os.path.basename(src) + ".o")
    cmd = ["gcc", "-O2", "-fPIC", "-std=c11", "-Wall", "-I", INCLUDE, "-c", src, "-o", obj]
    res = subprocess.run(cmd, capture_output=True, text=True)
    log.append((src, res.stdout + res.stderr))
    if res.returncode:
        raise RuntimeError(f"gcc failed for {src}:\n{res.stderr[-4000:]}")
    return obj


def build(force: bool = False, verbose: bool = False) -> str:
    os.makedirs(BUILD, exist_ok=True)
    hdr = _newest_header()
    log: list = []
    jobs = []
    objs = []
    with cf.ThreadPoolExecutor(max_workers=max(2, (os.cpu_count() or 4))) as pool:
        for name, exact in CUDA_SOURCES:
            src = os.path.join(CSRC, name)
            obj = os.path.join(BUILD, name + ".o")
            objs.append(obj)
            if force or _stale(src, obj, hdr):
                jobs.append(pool.submit(_compile_cuda, src, exact, log))
        for name in C_SOURCES:
            src = os.path.join(CSRC, name)
            obj = os.path.join(BUILD, name + ".o")
            objs.append(obj)
            if force or _stale(src, obj, hdr):
                jobs.append(pool.submit(_compile_c, src, log))
        for j in jobs:
            j.result()
    if force or jobs or not os.path.exists(LIB):
        cmd = [_nvcc()] + ARCH + ["-shared", "-o", LIB] + objs + ["-lcudart"]
        res = subprocess.run(cmd, capture_output=True, text=True)
        if res.returncode:
            raise RuntimeError(f"link failed:\n{res.stderr[-4000:]}")
    if verbose:
        for src, out in log:
            print(f"== {os.path.basename(src)}\n{out}")
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose="-v" in sys.argv)
    print(LIB)
