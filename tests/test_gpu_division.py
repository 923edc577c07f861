"""The branch-free FP64 divisions and square roots of the stage kernels, bit
for bit against the IEEE operations on the GPU.

The FP64 stage kernels form the WENO weights with a Newton-Raphson reciprocal
and Markstein corrections (overheatingproblem_b200/csrc/eb2_fdiv.cuh) instead
of `/`, and fall back to `/` where an operand leaves the range in which that
is exact.  tests/pointcheck/eb2_divcheck.cu runs random operands (near-all-ones,
near-zero and few-bit significands, every exponent of the stated range) and
random WENO stencils (jumps, signed zeros, tiny, huge, infinite, NaN and
subnormal values) and random pairs of primitive states for the Roe average
through both and counts differing bits.  The stage-level
parity tests cover the same code on the reference's own data.
"""
from __future__ import annotations

import ctypes as C
import os
import shutil
import subprocess

import pytest

from conftest import ROOT

pytestmark = pytest.mark.gpu

HERE = os.path.join(ROOT, "tests", "pointcheck")
LIB = os.path.join(HERE, "libdivcheck.so")
CSRC = os.path.join(ROOT, "overheatingproblem_b200", "csrc")
NAMES = ["rcp_rn", "div_rn", "div by 6", "weno5_js_rn", "weno5_z_rn", "weno3_rn",
         "js fallback", "z fallback", "w3 fallback", "all-ones divisors", "roe_average_rn",
         "roe fallback", "div_rn_tiny", "sqrt_rn"]


@pytest.fixture(scope="module")
def dc():
    src = os.path.join(HERE, "eb2_divcheck.cu")
    deps = [src] + [os.path.join(CSRC, f) for f in ("eb2_fdiv.cuh", "eb2_point_fp64.cuh",
                                                     "eb2_common.cuh")]
    if not os.path.exists(LIB) or os.path.getmtime(LIB) < max(map(os.path.getmtime, deps)):
        nvcc = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
        subprocess.run([nvcc, "-O3", "-std=c++17", "-shared", "-Xcompiler", "-fPIC",
                        "-fmad=false", "-gencode", "arch=compute_100a,code=sm_100a", "-I", CSRC,
                        src, "-o", LIB], check=True, capture_output=True)
    lib = C.CDLL(LIB)
    lib.dc_run.argtypes = [C.c_ulonglong, C.c_int, C.POINTER(C.c_ulonglong)]
    lib.dc_run.restype = C.c_int
    return lib


def test_branch_free_divisions_match_ieee(dc):
    # 2^22 cases per launch; EB2_DIVCHECK_LAUNCHES=512 runs 2.1e9 (about 10 s)
    launches = int(os.environ.get("EB2_DIVCHECK_LAUNCHES", "32"))
    counts = (C.c_ulonglong * 14)()
    assert dc.dc_run(20261203, launches, counts) == 0
    got = dict(zip(NAMES, list(counts)))
    total = launches * (1 << 22)
    for name in NAMES[:6] + ["roe_average_rn", "div_rn_tiny", "sqrt_rn"]:
        assert got[name] == 0, got
    # the guard sends the stencils with infinite, NaN, subnormal or huge values
    # to `/`, and only those: most random stencils stay on the fast path
    for name in NAMES[6:9]:
        assert 0 < got[name] < total // 2, got
    # divisors with an all-ones significand (about one case in 2^18 here) are
    # reported by the guard rather than divided
    assert got["all-ones divisors"] > 0, got
    # Roe averages of states with densities or c^2 outside [2^-60, 2^400)
    assert 0 < got["roe fallback"] < total // 4, got
