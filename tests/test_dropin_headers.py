"""The drop-in header set include/rp_fvm/ (CPU only): it declares the
reference's entry points, the library exports every runtime function it
forwards to, the reference's own caller compiles against it unchanged, and
without a GPU the built caller stops with an error instead of computing."""
from __future__ import annotations

import os
import re
import subprocess

import pytest

from conftest import HAVE_GPU, ROOT
from oracle.bind import REFERENCE_TREE

SHIM = os.path.join(ROOT, "include", "rp_fvm")
REF_CALLER = os.path.join(REFERENCE_TREE, "src", "RP_FVM.c")

# (header, entry point) pairs of the reference's operator API the set carries
ENTRY_POINTS = [
    ("mesh.h", "Mesh_2D"), ("initialize.h", "Init_Euler_2D"), ("initialize.h", "Init_Precision"),
    ("initialize.h", "Con_to_Pri_2D"), ("initialize.h", "getTestCaseShortName"),
    ("Boundary_Condition.h", "Boundary_Conditions"), ("function.h", "Get_Delta_T_2D"),
    ("function.h", "Precision_Get_Delta_T_2D"), ("Characteriz.h", "Compute_Eigen_2DX"),
    ("Characteriz.h", "Compute_Eigen_2DY"), ("Reconstruction.h", "WENO5_Reconstruction"),
    ("Reconstruction.h", "TVD_Reconstruction"), ("scheme.h", "HLL_Flux"),
    ("scheme.h", "HLLC_Flux"), ("scheme.h", "Roe_Flux"), ("scheme.h", "LLF_Flux"),
    ("scheme.h", "Space_Discrete_Item"), ("CFD_convection.h", "Flux_Reconstruction_RP"),
    ("time_advance.h", "RK1_TimeAd"), ("time_advance.h", "RK2_TimeAd"),
    ("time_advance.h", "RK3_TimeAd"), ("time_advance.h", "RK1_TimeAd_BS"),
    ("Error.h", "TEST_Scheme_Error_L1"),
    ("Error.h", "calculate_orders"), ("Error.h", "print_error_table"),
]


def test_headers_carry_the_reference_entry_points():
    for header, name in ENTRY_POINTS:
        text = open(os.path.join(SHIM, header)).read()
        assert re.search(rf"\b{name}\s*\(", text), (header, name)


def test_library_exports_the_runtime():
    from overheatingproblem_b200 import lib as L
    text = re.sub(r"/\*.*?\*/", "", open(os.path.join(SHIM, "rpf_runtime.h")).read(), flags=re.S)
    declared = set(re.findall(r"\b(rpf_[a-z_]+)\s*\(", text))
    assert {"rpf_init", "rpf_rk", "rpf_delta_t", "rpf_boundary"} <= declared
    out = subprocess.run(["nm", "-D", "--defined-only", L.library_path()], capture_output=True,
                         text=True, check=True).stdout
    exported = {line.split()[-1] for line in out.splitlines() if " T " in line}
    assert declared <= exported, declared - exported


def test_a_caller_compiles_against_the_set(tmp_path):
    """A caller that includes every header the way src/RP_FVM.c does."""
    src = tmp_path / "caller.c"
    src.write_text("""
#include <stdlib.h>
#include "mesh.h"
#include "initialize.h"
#include "CFD_convection.h"
#include "CFD_diffusion.h"
#include "Boundary_Condition.h"
#include "time_advance.h"
#include "scheme.h"
#include "Golbal.h"
#include "Error.h"
BoundaryConfig bc_config = {BC_OUTFLOW, BC_OUTFLOW, BC_OUTFLOW, BC_OUTFLOW};
int main(void) {
    int rows = 24, cols = 20;
    double (*U)[rows][cols] = malloc(4 * sizeof(double[rows][cols]));
    double (*P)[rows][cols] = malloc(4 * sizeof(double[rows][cols]));
    double Lx, Ly, Tm;
    M_gamma = 1.4;
    Init_Euler_2D(TEST_2D_SHOCKTUBE_CASE3, var, rows, cols, GhostCell, P, U, U, U, &Lx, &Ly, &Tm);
    double dt = Get_Delta_T_2D(var, rows, cols, U, Lx / 16, Ly / 12);
    RK3_TimeAd(2, var, rows, cols, GhostCell, U, dt, Lx / 16, Ly / 12);
    Con_to_Pri_2D(var, rows, cols, P, U);
    free(U); free(P);
    return 0;
}
""")
    res = subprocess.run(["gcc", "-std=gnu11", "-Wall", "-Werror", "-Wno-unused-variable",
                          "-Wno-unused-function", "-fsyntax-only", "-I", SHIM, str(src)],
                         capture_output=True, text=True)
    assert res.returncode == 0, res.stderr


@pytest.mark.skipif(not os.path.exists(REF_CALLER), reason="reference tree not present")
def test_reference_caller_compiles_unchanged():
    res = subprocess.run(["gcc", "-std=gnu11", "-fopenmp", "-fsyntax-only", "-I", SHIM,
                          REF_CALLER], capture_output=True, text=True)
    assert res.returncode == 0, res.stderr[-3000:]


@pytest.mark.skipif(HAVE_GPU, reason="checks the no-GPU failure path")
def test_built_caller_stops_without_a_gpu(tmp_path):
    binary = os.path.join(ROOT, "oracle", "_ref", "rp_fvm_b200")
    if not os.path.exists(binary):
        pytest.skip("drop-in caller not built")
    ctl = tmp_path / "c.txt"
    ctl.write_text("TestCase: 2D_Riemann_Case3\nL_nx: 16\nL_ny: 16\noutput_dir: out\n")
    res = subprocess.run([binary, str(ctl)], cwd=tmp_path, capture_output=True, text=True,
                         errors="replace", timeout=120)
    assert res.returncode == 1
    assert "no CUDA device" in res.stderr
    assert not (tmp_path / "out").exists() or not os.listdir(tmp_path / "out")
