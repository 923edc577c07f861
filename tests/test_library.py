"""The C-ABI library loads and exports every entry point include/*.h declares
(CPU only: no compute calls), and fails loudly without a GPU."""
from __future__ import annotations

import ctypes as C
import os
import re
import subprocess

import pytest

from conftest import HAVE_GPU, ROOT

HEADERS = [os.path.join(ROOT, "include", f) for f in sorted(os.listdir(os.path.join(ROOT, "include")))
           if f.endswith(".h")]


def declared_symbols():
    names = set()
    for h in HEADERS:
        text = open(h).read()
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
        for m in re.finditer(r"\b(eb2_[a-z0-9_]+)\s*\(", text):
            names.add(m.group(1))
    return names


def test_headers_declare_entry_points():
    names = declared_symbols()
    assert {"eb2_ctx_create", "eb2_rk_step", "eb2_run", "eb2_delta_t", "eb2_bc_apply",
            "eb2_reconstruct", "eb2_eigen", "eb2_flux_reconstruction",
            "eb2_read_control_file"} <= names


def test_library_exports_every_declared_symbol():
    from overheatingproblem_b200 import lib as L
    path = L.library_path()
    assert os.path.exists(path), "libeuler_b200.so not built"
    out = subprocess.run(["nm", "-D", "--defined-only", path], capture_output=True, text=True,
                         check=True).stdout
    exported = {line.split()[-1] for line in out.splitlines() if " T " in line}
    missing = declared_symbols() - exported
    assert not missing, missing
    lib = L.library()
    for name in declared_symbols():
        assert hasattr(lib, name)
    # every declared symbol has a ctypes signature in the binding
    assert declared_symbols() <= set(L.SIGNATURES)


@pytest.mark.skipif(HAVE_GPU, reason="checks the no-GPU failure path")
def test_no_gpu_fails_loudly():
    from overheatingproblem_b200 import EB2Error, Solver
    with pytest.raises(EB2Error) as ei:
        Solver(8, 8)
    assert "no CUDA device" in str(ei.value) or "CUDA" in str(ei.value)


def test_version_string():
    from overheatingproblem_b200 import lib as L
    assert b"sm_100a" in L.library().eb2_version()
