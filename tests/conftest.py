"""Shared fixtures and helpers.

Markers: ``gpu`` tests need a CUDA device and the built libeuler_b200.so; all
other tests run on the CPU (oracle pinning, host logic, library exports).
"""
from __future__ import annotations

import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

GOLDEN = os.path.join(ROOT, "tests", "golden")
GC = 4


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200) and libeuler_b200.so")


def golden(name: str):
    return np.load(os.path.join(GOLDEN, name + ".npz"))


def noncorner_mask(shape, gc: int = GC) -> np.ndarray:
    """All cells except the four gc x gc ghost corners (never read by the solver)."""
    m = np.ones(shape[-2:], dtype=bool)
    m[:gc, :gc] = m[:gc, -gc:] = m[-gc:, :gc] = m[-gc:, -gc:] = False
    return m


def interior(a, gc: int = GC):
    return a[..., gc:-gc, gc:-gc]


def same_bits(a, b) -> bool:
    """Bitwise equality of float64 arrays, NaNs equal to NaNs of any payload."""
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    if a.shape != b.shape:
        return False
    na, nb = np.isnan(a), np.isnan(b)
    if not np.array_equal(na, nb):
        return False
    return np.array_equal(a[~na].view(np.int64), b[~nb].view(np.int64))


def bit_report(a, b) -> str:
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    diff = ~((a == b) | (np.isnan(a) & np.isnan(b)))
    n = int(diff.sum())
    if not n:
        return "identical"
    idx = np.argwhere(diff)[:5].tolist()
    return f"{n} differing entries, first {idx}, max |d| {np.nanmax(np.abs(a - b)):.3e}"


@pytest.fixture(scope="session")
def oracle():
    from oracle.bind import Oracle
    return Oracle()


def _gpu_available() -> bool:
    try:
        import ctypes
        rt = ctypes.CDLL("libcudart.so.12")
        n = ctypes.c_int(0)
        return rt.cudaGetDeviceCount(ctypes.byref(n)) == 0 and n.value > 0
    except OSError:
        return False


HAVE_GPU = _gpu_available()


@pytest.fixture(scope="session")
def gpu():
    """The product library on a GPU.  Fails loudly (not skip) when the library
    is missing; skips only when no CUDA device exists."""
    if not HAVE_GPU:
        pytest.skip("no CUDA device")
    import overheatingproblem_b200 as eb2
    eb2.library()
    return eb2
