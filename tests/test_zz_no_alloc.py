"""eb2_rk_step_noalloc: the RK step for callers that cannot allocate device
memory (a host application whose own pool owns the GPU's memory, a real-time
loop that forbids allocation after start-up, a plug-in that is only handed
device pointers).  It keeps its scratch in a static device array of the
library, so the caller only passes its own device state.

Checked through the C ABI against the context-based eb2_rk_step on two calls
in a row, to the same tolerance as the other FP64 tests: identical bits.  This
file is collected last so that a failure here does not hide any other test;
it also passes alone in a fresh process.
"""
from __future__ import annotations

import ctypes as C

import numpy as np
import pytest

from conftest import bit_report, noncorner_mask, same_bits

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("order,scheme,recon,ch", [(3, 2, 5, 1), (2, 3, 2, 0)])
def test_noalloc_step_matches_context_step(gpu, order, scheme, recon, ch):
    import torch

    L = gpu.lib
    lib = L.library()
    nx, ny = 64, 48
    dx, dy = 1.0 / nx, 1.0 / ny
    # the existing entry point: two steps on a context
    ref = []
    with gpu.Solver(nx, ny, recon=recon, characteristic=bool(ch), weno_z=False) as s:
        s.init_case(L.CASE_FOUR_QUADRANT)
        U0 = s.download()
        for _ in range(2):
            dt = s.delta_t(dx, dy)
            s.rk_step(order, scheme, dt, dx, dy)
            ref.append((dt, s.download()))
    cfg = L.NoallocConfig(gamma=1.4, recon=recon, characteristic=ch, weno_z=0, bc_left=0,
                          bc_right=0, bc_bottom=0, bc_top=0, source=0, gravity=1.0)
    # the caller owns the device state; the entry point allocates nothing
    dev = torch.from_numpy(U0).to("cuda")
    stream = torch.cuda.current_stream()
    for dt, U_ref in ref:
        rc = lib.eb2_rk_step_noalloc(C.c_void_p(dev.data_ptr()), nx, ny, C.byref(cfg), order,
                                     scheme, dt, dx, dy, 0.0, C.c_void_p(stream.cuda_stream))
        assert rc == L.EB2_OK, lib.eb2_last_error()
        got = dev.cpu().numpy()
        m = noncorner_mask(got.shape)
        assert same_bits(got[:, m], U_ref[:, m]), bit_report(got[:, m], U_ref[:, m])


def test_noalloc_rejects_grids_beyond_its_scratch(gpu):
    import torch

    L = gpu.lib
    lib = L.library()
    cfg = L.NoallocConfig(gamma=1.4, recon=5, characteristic=1, weno_z=0)
    n = int(np.sqrt(L.NOALLOC_MAX_CELLS))   # (n+8)^2 exceeds the limit
    dev = torch.zeros(8, dtype=torch.float64, device="cuda")  # never touched: rejected first
    rc = lib.eb2_rk_step_noalloc(C.c_void_p(dev.data_ptr()), n, n, C.byref(cfg), 3, 2, 1e-3,
                                 1.0 / n, 1.0 / n, 0.0, None)
    assert rc == L.EB2_EARG
    assert b"EB2_NOALLOC_MAX_CELLS" in lib.eb2_last_error()
