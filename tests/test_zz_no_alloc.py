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


# (order, AR_scheme, recon, characteristic, bc kinds left/right/bottom/top,
# gravity source): the three step orders (order 1 writes into the scratch then
# copies back), every reconstruction family, a heat-conduction flux, and
# reflecting, periodic and inflow ghost fills with the gravity source on
CASES = [
    (3, 2, 5, 1, (0, 0, 0, 0), 0),
    (2, 3, 2, 0, (0, 0, 0, 0), 0),
    (1, 1, 1, 0, (1, 0, 2, 2), 0),
    (3, 22, 3, 1, (1, 1, 2, 2), 1),
    (2, 2, 5, 0, (2, 2, 1, 1), 1),
    (3, 33, 5, 1, (3, 0, 1, 0), 0),
]


@pytest.mark.parametrize("order,scheme,recon,ch,kinds,src", CASES)
def test_noalloc_step_matches_context_step(gpu, order, scheme, recon, ch, kinds, src):
    import torch

    L = gpu.lib
    lib = L.library()
    nx, ny = 64, 48
    dx, dy = 1.0 / nx, 1.0 / ny
    # the existing entry point: two steps on a context
    ref = []
    with gpu.Solver(nx, ny, recon=recon, characteristic=bool(ch), weno_z=False,
                    source=bool(src), gravity=1.0) as s:
        s.init_case(L.CASE_FOUR_QUADRANT)
        s.set_bc(*kinds)
        U0 = s.download()
        for _ in range(2):
            dt = s.delta_t(dx, dy)
            rc = s.rk_step(order, scheme, dt, dx, dy)
            ref.append((dt, rc, s.download()))
    cfg = L.NoallocConfig(gamma=1.4, recon=recon, characteristic=ch, weno_z=0,
                          bc_left=kinds[0], bc_right=kinds[1], bc_bottom=kinds[2],
                          bc_top=kinds[3], source=src, gravity=1.0)
    # the caller owns the device state; the entry point allocates nothing
    dev = torch.from_numpy(U0).to("cuda")
    stream = torch.cuda.current_stream()
    seen_nonphys = False
    for dt, rc_ref, U_ref in ref:
        rc = lib.eb2_rk_step_noalloc(C.c_void_p(dev.data_ptr()), nx, ny, C.byref(cfg), order,
                                     scheme, dt, dx, dy, 0.0, C.c_void_p(stream.cuda_stream))
        # the same status as the context step; the context reports a
        # non-physical state once, the no-allocation step on every call
        assert rc in (L.EB2_OK, L.EB2_ENONPHYS), lib.eb2_last_error()
        assert rc == rc_ref or (rc == L.EB2_ENONPHYS and seen_nonphys), lib.eb2_last_error()
        seen_nonphys = seen_nonphys or rc_ref == L.EB2_ENONPHYS
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
