"""GPU parity at the benchmark configurations' own grid sizes.

The other parity tests run on grids of at most 400 x 8 or 96 x 80 cells.  These
run the FP64 form at the sizes the benchmark configurations name -- the
1024^2 and 4096^2 four-quadrant problems and the 1920 x 480 double-Mach
reflection -- where a stage launch covers thousands of tiles, the ragged
last tile row and column sit at other offsets, and the state no longer fits
in L2.  The checker is the reference itself, built from its own sources into
oracle/_ref (RK3_TimeAd, include/time_advance.h:788-882, with Get_Delta_T_2D,
include/function.h:144-175), run on the host cores; where that build is absent
the C restatement (oracle/euler_oracle.c), which is pinned to it bit for bit,
stands in.  The bar is identical bits, with the CFL step equal at every step.
"""
from __future__ import annotations

import numpy as np
import pytest

from conftest import bit_report, interior, noncorner_mask, same_bits
from oracle.bind import DOUBLE_MACH, FOUR_QUADRANT, Reference

pytestmark = pytest.mark.gpu

# TestCase2D value of the reference's own double-Mach case (include/Golbal.h)
REF_DOUBLE_MACH = 16


def checker(oracle, variant: str):
    """The reference build of the given variant, else the oracle."""
    return Reference(variant) if Reference.available(variant) else oracle


def steps_against(ref, s, p, U, nsteps, scheme, dx, dy, t0=0.0, order=3):
    """`nsteps` steps on the GPU context `s` and on the checker from the same
    state U (modified in place); the CFL step must agree at every step."""
    t = t0
    for _ in range(nsteps):
        dt = ref.dt(p, U, dx, dy)
        assert s.delta_t(dx, dy) == dt
        ref.rk(p, order, scheme, U, dt, dx, dy, t)
        s.rk_step(order, scheme, dt, dx, dy, t)
        t += dt
    return U


@pytest.mark.parametrize("n,nsteps", [(1024, 10), (4096, 1)])
def test_four_quadrant_at_size(gpu, oracle, n, nsteps):
    """The four-quadrant Riemann problem at 1024^2 (ten steps from the initial
    state) and at 4096^2 (one step): characteristic WENO5-JS + HLLC + SSP-RK3,
    CFL 0.5, all sides outflow."""
    ref = checker(oracle, "wjs")
    p = oracle.params(n, n, recon=5, characteristic=1, weno_z=0, cfl=0.5)
    U0, lx, ly, _ = oracle.init_case(p, FOUR_QUADRANT)
    dx, dy = lx / n, ly / n
    with gpu.Solver(n, n, recon=5, characteristic=True, weno_z=False, cfl=0.5) as s:
        s.init_case(gpu.lib.CASE_FOUR_QUADRANT)
        U = s.download()
        assert same_bits(interior(U), interior(U0))
        steps_against(ref, s, p, U, nsteps, 2, dx, dy)
        assert s.status() == 0
        Ug = s.download()
    m = noncorner_mask(U.shape)
    assert same_bits(Ug[:, m], U[:, m]), bit_report(Ug[:, m], U[:, m])


def test_double_mach_reference_setup_at_size(gpu, oracle):
    """The reference's own double-Mach case (Init_Euler_2D, include/initialize.h
    :886-965) on the 1920 x 480 grid of the benchmark configuration, with the
    boundary kinds that case sets (inflow left, outflow right, reflecting
    bottom and top, :897-901): its initial state, and the first three
    characteristic WENO5-JS + HLLC + SSP-RK3 steps at CFL 0.4."""
    nx, ny = 1920, 480
    p = oracle.params(nx, ny, recon=5, characteristic=1, weno_z=0, cfl=0.4)
    if Reference.available("wjs"):
        ref = Reference("wjs")
        U, lx, ly, _, kinds = ref.init(REF_DOUBLE_MACH, nx, ny)
        for q in range(4):
            p.bc[q] = kinds[q]
    else:
        ref = oracle
        U, lx, ly, _ = oracle.init_case(p, DOUBLE_MACH)
    dx, dy = lx / nx, ly / ny
    with gpu.Solver(nx, ny, recon=5, characteristic=True, weno_z=False, cfl=0.4) as s:
        lx2, ly2, _ = s.init_case(gpu.lib.CASE_DOUBLE_MACH)
        assert (lx2, ly2) == (lx, ly)
        assert tuple(s.get_bc()) == tuple(p.bc)
        assert same_bits(interior(s.download()), interior(U))
        s.upload(U)
        steps_against(ref, s, p, U, 3, 2, dx, dy)
        Ug = s.download()
    m = noncorner_mask(U.shape)
    assert same_bits(Ug[:, m], U[:, m]), bit_report(Ug[:, m], U[:, m])


def test_double_mach_exact_boundary_at_size(gpu, oracle):
    """One step of the 1920 x 480 double-Mach reflection with the exact
    moving-shock boundary BC_DoubleMach_2D (include/Boundary_Condition.h
    :480-692) on every stage input, checked against the reference's own
    RK3_TimeAd with its commented-out BC_DoubleMach_2D lines switched on (the
    wjs_dmr build).  As at 48 x 12, the reference's scheme reconstructs
    non-physical states at the wall on the first step and goes non-finite; the
    GPU flags it and leaves the same values, NaNs included."""
    nx, ny = 1920, 480
    ref = checker(oracle, "wjs_dmr")
    p = oracle.params(nx, ny, recon=5, characteristic=1, weno_z=0, cfl=0.4)
    U0, lx, ly, _ = oracle.init_case(p, DOUBLE_MACH)
    p.dmr = 1
    dx, dy = lx / nx, ly / ny
    with gpu.Solver(nx, ny, recon=5, characteristic=True, weno_z=False, cfl=0.4) as s:
        s.init_case(gpu.lib.CASE_DOUBLE_MACH)
        s.set_double_mach(True)
        U = s.download()
        assert same_bits(interior(U), interior(U0))
        dt = ref.dt(p, U, dx, dy)
        assert s.delta_t(dx, dy) == dt
        ref.rk(p, 3, 2, U, dt, dx, dy, 0.0)
        rc = s.rk_step(3, 2, dt, dx, dy, 0.0)
        assert rc == gpu.lib.EB2_ENONPHYS
        assert s.status() & gpu.lib.ST_NONPHYSICAL
        Ug = s.download()
    assert np.isnan(interior(U)).any()
    assert same_bits(interior(Ug), interior(U)), bit_report(interior(Ug), interior(U))
