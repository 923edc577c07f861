"""Mixed-precision form: FP32 reconstruction and fluxes, FP64 state, RK sums and
CFL reduction.  Checked against the FP64 form (itself bit-identical to the
reference) with the stated tolerance, for conservation to FP64 round-off,
and for its near-vacuum FP64 eigenvector path."""
from __future__ import annotations

import numpy as np
import pytest

from conftest import GC, interior

pytestmark = pytest.mark.gpu

# Density L1 error of the mixed form against the FP64 form (mean |drho| over
# the interior) allowed after the runs below.
L1_TOL = 1.0e-6


def pair(gpu, nx, ny, case, **kw):
    a = gpu.Solver(nx, ny, precision=gpu.lib.FP64, **kw)
    b = gpu.Solver(nx, ny, precision=gpu.lib.MIXED, **kw)
    a.init_case(case)
    b.init_case(case)
    return a, b


@pytest.mark.parametrize("scheme,wz", [(2, False), (3, False), (2, True), (1, False)])
def test_mixed_four_quadrant_error(gpu, scheme, wz):
    """256^2 four-quadrant problem to t = 0.05: mixed vs FP64 density L1."""
    a, b = pair(gpu, 256, 256, gpu.lib.CASE_FOUR_QUADRANT, recon=5, characteristic=True,
                weno_z=wz)
    with a, b:
        na, ta = a.run(3, scheme, 1 / 256, 1 / 256, 0.05)
        nb, tb = b.run(3, scheme, 1 / 256, 1 / 256, 0.05)
        assert b.status() == 0
        ra, rb = interior(a.download())[0], interior(b.download())[0]
    assert tb == pytest.approx(0.05, abs=1e-15)
    l1 = float(np.mean(np.abs(ra - rb)))
    linf = float(np.max(np.abs(ra - rb)))
    print(f"scheme {scheme} weno_z {wz}: steps {na}/{nb}  L1 {l1:.3e}  Linf {linf:.3e}")
    assert abs(na - nb) <= 1
    assert l1 < L1_TOL, (l1, linf)


def test_mixed_conserves_to_round_off(gpu):
    """Periodic box, smooth random state: the FP64 flux differences telescope,
    so the totals of all four conserved fields stay fixed to FP64 round-off."""
    nx, ny = 96, 64
    rng = np.random.default_rng(3)
    x = np.linspace(0, 2 * np.pi, nx, endpoint=False)[:, None]
    y = np.linspace(0, 2 * np.pi, ny, endpoint=False)[None, :]
    U = np.zeros((4, nx + 8, ny + 8))
    rho = 1.0 + 0.2 * np.sin(x) * np.cos(y) + 0.01 * rng.random((nx, ny))
    u = 0.5 * np.cos(y) + 0 * x
    v = 0.3 * np.sin(x) + 0 * y
    p = 1.0 + 0.1 * np.cos(x + y)
    U[0, GC:-GC, GC:-GC] = rho
    U[1, GC:-GC, GC:-GC] = rho * u
    U[2, GC:-GC, GC:-GC] = rho * v
    U[3, GC:-GC, GC:-GC] = p / 0.4 + 0.5 * rho * (u * u + v * v)
    with gpu.Solver(nx, ny, precision=gpu.lib.MIXED, recon=5, characteristic=True,
                    weno_z=False) as s:
        s.set_bc(2, 2, 2, 2)
        s.upload(U)
        s.advance(3, 2, 1 / nx, 1 / ny, 50)
        V = s.download()
    t0 = interior(U).sum(axis=(1, 2))
    t1 = interior(V).sum(axis=(1, 2))
    assert np.all(np.abs(t1 - t0) <= 1e-12 * np.maximum(np.abs(t0), 1.0) * nx * ny / 100), (t0, t1)


def test_mixed_wall_heating_profile(gpu):
    """The 400x8 wall-heating run to t = 0.6 in the mixed form against FP64."""
    a, b = pair(gpu, 400, 8, gpu.lib.CASE_WALL_HEATING, recon=5, characteristic=True,
                weno_z=False)
    with a, b:
        a.run(3, 2, 1 / 400, 0.02 / 8, 0.6)
        b.run(3, 2, 1 / 400, 0.02 / 8, 0.6)
        assert b.status() == 0
        ra, rb = interior(a.download())[0], interior(b.download())[0]
    l1 = float(np.mean(np.abs(ra - rb)))
    print(f"wall heating mixed vs FP64: L1 {l1:.3e}  Linf {np.max(np.abs(ra - rb)):.3e}")
    assert l1 < 10 * L1_TOL
    # the wall-heating density dip survives: lowest density at the wall
    prof = rb.mean(axis=1)
    assert prof[0] < prof[10] and prof[0] == prof[:40].min()


def test_mixed_near_vacuum_path(gpu):
    """Two strong rarefactions (u = -+3) open a near-vacuum region; the FP64
    eigenvector path keeps the mixed form finite and positive."""
    nx, ny = 128, 8
    U = np.zeros((4, nx + 8, ny + 8))
    rho, p = 1.0, 0.4
    u = np.where(np.arange(nx) < nx // 2, -3.0, 3.0)[:, None] * np.ones((1, ny))
    U[0, GC:-GC, GC:-GC] = rho
    U[1, GC:-GC, GC:-GC] = rho * u
    U[3, GC:-GC, GC:-GC] = p / 0.4 + 0.5 * rho * u * u
    with gpu.Solver(nx, ny, precision=gpu.lib.MIXED, recon=5, characteristic=True,
                    weno_z=False) as s:
        s.upload(U)
        s.run(3, 2, 1 / nx, 1 / ny, 0.15)
        V = s.download()
        st = s.status()
        pri = s.con_to_pri()
    assert st == 0
    pin = interior(pri)
    assert np.all(np.isfinite(pin)) and pin[0].min() > 0 and pin[3].min() > 0
    assert pin[3].min() < 1e-3 * pin[3].mean()   # the near-vacuum path was exercised
