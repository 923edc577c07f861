"""Pin the CPU oracle (oracle/euler_oracle.c) to the reference.

Against the golden vectors that tests/golden/make_golden.py produced from the
reference built from its own sources, bit for bit; and, where oracle/_ref is
built (in the container that holds the reference tree), against the live
reference on extra cases.
"""
from __future__ import annotations

import numpy as np
import pytest

from conftest import GC, bit_report, golden, interior, noncorner_mask, same_bits
from oracle.bind import (DOUBLE_MACH, FIXED, FOUR_QUADRANT, INFLOW, OUTFLOW, PERIODIC,
                         REFLECT, WALL_HEATING, Reference)

FQ = ["charjs_hllc_rk3", "comp_weno_hllc_rk3", "charz_roe_rk3", "charz_hll_rk2",
      "comp_weno_llf_rk1", "tvd_char_hllc_rk3", "tvd_comp_roe_rk3", "godunov_char_hll_rk3",
      "godunov_comp_hllc_rk1",
      "charjs_hllhc_rk3", "comp_weno_hllchc_rk3", "charz_roehc_rk3",
      "tvd_char_hllchc_rk2", "godunov_comp_roehc_rk1",
      "weno3_char_hllc_rk3", "weno3_comp_roe_rk2"]


@pytest.mark.parametrize("name", FQ)
def test_rk_steps_match_reference(oracle, name):
    z = golden(f"fq_{name}")
    p = oracle.params(32, 24, recon=int(z["recon"]), characteristic=int(z["characteristic"]),
                      weno_z=int(z["weno_z"]), cfl=0.5)
    U0, *_ = oracle.init_case(p, FOUR_QUADRANT)
    assert same_bits(interior(U0), interior(z["U0"]))
    U = z["U0"].copy()
    for dt_ref in z["dts"]:
        dt = oracle.dt(p, U, 1 / 32, 1 / 24)
        assert dt == dt_ref
        oracle.rk(p, int(z["order"]), int(z["scheme"]), U, dt, 1 / 32, 1 / 24)
    m = noncorner_mask(U.shape)
    assert same_bits(U[:, m], z["U"][:, m]), bit_report(U[:, m], z["U"][:, m])


@pytest.mark.parametrize("name,scheme", [("wall_heating_400x8_t0.6", 2),
                                         ("wall_heating_400x8_t0.6_hllchc", 22)])
def test_wall_heating_full_run(oracle, name, scheme):
    """The 400x8 wall-heating configuration to t = 0.6 (754 steps), with HLLC
    and with the anti-overheating HLLCHC flux."""
    z = golden(name)
    p = oracle.params(400, 8, recon=5, characteristic=1, weno_z=0, cfl=0.5)
    U0, lx, ly, tmax = oracle.init_case(p, WALL_HEATING)
    assert same_bits(U0, z["U0"])
    U = U0.copy()
    n, tf = oracle.run(p, 3, scheme, U, lx / 400, ly / 8, tmax, 1)
    assert n == int(z["steps"]) and tf == float(z["t_final"])
    m = noncorner_mask(U.shape)
    assert same_bits(U[:, m], z["U"][:, m]), bit_report(U[:, m], z["U"][:, m])


def test_rayleigh_taylor_full_run(oracle):
    """Rayleigh-Taylor (TestCase2D 15), 16x64 to t = 0.5 (254 steps): the
    gravity source and the fixed-value bottom and top boundaries (the Mach-3
    state the reference's globals hold) in a full time loop, started from the
    reference's own initial state."""
    z = golden("rayleigh_taylor_16x64_t0.5")
    bc = tuple(int(b) for b in z["bc"])
    assert bc == (REFLECT, REFLECT, FIXED, FIXED)
    p = oracle.params(16, 64, recon=5, characteristic=1, weno_z=1, cfl=0.5, source=1,
                      gravity=1.0, bc=bc)
    U = z["U0"].copy()
    n, tf = oracle.run(p, 3, 2, U, float(z["lx"]) / 16, float(z["ly"]) / 64, 0.5, 1)
    assert n == int(z["steps"]) and tf == float(z["t_final"])
    m = noncorner_mask(U.shape)
    assert same_bits(U[:, m], z["U"][:, m]), bit_report(U[:, m], z["U"][:, m])


@pytest.mark.parametrize("tag,ch,wz,scheme", [("charjs_hllc", 1, 0, 2)])
def test_double_mach_exact_boundary_step(oracle, tag, ch, wz, scheme):
    """The exact double-Mach boundary: the reference goes non-finite on the
    first step; the oracle reproduces where and how."""
    z = golden(f"dmr_{tag}_48x12_step1")
    p = oracle.params(48, 12, recon=5, characteristic=ch, weno_z=wz, cfl=0.4)
    U0, lx, ly, _ = oracle.init_case(p, DOUBLE_MACH)
    p.dmr = 1
    assert same_bits(interior(U0), interior(z["U0"]))
    U = U0.copy()
    dt = oracle.dt(p, U, lx / 48, ly / 12)
    assert dt == float(z["dt"])
    oracle.rk(p, 3, scheme, U, dt, lx / 48, ly / 12, 0.0)
    assert np.isnan(interior(z["U"])).any()
    assert same_bits(interior(U), interior(z["U"])), bit_report(interior(U), interior(z["U"]))


def test_precision_known_answer(oracle):
    """Precision_test (src/RP_FVM.c:974-1072): fifth-order convergence, and the
    same bits as the reference on every grid."""
    import json
    import os
    from conftest import GOLDEN
    with open(os.path.join(GOLDEN, "manifest.json")) as fh:
        l1_ref = {int(k): v for k, v in json.load(fh)["precision"].items()}
    l1 = {}
    for nx in (10, 20, 40, 80):
        z = golden(f"precision_nx{nx}")
        p = oracle.params(nx, 1, recon=5, characteristic=0)
        U0, lx, ly, tmax = oracle.init_case(p, 4)
        assert same_bits(U0, z["U0"])
        U = U0.copy()
        dx, dy = lx / nx, ly / 1
        t = 0.0
        while t < tmax:
            dt = 0.5 * dx ** (5.0 / 3)
            if t + dt >= tmax:
                dt = tmax - t
            oracle.rk(p, 3, 2, U, dt, dx, dy)
            t = t + dt
        assert same_bits(U[0, GC:-GC, GC], z["U"][0, GC:-GC, GC])
        xc = (np.arange(nx) + 0.5) * dx
        l1[nx] = float(np.sum(np.abs(1.0 + 0.2 * np.sin(xc - t) - U[0, GC:-GC, GC])) * dx)
        assert l1[nx] == l1_ref[nx]
    orders = [np.log2(l1[a] / l1[2 * a]) for a in (10, 20, 40)]
    assert orders[-1] > 4.5, orders


def test_granular_operators(oracle):
    z = golden("granular_20x16")
    p = oracle.params(20, 16, recon=5, characteristic=1, weno_z=1)
    dx, dy = 1 / 20, 1 / 16
    U = z["U"].copy()
    oracle.bc(p, U)
    m = noncorner_mask(U.shape)
    assert same_bits(U[:, m], z["Ub"][:, m])
    Ub = z["Ub"]
    pri = oracle.con_to_pri(p, Ub)
    box = (slice(None), slice(GC - 1, -GC + 1), slice(GC - 1, -GC + 1))
    assert same_bits(pri[box], z["pri"][box])
    for d in (1, 2):
        el, er = oracle.eigen(p, d, z["pri"])
        # interfaces whose two cells lie in the primitive box
        sl = (slice(None), slice(None), slice(GC - 1, -GC), slice(GC, -GC)) if d == 1 else \
             (slice(None), slice(None), slice(GC, -GC), slice(GC - 1, -GC))
        assert same_bits(el[sl], z[f"eig_l{d}"][sl])
        assert same_bits(er[sl], z[f"eig_r{d}"][sl])
        face = (slice(None), slice(GC - 1, -GC), slice(GC, -GC)) if d == 1 else \
               (slice(None), slice(GC, -GC), slice(GC - 1, -GC))
        for tag, (recon, ch, wz) in {"charz": (5, 1, 1), "charjs": (5, 1, 0), "comp": (5, 0, 1),
                                     "tvdc": (2, 1, 1), "tvdm": (2, 0, 1),
                                     "god": (1, 1, 1), "w3c": (3, 1, 1), "w3m": (3, 0, 1)}.items():
            q = oracle.params(20, 16, recon=recon, characteristic=ch, weno_z=wz)
            ql, qr = oracle.recon(q, d, Ub, dx, dy)
            assert same_bits(ql[face], z[f"ql_{tag}{d}"][face]), tag
            assert same_bits(qr[face], z[f"qr_{tag}{d}"][face]), tag
        for scheme in (1, 2, 3, 4, 11, 22, 33):
            fl = oracle.riemann(p, scheme, d, z[f"ql_charz{d}"], z[f"qr_charz{d}"])
            assert same_bits(fl[face], z[f"flux{scheme}_{d}"][face]), (scheme, d)
    f, g = oracle.flux_recon(p, 2, Ub, dx, dy)
    fx = (slice(None), slice(GC - 1, -GC), slice(GC, -GC))
    gy = (slice(None), slice(GC, -GC), slice(GC - 1, -GC))
    assert same_bits(f[fx], z["f"][fx]) and same_bits(g[gy], z["g"][gy])
    Lt = oracle.space_item(p, dx, dy, z["f"], z["g"], np.zeros_like(Ub))
    assert same_bits(interior(Lt), interior(z["L"]))
    assert oracle.dt(p, z["U"], dx, dy) == float(z["dt"])


def test_boundary_kinds(oracle):
    z = golden("boundary_12x10")
    for key in z.files:
        U, Ub = z[key][0].copy(), z[key][1]
        p = oracle.params(12, 10)
        if key == "bc_dmr_t0.05":
            p.dmr = 1
            oracle.bc(p, U, 0.05)
        else:
            kinds = [int(c) for c in key[3:]]
            for s in range(4):
                p.bc[s] = kinds[s]
            oracle.bc(p, U)
        m = noncorner_mask(U.shape)
        assert same_bits(U[:, m], Ub[:, m]), (key, bit_report(U[:, m], Ub[:, m]))


# --- live comparisons against the reference build (only where it exists) ---

need_ref = pytest.mark.skipif(not Reference.available() or not Reference.available("wjs"),
                              reason="oracle/_ref not built (needs the reference tree)")


@need_ref
@pytest.mark.parametrize("kinds", [(REFLECT, OUTFLOW, PERIODIC, PERIODIC),
                                   (PERIODIC, PERIODIC, REFLECT, REFLECT),
                                   (INFLOW, OUTFLOW, REFLECT, OUTFLOW)])
@pytest.mark.parametrize("scheme", [1, 2, 3, 4])
def test_live_reference_random_state(oracle, kinds, scheme):
    """A smooth random state under mixed boundaries, 3 RK3 steps."""
    ref = Reference("wjs")
    p = oracle.params(18, 14, recon=5, characteristic=1, weno_z=0, bc=kinds)
    rng = np.random.default_rng(scheme)
    W = np.zeros((4, 26, 22))
    x = np.linspace(0, 2 * np.pi, 18)[:, None]
    y = np.linspace(0, 2 * np.pi, 14)[None, :]
    W[0, GC:-GC, GC:-GC] = 1.0 + 0.3 * np.sin(x) * np.cos(y) + 0.05 * rng.random((18, 14))
    W[1, GC:-GC, GC:-GC] = 0.4 * np.cos(x + y)
    W[2, GC:-GC, GC:-GC] = -0.3 * np.sin(2 * y) + 0.1 * rng.random((18, 14))
    W[3, GC:-GC, GC:-GC] = 1.0 + 0.2 * np.cos(x - y)
    U = np.zeros_like(W)
    U[0] = W[0]
    U[1] = W[1] * W[0]
    U[2] = W[2] * W[0]
    U[3] = W[3] / 0.4 + 0.5 * W[0] * (W[1] ** 2 + W[2] ** 2)
    Ua, Ub = U.copy(), U.copy()
    for _ in range(3):
        dt = oracle.dt(p, Ua, 1 / 18, 1 / 14)
        assert dt == ref.dt(p, Ub, 1 / 18, 1 / 14)
        oracle.rk(p, 3, scheme, Ua, dt, 1 / 18, 1 / 14)
        ref.rk(p, 3, scheme, Ub, dt, 1 / 18, 1 / 14)
    m = noncorner_mask(U.shape)
    assert same_bits(Ua[:, m], Ub[:, m]), bit_report(Ua[:, m], Ub[:, m])


@need_ref
def test_live_reference_time_loop(oracle):
    """The time loop (CFL dt, clipping at output times) on the reference's own
    double-Mach case with its own boundary kinds, characteristic WENO5-Z + Roe."""
    p = oracle.params(60, 15, recon=5, characteristic=1, weno_z=1, cfl=0.4)
    U0, lx, ly, _ = oracle.init_case(p, DOUBLE_MACH)
    ref = Reference("")
    Ua, Ub = U0.copy(), U0.copy()
    na, ta = oracle.run(p, 3, 3, Ua, lx / 60, ly / 15, 0.01, 3)
    nb, tb = ref.run(p, 3, 3, Ub, lx / 60, ly / 15, 0.01, 3)
    assert (na, ta) == (nb, tb)
    m = noncorner_mask(Ua.shape)
    assert same_bits(Ua[:, m], Ub[:, m]), bit_report(Ua[:, m], Ub[:, m])


need_dmr = pytest.mark.skipif(not Reference.available("wjs_dmr"),
                              reason="oracle/_ref not built (needs the reference tree)")


@need_dmr
@pytest.mark.parametrize("scheme", [2, 3])
def test_double_mach_step_is_the_references_own(oracle, scheme):
    """One step with the exact double-Mach boundary.  The reference carries a
    BC_DoubleMach_2D call, commented out, beside each stage's ghost fill of its
    RK stages (include/time_advance.h:747-862); the wjs_dmr build switches
    those lines on, so its RK3_TimeAd is the reference's own double-Mach step.
    The composed ref_rk_dmr, the oracle and the committed golden vector (the
    GPU's check) all give its bits -- NaNs where the scheme breaks down
    included.  (HLL is left out: where it skips an interface the reference
    copies a flux entry it never wrote from an uninitialised temporary, so two
    reference builds need not agree there.)"""
    dmr = Reference("wjs_dmr")
    wjs = Reference("wjs")
    p = oracle.params(48, 12, recon=5, characteristic=1, weno_z=0, cfl=0.4)
    U0, lx, ly, _ = oracle.init_case(p, DOUBLE_MACH)
    p.dmr = 1
    dx, dy = lx / 48, ly / 12
    Ua, Ub, Uc = U0.copy(), U0.copy(), U0.copy()
    for t in (0.0, 1e-3):
        dt = dmr.dt(p, Ua, dx, dy)
        assert dt == wjs.dt(p, Ub, dx, dy) == oracle.dt(p, Uc, dx, dy)
        dmr.rk(p, 3, scheme, Ua, dt, dx, dy, t)
        wjs.rk(p, 3, scheme, Ub, dt, dx, dy, t)
        oracle.rk(p, 3, scheme, Uc, dt, dx, dy, t)
        m = noncorner_mask(Ua.shape)
        assert same_bits(Ua[:, m], Ub[:, m]), bit_report(Ua[:, m], Ub[:, m])
        assert same_bits(Ua[:, m], Uc[:, m]), bit_report(Ua[:, m], Uc[:, m])
        if scheme == 2 and t == 0.0:
            z = golden("dmr_charjs_hllc_48x12_step1")
            assert dt == float(z["dt"])
            assert same_bits(interior(Ua), interior(z["U"]))
