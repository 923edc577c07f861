"""Generate the golden vectors in tests/golden/ from the reference itself.

    make -C oracle ref && python tests/golden/make_golden.py

Every array here comes out of oracle/_ref/libref*.so: the reference's own
src/RP_FVM.c and headers compiled from the reference tree by oracle/Makefile
(libref_wjs.so differs only in calling the Jiang-Shu WENO5 weights from the
characteristic branch).  Inputs are the reference's own initial states or the
synthetic states of the benchmark configurations, at sizes small enough to
commit.  The tests compare the CPU oracle (tests/test_oracle_pin.py) and the
GPU path (tests/test_gpu_parity.py) against these files bit for bit.
"""
from __future__ import annotations

import ctypes as C
import json
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)
from oracle.bind import (DOUBLE_MACH, FOUR_QUADRANT, INFLOW, OUTFLOW, PERIODIC,  # noqa: E402
                         REFLECT, WALL_HEATING, Oracle, Reference, _ptr)

OUT = os.path.dirname(os.path.abspath(__file__))
GC = 4


def save(name: str, **arrays) -> None:
    """Write a fixture, unless the committed one already holds the same bits."""
    path = os.path.join(OUT, name + ".npz")
    if os.path.exists(path):
        old = np.load(path)

        def same(a, b):
            a, b = np.atleast_1d(np.asarray(a)), np.atleast_1d(np.asarray(b))
            return (a.shape == b.shape and a.dtype == b.dtype and
                    np.ascontiguousarray(a).tobytes() == np.ascontiguousarray(b).tobytes())
        if set(old.files) == set(arrays) and all(same(old[k], arrays[k]) for k in arrays):
            return
    np.savez_compressed(path, **arrays)


def ref_steps(ref: Reference, p, U, steps, scheme, order=3, dmr_t=None):
    """`steps` steps with the reference's CFL dt; returns states and dts."""
    dx, dy = 1.0 / p.nx, 1.0 / p.ny
    dts = []
    t = 0.0
    for _ in range(steps):
        dt = ref.dt(p, U, dx, dy)
        ref.rk(p, order, scheme, U, dt, dx, dy, t)
        t += dt
        dts.append(dt)
    return U, np.array(dts)


def main() -> None:
    orc = Oracle()
    ref = Reference("")
    wjs = Reference("wjs")
    manifest = {}

    # 1. RK steps on the four-quadrant problem, 32 x 24, one file per scheme
    combos = [
        # name, recon, characteristic, weno_z, scheme, order, library
        ("charjs_hllc_rk3", 5, 1, 0, 2, 3, wjs),     # the benchmark scheme
        ("comp_weno_hllc_rk3", 5, 0, 1, 2, 3, ref),  # the reference as shipped
        ("charz_roe_rk3", 5, 1, 1, 3, 3, ref),
        ("charz_hll_rk2", 5, 1, 1, 1, 2, ref),
        ("comp_weno_llf_rk1", 5, 0, 1, 4, 1, ref),
        ("tvd_char_hllc_rk3", 2, 1, 1, 2, 3, ref),
        ("tvd_comp_roe_rk3", 2, 0, 1, 3, 3, ref),
        ("godunov_char_hll_rk3", 1, 1, 1, 1, 3, ref),
        ("godunov_comp_hllc_rk1", 1, 0, 1, 2, 1, ref),
        # the heat-conduction fluxes, AR_scheme 11 / 22 / 33
        ("charjs_hllhc_rk3", 5, 1, 0, 11, 3, wjs),
        ("comp_weno_hllchc_rk3", 5, 0, 1, 22, 3, ref),
        ("charz_roehc_rk3", 5, 1, 1, 33, 3, ref),
        ("tvd_char_hllchc_rk2", 2, 1, 1, 22, 2, ref),
        ("godunov_comp_roehc_rk1", 1, 0, 1, 33, 1, ref),
        # third-order WENO (Recon_Accur 3)
        ("weno3_char_hllc_rk3", 3, 1, 1, 2, 3, ref),
        ("weno3_comp_roe_rk2", 3, 0, 1, 3, 2, ref),
    ]
    for name, recon, ch, wz, scheme, order, lib in combos:
        p = orc.params(32, 24, recon=recon, characteristic=ch, weno_z=wz, cfl=0.5)
        U0, *_ = orc.init_case(p, FOUR_QUADRANT)
        U, dts = ref_steps(lib, p, U0.copy(), 4, scheme, order)
        save(f"fq_{name}", U0=U0, U=U, dts=dts, recon=recon, characteristic=ch, weno_z=wz,
             scheme=scheme, order=order)
        manifest[f"fq_{name}"] = "four-quadrant 32x24, 4 steps"

    # 2. the wall-heating configuration, 400 x 8 to t = 0.6 (characteristic
    #    WENO5-JS + HLLC + SSP-RK3, CFL 0.5): the full reference run
    p = orc.params(400, 8, recon=5, characteristic=1, weno_z=0, cfl=0.5)
    U0, lx, ly, tmax = orc.init_case(p, WALL_HEATING)
    U = U0.copy()
    n, tf = wjs.run(p, 3, 2, U, lx / 400, ly / 8, tmax, 1)
    save("wall_heating_400x8_t0.6", U0=U0, U=U, steps=n, t_final=tf)
    manifest["wall_heating_400x8_t0.6"] = f"{n} steps to t={tf}"
    # the same run with the anti-overheating HLLCHC flux (AR_scheme 22)
    U = U0.copy()
    n, tf = wjs.run(p, 3, 22, U, lx / 400, ly / 8, tmax, 1)
    save("wall_heating_400x8_t0.6_hllchc", U0=U0, U=U, steps=n, t_final=tf)
    manifest["wall_heating_400x8_t0.6_hllchc"] = f"{n} steps to t={tf}, AR_scheme 22"

    # 2b. Rayleigh-Taylor (TestCase2D 15) on 16 x 64 from the reference's own
    #     Init_Euler_2D state and boundary kinds (reflecting sides, fixed-value
    #     bottom and top), gravity source on (Gravity 1.0, the control-file
    #     default), characteristic WENO5 as shipped + HLLC + SSP-RK3, CFL 0.5,
    #     run by the reference's time loop to t = 0.5
    nx, ny = 16, 64
    rows, cols = nx + 2 * GC, ny + 2 * GC
    pri = np.zeros((4, rows, cols)); U = np.zeros_like(pri)
    F = np.zeros_like(pri); G = np.zeros_like(pri)
    lx, ly, tm = C.c_double(), C.c_double(), C.c_double()
    ref.lib.ref_set_params(1.4, 0.5, 5, 1, 1, 1.0)
    ref.lib.ref_init(15, rows, cols, _ptr(pri), _ptr(U), _ptr(F), _ptr(G), C.byref(lx),
                     C.byref(ly), C.byref(tm))
    b = (C.c_int * 4)()
    ref.lib.ref_get_bc(b)
    U0 = U.copy()
    tf = C.c_double()
    n = ref.lib.ref_run(3, 2, rows, cols, _ptr(U), lx.value / nx, ly.value / ny, 0.5, 1, 0,
                        C.byref(tf))
    save("rayleigh_taylor_16x64_t0.5", U0=U0, U=U, steps=n, t_final=tf.value,
         lx=lx.value, ly=ly.value, bc=np.array(list(b)))
    manifest["rayleigh_taylor_16x64_t0.5"] = f"{n} steps to t={tf.value}, gravity source"

    # 2c. backward step (TestCase2D 20) by the reference's two-block
    #     RK1_TimeAd_BS (include/time_advance.h:886): 40 x 20 from the case's
    #     Init_Euler_2D state, HLLC, dt = 0.1 dx (the caller's step control),
    #     6 steps; component WENO5 without source, and characteristic WENO5 with
    #     the gravity source
    ref.lib.ref_rk1_bs.argtypes = [C.c_int, C.c_int, C.c_int, C.POINTER(C.c_double), C.c_double,
                                   C.c_double, C.c_double]
    for tag, ch, src in (("comp", 0, 0), ("char_gravity", 1, 1)):
        nx, ny = 40, 20
        rows, cols = nx + 2 * GC, ny + 2 * GC
        pri = np.zeros((4, rows, cols)); U = np.zeros_like(pri)
        F = np.zeros_like(pri); G = np.zeros_like(pri)
        lx, ly, tm = C.c_double(), C.c_double(), C.c_double()
        ref.lib.ref_set_params(1.4, 0.5, 5, ch, src, 1.0)
        ref.lib.ref_init(20, rows, cols, _ptr(pri), _ptr(U), _ptr(F), _ptr(G), C.byref(lx),
                         C.byref(ly), C.byref(tm))
        U0 = U.copy()
        dx, dy = lx.value / nx, ly.value / ny
        dt = 0.1 * dx
        for _ in range(6):
            ref.lib.ref_rk1_bs(2, rows, cols, _ptr(U), dt, dx, dy)
        save(f"backward_step_{tag}_40x20_rk1bs", U0=U0, U=U, dt=dt, dx=dx, dy=dy,
             characteristic=ch, source=src)
        manifest[f"backward_step_{tag}_40x20_rk1bs"] = "RK1_TimeAd_BS, 6 steps"

    # 3. double Mach reflection with the exact boundary, 48 x 12: one step of
    #    characteristic WENO5-JS + HLLC, which goes non-finite in the reference
    #    (negative interface pressure at the wall next to the shock foot).  HLL
    #    is not used here: its skipped interfaces keep whatever the reference's
    #    reused flux buffer held, which the reference does not define.
    for tag, ch, wz, scheme, lib in [("charjs_hllc", 1, 0, 2, wjs)]:
        p = orc.params(48, 12, recon=5, characteristic=ch, weno_z=wz, cfl=0.4)
        U0, lx, ly, tmax = orc.init_case(p, DOUBLE_MACH)
        p.dmr = 1
        dx, dy = lx / 48, ly / 12
        U = U0.copy()
        dt = lib.dt(p, U, dx, dy)
        lib.rk(p, 3, scheme, U, dt, dx, dy, 0.0)
        save(f"dmr_{tag}_48x12_step1", U0=U0, U=U, dt=dt)
        manifest[f"dmr_{tag}_48x12_step1"] = "exact double-Mach boundary, one step"

    # 4. the precision test (Precision_test, src/RP_FVM.c:974-1072): RK3 +
    #    HLLC + component WENO5 with dt = 0.5 dx^(5/3) to t = 2
    lib = ref.lib
    prec = {}
    for nx in (10, 20, 40, 80):
        rows, cols = nx + 2 * GC, 1 + 2 * GC
        pri = np.zeros((4, rows, cols)); U = np.zeros_like(pri)
        F = np.zeros_like(pri); G = np.zeros_like(pri)
        lx, ly, tm = C.c_double(), C.c_double(), C.c_double()
        ref.lib.ref_set_params(1.4, 0.5, 5, 0, 0, 1.0)
        lib.ref_init(0, rows, cols, _ptr(pri), _ptr(U), _ptr(F), _ptr(G), C.byref(lx),
                     C.byref(ly), C.byref(tm))
        U0 = U.copy()
        dx, dy = lx.value / nx, ly.value / 1
        t = 0.0
        while t < tm.value:
            dt = 0.5 * dx ** (5.0 / 3)
            if t + dt >= tm.value:
                dt = tm.value - t
            lib.ref_rk(3, 2, rows, cols, _ptr(U), dt, dx, dy)
            t = t + dt
        xc = (np.arange(nx) + 0.5) * dx
        l1 = float(np.sum(np.abs(1.0 + 0.2 * np.sin(xc - t) - U[0, GC:-GC, GC])) * dx)
        prec[nx] = l1
        save(f"precision_nx{nx}", U0=U0, U=U, t_final=t)
    manifest["precision"] = {str(k): v for k, v in prec.items()}

    # 5. granular operators on a developed four-quadrant state, 20 x 16
    p = orc.params(20, 16, recon=5, characteristic=1, weno_z=1, cfl=0.5)
    U0, *_ = orc.init_case(p, FOUR_QUADRANT)
    dx, dy = 1.0 / 20, 1.0 / 16
    U, _ = ref_steps(ref, p, U0.copy(), 3, 2)
    rows, cols = U.shape[1:]
    ref.configure(p)
    Ub = U.copy()
    lib.ref_bc(rows, cols, _ptr(Ub))
    pri = np.zeros_like(U)
    lib.ref_con_to_pri(rows, cols, _ptr(pri), _ptr(Ub))
    out = dict(U=U, Ub=Ub, pri=pri, dt=ref.dt(p, U, dx, dy))
    for d in (1, 2):
        el = np.zeros((4, 4, rows, cols)); er = np.zeros_like(el)
        lib.ref_eigen(d, rows, cols, _ptr(pri), _ptr(el), _ptr(er))
        out[f"eig_l{d}"], out[f"eig_r{d}"] = el, er
        for tag, (recon, ch, wz, variant) in {"charz": (5, 1, 1, ref), "charjs": (5, 1, 0, wjs),
                                              "comp": (5, 0, 1, ref), "tvdc": (2, 1, 1, ref),
                                              "tvdm": (2, 0, 1, ref), "god": (1, 1, 1, ref),
                                              "w3c": (3, 1, 1, ref), "w3m": (3, 0, 1, ref)}.items():
            variant.lib.ref_set_params(1.4, 0.5, recon, ch, 0, 1.0)
            ql = np.zeros_like(U); qr = np.zeros_like(U)
            variant.lib.ref_recon(d, rows, cols, _ptr(Ub), _ptr(ql), _ptr(qr), dx, dy)
            out[f"ql_{tag}{d}"], out[f"qr_{tag}{d}"] = ql, qr
        ql, qr = out[f"ql_charz{d}"], out[f"qr_charz{d}"]
        for scheme in (1, 2, 3, 4, 11, 22, 33):
            fl = np.zeros_like(U)
            lib.ref_riemann(scheme, d, rows, cols, _ptr(ql), _ptr(qr), _ptr(fl))
            out[f"flux{scheme}_{d}"] = fl
    ref.lib.ref_set_params(1.4, 0.5, 5, 1, 0, 1.0)
    f = np.zeros_like(U); g = np.zeros_like(U)
    lib.ref_flux_recon(2, rows, cols, _ptr(Ub), _ptr(f), _ptr(g), 0.0, dx, dy)
    s = np.zeros_like(U); Lt = np.zeros_like(U)
    lib.ref_space_item(rows, cols, dx, dy, _ptr(f), _ptr(g), _ptr(s), _ptr(Lt))
    out.update(f=f, g=g, L=Lt)
    save("granular_20x16", **out)
    manifest["granular_20x16"] = "boundary, primitives, eigenvectors, reconstructions, fluxes"

    # 6. boundary kinds, including the mirrored/copied reflections and the
    #    exact double-Mach boundary, on a random state 12 x 10
    rng = np.random.default_rng(7)
    bcs = {}
    for kinds in [(REFLECT, REFLECT, REFLECT, REFLECT), (PERIODIC, PERIODIC, PERIODIC, PERIODIC),
                  (OUTFLOW, OUTFLOW, OUTFLOW, OUTFLOW), (INFLOW, OUTFLOW, REFLECT, REFLECT)]:
        p = orc.params(12, 10, bc=kinds)
        U = rng.uniform(0.5, 2.0, size=(4, 20, 18))
        Ub = U.copy()
        ref.configure(p)
        lib.ref_bc(20, 18, _ptr(Ub))
        bcs["bc_" + "".join(map(str, kinds))] = np.stack([U, Ub])
    U = rng.uniform(0.5, 2.0, size=(4, 20, 18))
    Ub = U.copy()
    lib.ref_bc_dmr(20, 18, _ptr(Ub), 0.05)
    bcs["bc_dmr_t0.05"] = np.stack([U, Ub])
    save("boundary_12x10", **bcs)
    manifest["boundary_12x10"] = "Boundary_Conditions per kind, BC_DoubleMach_2D at t=0.05"

    # 7. the reference's own initial states (Init_Euler_2D) on 16 x 12
    inits = {}
    # one thread: the 2D Noh initialiser draws rand() inside its OpenMP loop
    threads = ref.lib.ref_num_threads()
    ref.lib.ref_set_threads(1)
    for tc, (nx, ny) in {0: (16, 1), 1: (16, 12), 2: (16, 12), 3: (16, 12), 4: (16, 12),
                         5: (16, 12), 6: (16, 12), 7: (16, 12), 8: (16, 12), 9: (16, 12),
                         10: (16, 12), 11: (15, 13), 12: (16, 12), 13: (16, 12),
                         14: (16, 16), 15: (8, 24), 16: (24, 12), 17: (16, 16), 18: (16, 16),
                         19: (40, 8), 20: (24, 8)}.items():
        rows, cols = nx + 2 * GC, ny + 2 * GC
        pri = np.zeros((4, rows, cols)); U = np.zeros_like(pri)
        F = np.zeros_like(pri); G = np.zeros_like(pri)
        lx, ly, tm = C.c_double(), C.c_double(), C.c_double()
        ref.lib.ref_set_params(1.4, 0.5, 5, 0, 0, 1.0)
        lib.ref_init(tc, rows, cols, _ptr(pri), _ptr(U), _ptr(F), _ptr(G), C.byref(lx),
                     C.byref(ly), C.byref(tm))
        b = (C.c_int * 4)()
        lib.ref_get_bc(b)
        inits[f"case{tc}"] = U
        inits[f"case{tc}_meta"] = np.array([lx.value, ly.value, tm.value] + list(b))
    ref.lib.ref_set_threads(threads)
    save("init_cases", **inits)
    manifest["init_cases"] = "Init_Euler_2D of every TestCase2D value (0-20), one thread"

    # 8. control files parsed by the reference's ReadControlFile
    ctl = {}
    for fname in sorted(os.listdir(os.path.join(OUT, "controls"))):
        ints = (C.c_int * 10)()
        dbls = (C.c_double * 4)()
        outdir = C.create_string_buffer(256)
        lib.ref_read_control(os.path.join(OUT, "controls", fname).encode(), ints,
                             C.cast(dbls, C.POINTER(C.c_double)), outdir, 256)
        ctl[fname] = {"ints": list(ints), "dbls": list(dbls), "output_dir": outdir.value.decode()}
    with open(os.path.join(OUT, "controls.json"), "w") as fh:
        json.dump(ctl, fh, indent=1, sort_keys=True)
    manifest["controls"] = "ReadControlFile of tests/golden/controls/*"

    with open(os.path.join(OUT, "manifest.json"), "w") as fh:
        json.dump(manifest, fh, indent=1, sort_keys=True)


if __name__ == "__main__":
    main()
