"""Benchmark of the 2D Euler FVM step on B200.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Workload (one step = one SSP-RK3 step of the whole grid, CFL time step from the
device reduction): the four-quadrant Riemann problem on [0,1]^2, 1024 x 1024
cells, gamma 1.4, characteristic WENO5-JS + HLLC + SSP-RK3, CFL 0.5, plain
FP64 drop-in form (bit-identical to the reference).  Inputs are synthetic (the
benchmark's own initial state); nothing is downloaded.  Every timed window
starts from the state advanced, untimed, to t = 0.15 (mid-run: the quadrants'
waves have rolled up and few stencils are still uniform).

Our arm prints one JSON line with
  value     cell-updates/s over all ranks, device time (CUDA events) of K
            steps, max over ranks, L2 flushed between steps outside the timed
            intervals;
  e2e       the same metric through the reference-facing C-ABI calls with host
            buffers: per step upload of U from pinned host memory, CFL step,
            RK3 step, download of U (eb2_upload / eb2_delta_t / eb2_rk_step /
            eb2_download);
  roofline  algorithmic HBM bytes of the fused stage kernel (256 B per cell per
            RK3 step: 64 + 96 + 96) over its measured device time, against the
            measured copy bandwidth; beside it the counted FP64/FP32 operations
            per cell-stage against the same kernel's time;
  cpu_baseline  the reference built from its own sources (oracle/_ref), all
            host cores, on a bounded sample of the same workload;
  extra     (one GPU) whole runs to t = 0.3 and mid-run windows of the 1024^2
            and 4096^2 grids in the FP64 and mixed forms (HLLC; Roe), the
            mixed form's error against the FP64 form at every checkpoint with
            the FP32-sized floor of the flow itself, and the served stream of
            512 requests (batched mixed server against one-at-a-time mixed and
            one-at-a-time plain FP64 solves).
With --impl reference, rank 0 times the reference's CPU implementation on the
same workload and prints the reference line; other ranks exit.
For N > 1 (torchrun) every rank runs an independent replica (weak scaling):
a single solve of this size does not shard in this build.

--nx/--precision/--scheme/--no-e2e/--no-cpu-baseline/--no-extra select a single
measurement (used for profiling runs); --serve N runs only the served stream.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

ORDER = 3                     # SSP-RK3
SCHEMES = {"hllc": 2, "roe": 3, "hll": 1, "llf": 4}
BYTES_PER_CELL_STEP = 256     # 64 + 96 + 96 algorithmic HBM bytes (FP64 state)
FLUSH_BYTES = 256 << 20       # > 126 MB L2
METRIC = "cell-updates/s"
FALLBACK_HBM_GBS = 6650.0


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=500)
    ap.add_argument("--warmup", type=int, default=10)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--nx", type=int, default=1024)
    ap.add_argument("--precision", choices=["fp64", "mixed"], default="fp64")
    ap.add_argument("--scheme", choices=sorted(SCHEMES), default="hllc")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-extra", action="store_true")
    ap.add_argument("--serve", type=int, default=None, metavar="N",
                    help="served stream of N requests only (batched vs one-at-a-time)")
    ap.add_argument("--serve-rate", type=float, default=20.0)
    ap.add_argument("--serve-requests", type=int, default=512,
                    help="requests of the served stream in the default line (0: none)")
    ap.add_argument("--dmr", action="store_true",
                    help="double Mach reflection 1920x480 to t = 0.2, FP64 and mixed")
    ap.add_argument("--accuracy", type=float, default=None, metavar="T",
                    help="run the FP64 and mixed forms to time T and print their difference")
    return ap.parse_args()


def stream_trace(n, rate, seed, eb2):
    """The served stream: n requests arriving Poisson at `rate` per second;
    each a four-quadrant problem with per-quadrant rho ~ U[0.1,2],
    p ~ U[0.05,2], u, v ~ U[-1.5,1.5] (positive by construction), or a
    wall-heating problem with inflow speed ~ U[0.5,2] on the unit square
    (periodic in y, so dx = dy); square grids from {128,256,512,1024}, final
    time ~ U[0.1,0.3]."""
    import numpy as np

    from overheatingproblem_b200.server import Request
    rng = np.random.default_rng(seed)
    arrivals = np.cumsum(rng.exponential(1.0 / rate, size=n))
    arrivals -= arrivals[0]
    reqs = []
    for _ in range(n):
        size = int(rng.choice([128, 256, 512, 1024]))
        tmax = float(rng.uniform(0.1, 0.3))
        if rng.random() < 0.5:
            q = []
            for _ in range(4):
                q += [rng.uniform(0.1, 2.0), rng.uniform(-1.5, 1.5), rng.uniform(-1.5, 1.5),
                      rng.uniform(0.05, 2.0)]
            reqs.append(Request(eb2.lib.CASE_FOUR_QUADRANT, size, size, q=q, tmax=tmax))
        else:
            reqs.append(Request(eb2.lib.CASE_WALL_HEATING, size, size,
                                q=[float(rng.uniform(0.5, 2.0))], ly=1.0, tmax=tmax))
    return reqs, arrivals


def one_at_a_time(eb2, local, reqs, arr, precision, sample):
    """Each request on its own context, started when it has arrived and the
    previous one has finished (one solve on the GPU at a time); the final
    states of the `sample` requests are kept."""
    import numpy as np
    t0 = time.perf_counter()
    fin = np.zeros(len(reqs))
    status = np.zeros(len(reqs), dtype=np.uint32)
    kept = {}
    for i, r in enumerate(reqs):
        wait = arr[i] - (time.perf_counter() - t0)
        if wait > 0:
            time.sleep(wait)
        with eb2.Solver(r.nx, r.ny, device=local, recon=5, characteristic=True, weno_z=False,
                        cfl=r.cfl, precision=precision) as s:
            lx, ly, _ = s.init_case(r.test_case, r.q)
            ly = r.ly if r.ly > 0 else ly
            s.run(ORDER, 2, lx / r.nx, ly / r.ny, r.tmax)
            U = s.download()
            status[i] = s.status()
        if i in sample:
            kept[i] = U
        fin[i] = time.perf_counter() - t0
    return fin, status, kept


def arm_summary(n, makespan, lat, status):
    import numpy as np
    bad = [int(i) for i in np.nonzero(status)[0]]
    return {"solves_per_s": n / makespan, "makespan_s": float(makespan),
            "p50_latency_s": float(np.percentile(lat, 50)),
            "p99_latency_s": float(np.percentile(lat, 99)), "requests": n,
            "non_physical": len(bad), "non_physical_ids": bad,
            "physical_solves_per_s": (n - len(bad)) / makespan}


def serve_stream(eb2, local, n, rate, seed, reps=1, nsample=16):
    """The batched mixed-precision server against one-at-a-time mixed and
    one-at-a-time plain FP64 solves on the same trace: solves/s (all, and the
    solves that stayed physical), latency percentiles (finish - arrival), the
    requests that went non-physical by id, and the density error of the
    server's results against the one-at-a-time FP64 results on a sample of
    requests."""
    import numpy as np

    from overheatingproblem_b200.server import Server
    reqs, arr = stream_trace(n, rate, seed, eb2)
    sample = set(range(0, n, max(1, n // nsample)))
    # The trace is replayed in real time, so how requests meet in batches (and
    # the rate) varies from replay to replay; with reps > 1 the median replay
    # is reported and all are listed.
    runs = []
    with Server(device=local, precision=eb2.lib.MIXED, scheme=2,
                hbm_budget=120 * 10**9) as srv:
        for _ in range(reps):
            t0 = srv.timing()
            runs.append(srv.run_trace(reqs, arr, keep_results=sample))
            t1 = srv.timing()
            runs[-1]["timing"] = {k: t1[k] - t0[k] for k in t1}
    order = sorted(range(reps), key=lambda k: runs[k]["makespan"])
    out = runs[order[len(order) // 2]]
    batched = arm_summary(n, out["makespan"], out["finish"] - arr, out["status"])
    batched["steps"] = int(out["steps"].sum())
    batched["gpu_busy_frac"] = out["timing"]["busy_s"] / out["makespan"]
    batched["host_autotune_s"] = out["timing"]["tune_s"]
    batched["host_admin_s"] = out["timing"]["admin_s"]
    batched["replays_solves_per_s"] = [n / o["makespan"] for o in runs]
    fin_m, st_m, _ = one_at_a_time(eb2, local, reqs, arr, eb2.lib.MIXED, set())
    mixed1 = arm_summary(n, fin_m[-1], fin_m - arr, st_m)
    fin_d, st_d, kept = one_at_a_time(eb2, local, reqs, arr, eb2.lib.FP64, sample)
    fp641 = arm_summary(n, fin_d[-1], fin_d - arr, st_d)
    err = []
    for i in sorted(sample):
        if st_d[i] or out["status"][i]:
            continue
        a = kept[i][0, 4:-4, 4:-4]
        b = out["results"][i][0, 4:-4, 4:-4]
        d = np.abs(a - b)
        err.append({"request": i, "n": reqs[i].nx, "t_final": reqs[i].tmax,
                    "l1_rho": float(d.mean()), "linf_rho": float(d.max()),
                    "rel_l1_rho": float(d.sum() / np.abs(a).sum())})
    acc = {"vs": "one-at-a-time FP64 results of the same requests (density; L1 = mean "
                 "|d rho| over the cells, Linf = max)",
           "sample": err,
           "max_l1_rho": max((e["l1_rho"] for e in err), default=None),
           "median_l1_rho": float(np.median([e["l1_rho"] for e in err])) if err else None}
    return {"trace": f"{n} requests, Poisson arrivals at {rate}/s, seed {seed}",
            "batched_mixed": batched, "one_at_a_time_mixed": mixed1,
            "one_at_a_time_fp64": fp641,
            "speedup_solves_per_s": batched["solves_per_s"] / fp641["solves_per_s"],
            "speedup_vs_one_at_a_time_mixed": batched["solves_per_s"] / mixed1["solves_per_s"],
            "accuracy": acc}


MARKS = (0.05, 0.1, 0.15, 0.2, 0.25, 0.3)   # checkpoints of the whole runs
T_START = 0.15                               # every timed window starts here
L1_BOUND = 1e-6                              # the density L1 bound of the mixed form


def four_quadrant(eb2, local, n, precision):
    prec = eb2.lib.FP64 if precision == "fp64" else eb2.lib.MIXED
    s = eb2.Solver(n, n, device=local, recon=5, characteristic=True, weno_z=False, cfl=0.5,
                   precision=prec)
    lx, ly, _ = s.init_case(eb2.lib.CASE_FOUR_QUADRANT)
    return s, lx / n, ly / n


def fp32_perturbation(seed):
    """Every interior value of the initial state moved by a seeded relative
    2^-24 up or down: rounding of FP32 size applied everywhere once."""
    import numpy as np

    def apply(U):
        rng = np.random.default_rng(seed)
        inner = U[:, 4:-4, 4:-4]
        inner *= 1.0 + rng.choice([-1.0, 1.0], size=inner.shape) * 2.0 ** -24
    return apply


def whole_run(eb2, local, n, precision, scheme, marks=MARKS, perturb=None, save_at=None):
    """The four-quadrant problem run to marks[-1] by the device time loop
    (eb2_run), paused at every mark (the CFL step is clipped there, in every
    run alike) to record the density; the final primitives; the conserved
    state at `save_at`.  Seconds are those of the device loop segments."""
    s, dx, dy = four_quadrant(eb2, local, n, precision)
    if perturb is not None:
        U = s.download()
        perturb(U)
        s.upload(U)
    t, steps, el, rho, saved, pri = 0.0, 0, 0.0, [], None, None
    for tm in marks:
        t0 = time.perf_counter()
        k, t = s.run(ORDER, scheme, dx, dy, tm, t0=t)
        el += time.perf_counter() - t0
        steps += k
        pri = s.con_to_pri()
        rho.append(pri[0, 4:-4, 4:-4].copy())
        if save_at is not None and abs(tm - save_at) < 1e-12:
            saved = s.download()
    info = {"steps": steps, "t_final": t, "seconds": el, "status_flags": s.status(),
            "cell_updates_per_s": n * n * steps / el}
    return s, dx, dy, info, rho, pri[:, 4:-4, 4:-4].copy(), saved


def compare(ref, got, marks=MARKS):
    """Differences of a run against the reference run (FP64): density L1
    (mean |d rho| over the cells, i.e. dx dy sum |d rho| on the unit square,
    the norm of include/Error.h:129-160) and Linf at every checkpoint, all
    four primitives at the final time, and the last checkpoint up to which
    the density L1 stays within 1e-6."""
    import numpy as np
    (rho_a, fin_a), (rho_b, fin_b) = ref, got
    cps = []
    for tm, a, b in zip(marks, rho_a, rho_b):
        d = np.abs(a - b)
        cps.append({"t": tm, "l1_rho": float(d.mean()), "linf_rho": float(d.max())})
    last = None
    for c in cps:
        if c["l1_rho"] > L1_BOUND:
            break
        last = c["t"]
    d = np.abs(fin_a - fin_b)
    names = ["rho", "u", "v", "p"]
    return {"t_final": marks[-1], "l1": {q: float(d[i].mean()) for i, q in enumerate(names)},
            "linf": {q: float(d[i].max()) for i, q in enumerate(names)},
            "rel_l1_rho": float(d[0].sum() / np.abs(fin_a[0]).sum()), "checkpoints": cps,
            "last_t_with_l1_rho_le_1e-6": last}


def window(s, state, scheme, dx, dy, k, warmup=2):
    """Device time of k steps from `state` (L2 flushed between steps), after
    `warmup` untimed steps from the same state."""
    s.upload(state)
    if warmup:
        s.bench_steps(ORDER, scheme, dx, dy, warmup, 0)
        s.upload(state)
    step_ms, stage_ms, nstage, launches = s.bench_steps(ORDER, scheme, dx, dy, k, FLUSH_BYTES)
    return step_ms, stage_ms, nstage, launches, s.status()


def window_entry(n, k, step_ms, stage_ms, nstage, st, peak, whole=None):
    tot = float(sum(step_ms))
    e = {"value": n * n * k / (tot * 1e-3), "unit": METRIC, "ms_per_step": tot / k, "steps": k,
         "start": f"t = {T_START} (advanced untimed), L2 flushed between steps",
         "status_flags": st,
         "roofline_frac": n * n * BYTES_PER_CELL_STEP * k / (stage_ms * 1e-3) / 1e9 / peak,
         "step_roofline_frac": n * n * BYTES_PER_CELL_STEP * k / (tot * 1e-3) / 1e9 / peak,
         "stage_ms": stage_ms / nstage}
    if whole is not None:
        e["whole_run"] = whole
    return e


def short_accuracy(acc):
    return {"vs": "FP64 form", "t_final": acc["t_final"], "l1_rho": acc["l1"]["rho"],
            "linf_rho": acc["linf"]["rho"], "rel_l1_rho": acc["rel_l1_rho"],
            "last_t_with_l1_rho_le_1e-6": acc["last_t_with_l1_rho_le_1e-6"]}


def run_extras(eb2, local, peak, rate, nserve, extra, acc):
    """Whole runs, mid-run windows, accuracy and the served stream (one GPU),
    filled into `extra` and `acc` as each is measured."""
    # 1024^2: FP64 and mixed whole runs (HLLC, Roe), the FP32-sized floor
    for name, sch in (("hllc", 2), ("roe", 3)):
        s64, dx, dy, i64, r64, f64, _ = whole_run(eb2, local, 1024, "fp64", sch)
        s64.close()
        sm, dx, dy, im, rm, fm, um = whole_run(eb2, local, 1024, "mixed", sch, save_at=T_START)
        a = compare((r64, f64), (rm, fm))
        if sch == 2:
            extra["fp64_1024_hllc_whole_run"] = i64
            w = window(sm, um, sch, dx, dy, 200)
            extra["mixed_1024_hllc"] = window_entry(1024, 200, *w[:3], w[4], peak, im)
            extra["mixed_1024_hllc"]["accuracy"] = short_accuracy(a)
            sp, _, _, ip, rp, fp, _ = whole_run(eb2, local, 1024, "fp64", sch,
                                                perturb=fp32_perturbation(11))
            sp.close()
            a["floor_fp32_perturbed_fp64"] = compare((r64, f64), (rp, fp))["checkpoints"]
        else:
            extra["mixed_1024_roe_whole_run"] = im
            extra["mixed_1024_roe_whole_run"]["accuracy"] = short_accuracy(a)
        acc[f"four_quadrant_1024_{name}"] = a
        sm.close()
    # 4096^2: the FP64 HLLC run is the accuracy reference of the mixed HLLC run
    s64, dx, dy, i64, r64, f64, u64 = whole_run(eb2, local, 4096, "fp64", 2, save_at=T_START)
    w = window(s64, u64, 2, dx, dy, 10)
    extra["fp64_4096_hllc"] = window_entry(4096, 10, *w[:3], w[4], peak, i64)
    s64.close()
    del u64
    for name, sch in (("hllc", 2), ("roe", 3)):
        sm, dx, dy, im, rm, fm, um = whole_run(eb2, local, 4096, "mixed", sch, save_at=T_START)
        w = window(sm, um, sch, dx, dy, 40)
        extra[f"mixed_4096_{name}"] = window_entry(4096, 40, *w[:3], w[4], peak, im)
        if sch == 2:
            a = compare((r64, f64), (rm, fm))
            acc["four_quadrant_4096_hllc"] = a
            extra["mixed_4096_hllc"]["accuracy"] = short_accuracy(a)
        else:
            extra["mixed_4096_roe"]["accuracy"] = dict(
                short_accuracy(acc["four_quadrant_1024_roe"]),
                note="measured at 1024^2 (four_quadrant_1024_roe): an FP64 Roe run at 4096^2 "
                     "would add three minutes")
        sm.close()
        del um, rm, fm
    del r64, f64
    if nserve:
        extra["served_stream"] = serve_stream(eb2, local, nserve, rate, 7)


def run_accuracy(args, local):
    """FP64 vs mixed on the benchmark problem up to t = T with checkpoints,
    and the FP64 run from an initial state perturbed by a relative 2^-24 in
    every value (the floor the flow's own amplification sets for any
    arithmetic of FP32 size)."""
    import overheatingproblem_b200 as eb2

    nx, scheme, T = args.nx, SCHEMES[args.scheme], args.accuracy
    marks = tuple(t for t in MARKS if t < T) + (T,)
    runs, res = {}, {}
    for name, prec, pert in (("fp64", "fp64", None), ("mixed", "mixed", None),
                             ("fp64_fp32_floor", "fp64", fp32_perturbation(11))):
        s, _, _, info, rho, fin, _ = whole_run(eb2, local, nx, prec, scheme, marks, pert)
        s.close()
        runs[name] = info
        res[name] = (rho, fin)
    line = {"accuracy": workload(nx, "mixed", args.scheme) + f" vs FP64, t = {T}",
            "mixed_vs_fp64": compare(res["fp64"], res["mixed"], marks),
            "fp32_floor_vs_fp64": compare(res["fp64"], res["fp64_fp32_floor"], marks),
            "note": "checkpoint times clip the CFL step in all three runs alike",
            "runs": runs}
    print(json.dumps(line), flush=True)


def run_dmr(args, local):
    """Double Mach reflection on [0,4]x[0,1], 1920x480, Mach-10 shock at 60
    degrees, exact moving-shock top boundary, characteristic WENO5-JS + HLLC +
    SSP-RK3, CFL 0.4, t = 0.2, in the FP64 and the mixed form.  The
    reference's scheme reconstructs a negative pressure on the first step of
    this problem, so both runs use the first-order fallback at such
    interfaces.  Reports the mixed-vs-FP64 density error and the temperature
    T = p / rho along the reflecting wall (first cell row, x > 1/6)."""
    import numpy as np

    import overheatingproblem_b200 as eb2

    nx, ny = 1920, 480
    out, prim = {}, {}
    for name, prec in (("fp64", eb2.lib.FP64), ("mixed", eb2.lib.MIXED)):
        s = eb2.Solver(nx, ny, device=local, recon=5, characteristic=True, weno_z=False,
                       cfl=0.4, precision=prec)
        lx, ly, tmax = s.init_case(eb2.lib.CASE_DOUBLE_MACH)
        s.set_double_mach(True)
        s.set_positivity_fallback(True)
        t0 = time.perf_counter()
        n, tf = s.run(ORDER, 2, lx / nx, ly / ny, tmax)
        el = time.perf_counter() - t0
        prim[name] = s.con_to_pri()[:, 4:-4, 4:-4].copy()
        out[name] = {"steps": n, "t_final": tf, "seconds": el, "status_flags": s.status(),
                     "cell_updates_per_s": nx * ny * n / el}
        s.close()
    x = (np.arange(nx) + 0.5) * 4.0 / nx
    wall = x > 1.0 / 6.0

    def wall_temperature(p):
        # overshoot: the hottest wall cell against the hottest cell of rows
        # 4-12 above the wall, over the same stretch of wall
        T = p[3] / p[0]
        tw = T[wall, 0]
        above = float(T[wall, 4:12].max())
        return {"max": float(tw.max()), "mean": float(tw.mean()),
                "x_of_max": float(x[wall][int(np.argmax(tw))]), "max_rows_4_to_12": above,
                "overshoot": float(tw.max() / above - 1.0)}

    d = np.abs(prim["fp64"] - prim["mixed"])
    tw64 = prim["fp64"][3][wall, 0] / prim["fp64"][0][wall, 0]
    twm = prim["mixed"][3][wall, 0] / prim["mixed"][0][wall, 0]
    line = {"dmr": "double Mach reflection 1920x480, characteristic WENO5-JS + HLLC + SSP-RK3, "
                   "CFL 0.4, t = 0.2, exact moving-shock boundary, positivity fallback on",
            "l1": {"rho": float(d[0].mean()), "p": float(d[3].mean())},
            "linf": {"rho": float(d[0].max()), "p": float(d[3].max())},
            "rel_l1_rho": float(d[0].sum() / np.abs(prim["fp64"][0]).sum()),
            "wall_temperature": {"fp64": wall_temperature(prim["fp64"]),
                                 "mixed": wall_temperature(prim["mixed"]),
                                 "l1_mixed_vs_fp64": float(np.abs(tw64 - twm).mean()),
                                 "linf_mixed_vs_fp64": float(np.abs(tw64 - twm).max())},
            "runs": out}
    print(json.dumps(line), flush=True)


def workload(nx, precision, scheme):
    return (f"four-quadrant Riemann {nx}x{nx}, characteristic WENO5-JS + {scheme.upper()} + "
            f"SSP-RK3, {'FP64' if precision == 'fp64' else 'mixed FP32/FP64'}")


def config(args):
    return {"workload": workload(args.nx, args.precision, args.scheme), "nx": args.nx,
            "ny": args.nx, "order": ORDER, "scheme": args.scheme.upper(),
            "reconstruction": "WENO5-JS characteristic", "cfl": 0.5,
            "precision": args.precision,
            "window_start": f"t = {T_START}, advanced untimed from the initial state",
            "l2": "flushed between timed steps (256 MiB write outside the timed intervals)",
            "parallelism": "replicas"}


def measured_traffic(nx, precision, scheme):
    """DRAM bytes (read + write) per fused-stage launch of this workload, from
    the committed ncu summary profiles/traffic_<precision>_<nx>.md (taken with
    the same bench command), or None when there is none."""
    path = os.path.join(ROOT, "profiles", f"traffic_{precision}_{nx}.md")
    if scheme != "hllc" or not os.path.exists(path):
        return None
    for line in open(path):
        cells = [c.strip() for c in line.strip().strip("|").split("|")]
        if line.startswith("|") and cells[0] == "traffic per launch":
            return float(cells[1].split()[0]) * 1e6
    return None


def profile_rows(precision):
    """Rows of the committed ncu summary profiles/stage_<precision>_2048.md as
    {metric: value of its "now" column}."""
    path = os.path.join(ROOT, "profiles", f"stage_{precision}_2048.md")
    rows, col = {}, None
    if not os.path.exists(path):
        return rows
    for line in open(path):
        if not line.startswith("|"):
            continue
        cells = [c.strip() for c in line.strip().strip("|").split("|")]
        if cells[0] == "metric":
            col = next((i for i, c in enumerate(cells)
                        if c.startswith("now") or "(now)" in c or c == "value"), None)
        elif col is not None and len(cells) > col:
            rows[cells[0]] = cells[col]
    return rows


def gemm_tflops(local, dtype, n):
    """Measured dense GEMM rate (cuBLAS through torch, TF32 off) of `dtype` on
    this GPU: the compute peak the stage kernel's counted operations are set
    against."""
    import torch
    torch.backends.cuda.matmul.allow_tf32 = False
    dev = f"cuda:{local}"
    a = torch.randn(n, n, dtype=dtype, device=dev)
    b = torch.randn(n, n, dtype=dtype, device=dev)
    for _ in range(2):
        a @ b
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(5):
        a @ b
    e1.record()
    e1.synchronize()
    return 5 * 2 * n ** 3 / (e0.elapsed_time(e1) * 1e-3) / 1e12


def measured_compute(precision, cells, per_launch_ms, local):
    """The stage kernel against its on-chip limits: the binding pipe from the
    committed ncu summary (FP64 pipe for the FP64 form, instruction issue for
    the mixed form), and the arithmetic per cell-stage counted there by ncu
    (DADD/DMUL/DFMA and FADD/FMUL/FFMA plus the packed FADD2/FMUL2/FFMA2; an
    FMA counts two operations, a packed instruction two lanes) over the live
    per-launch time, against a measured GEMM rate of the same precision."""
    rows = profile_rows(precision)
    row = "FP64 pipe active" if precision == "fp64" else "issue active"
    out = {"limit": "fp64 pipe" if precision == "fp64" else "instruction issue",
           "source": f"profiles/stage_{precision}_2048.md (ncu, 2048^2 stage)"}
    key = next((k for k in rows if k.startswith(row)), None)
    try:
        out["active_frac"] = float(rows[key].split()[0]) / 100.0 if key else None
    except ValueError:
        out["active_frac"] = None
    for prec, dt, n in (("fp64", "float64", 8192), ("fp32", "float32", 8192)):
        k = next((r for r in rows if r.startswith(f"{prec} operations per cell-stage")), None)
        if k is None:
            continue
        try:
            ops = float(rows[k].split()[0])
        except ValueError:
            continue
        achieved = ops * cells / (per_launch_ms * 1e-3) / 1e12
        entry = {"ops_per_cell_stage": ops, "achieved_tflops": achieved}
        if local is not None:
            import torch
            peak = gemm_tflops(local, getattr(torch, dt), n)
            entry.update(peak_tflops=peak, peak_kind=f"measured: cuBLAS {prec.upper()} GEMM "
                         f"{n}^3 on this GPU", frac=achieved / peak)
        out[prec] = entry
    return out


def hbm_peak():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(p) as fh:
            return float(json.load(fh)["hbm_gbs"]), "measured"
    except (OSError, KeyError, ValueError):
        return FALLBACK_HBM_GBS, "fallback"


# --------------------------------------------------------------------------- clocks
class ClockSampler:
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.path = tempfile.mktemp(suffix=".csv")
        self.proc = None
        try:
            self.fh = open(self.path, "w")
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "100", "-i", str(gpu_index)], stdout=self.fh, stderr=subprocess.DEVNULL)
        except OSError:
            self.proc = None

    def stop(self):
        if self.proc is None:
            return None
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        self.fh.close()
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        with open(self.path) as fh:
            for line in fh:
                f = [x.strip() for x in line.split(",")]
                if len(f) < 9:
                    continue
                try:
                    sm.append(float(f[1]))
                    smax = float(f[2])
                except ValueError:
                    continue
                for n, v in zip(names, f[5:9]):
                    if v.lower() == "active":
                        reasons.add(n)
        os.unlink(self.path)
        if not sm:
            return None
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": smax, "samples": len(sm),
                "reasons": sorted(reasons)}


# --------------------------------------------------------------------------- dist
def dist_setup(collective=True, backend="nccl"):
    """One process per GPU: rank, world size and local rank from the launcher's
    environment; a process group (NCCL on GPUs, gloo for CPU checks) only when
    the ranks exchange timings.  The short timeout ends ranks that wait for one
    another with an error instead of a hang."""
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1 and collective:
        import datetime

        import torch
        import torch.distributed as dist
        if backend == "nccl":
            torch.cuda.set_device(local)
        dist.init_process_group(backend, timeout=datetime.timedelta(seconds=180))
    return world, rank, local


def allreduce_max(x: float, world: int) -> float:
    """Max over ranks (the whole job's device time is the slowest rank's)."""
    if world == 1:
        return x
    import torch
    import torch.distributed as dist
    dev = "cuda" if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor([x], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def barrier(world):
    if world > 1:
        import torch.distributed as dist
        dist.barrier()


def physical_gpu(local: int) -> int:
    vis = os.environ.get("CUDA_VISIBLE_DEVICES")
    if vis:
        ids = [v for v in vis.split(",") if v.strip()]
        if local < len(ids) and ids[local].strip().isdigit():
            return int(ids[local])
    return local


# --------------------------------------------------------------------------- CPU
def reference_lib():
    """The reference built from its own sources, else the oracle port."""
    os.environ.setdefault("OMP_NUM_THREADS", str(os.cpu_count() or 1))
    os.environ.setdefault("OMP_PROC_BIND", "true")
    from oracle.bind import Oracle, Reference
    if Reference.available("wjs"):
        return Reference("wjs"), "reference"
    return Oracle(), "port"


def cpu_rate(nx: int, scheme: int, budget_s: float, max_steps: int, warmup: int):
    """Cell-updates/s of the CPU implementation on the benchmark workload:
    full nx^2 RK3 steps until the time budget is spent."""
    from oracle.bind import FOUR_QUADRANT, Oracle
    lib, kind = reference_lib()
    orc = Oracle()
    p = orc.params(nx, nx, recon=5, characteristic=1, weno_z=0, cfl=0.5)
    U, lx, ly, _ = orc.init_case(p, FOUR_QUADRANT)
    dx, dy = lx / nx, ly / nx
    for _ in range(warmup):
        lib.rk(p, ORDER, scheme, U, lib.dt(p, U, dx, dy), dx, dy)
    n, t0 = 0, time.perf_counter()
    while n < max(1, max_steps):
        dt = lib.dt(p, U, dx, dy)
        lib.rk(p, ORDER, scheme, U, dt, dx, dy)
        n += 1
        if time.perf_counter() - t0 > budget_s:
            break
    el = time.perf_counter() - t0
    cores = int(os.environ.get("OMP_NUM_THREADS", os.cpu_count() or 1))
    return nx * nx * n / el, el / n, n, kind, cores


def run_reference(args, world, rank):
    if rank != 0:
        return
    # bounded: at most ~150 s of timed CPU work whatever K is
    warm = min(args.warmup, 3)
    rate, per_step, n, kind, cores = cpu_rate(args.nx, SCHEMES[args.scheme], 150.0, args.steps,
                                              warm)
    cfg = config(args)
    # The reference's CPU step has no shortcut for uniform regions, so its cost
    # does not depend on the state: after warm-up a 256^2 step took 34.5 ms at
    # t = 0 and 34.1 ms at t = 0.15.  Its steps are timed from the initial state
    # (advancing it to t = 0.15 on the CPU would take minutes).
    cfg["window_start"] = ("t = 0 (the reference CPU path costs the same per step at any t; "
                           "its steps are timed from the initial state)")
    line = {
        "metric": METRIC, "value": rate, "unit": "cell-updates/s", "n_gpus": args.gpus,
        "steps": n, "warmup": warm, "ms_per_step": per_step * 1e3,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic", "config": cfg, "impl": "reference",
        "cpu_baseline": {"value": rate, "unit": "cell-updates/s", "cores": cores, "kind": kind,
                         "sample": f"{n} full SSP-RK3 steps of the {args.nx}^2 grid"},
        "e2e": {"value": rate, "unit": "cell-updates/s", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


# --------------------------------------------------------------------------- GPU
def run_ours(args, world, rank, local):
    import numpy as np
    import torch

    import overheatingproblem_b200 as eb2

    nx, scheme = args.nx, SCHEMES[args.scheme]
    torch.cuda.init()
    # the state at t = T_START, advanced untimed; every step below starts there
    s, dx, dy = four_quadrant(eb2, local, nx, args.precision)
    s.run(ORDER, scheme, dx, dy, T_START)
    state = s.download()
    torch.cuda.synchronize(local)
    # clocks are sampled from the warm-up (at least ~1 s of steps, so that the
    # sampler sees the GPU under load) through the timed steps
    sampler = ClockSampler(physical_gpu(local)) if rank == 0 else None
    t_w = time.perf_counter()
    nw = 0
    while nw < max(args.warmup, 3) or time.perf_counter() - t_w < 1.0:
        s.upload(state)
        s.bench_steps(ORDER, scheme, dx, dy, max(args.warmup, 3), 0)
        nw += max(args.warmup, 3)
    s.upload(state)
    torch.cuda.synchronize(local)
    barrier(world)
    torch.cuda.synchronize(local)
    # the NVTX range names the timed steps for profilers (ncu --nvtx-include)
    torch.cuda.nvtx.range_push("timed_steps")
    step_ms, stage_ms, nstage, launches = s.bench_steps(ORDER, scheme, dx, dy, args.steps,
                                                         FLUSH_BYTES)
    torch.cuda.nvtx.range_pop()
    st = s.status()
    torch.cuda.synchronize(local)
    barrier(world)
    clocks = sampler.stop() if sampler else None
    total_ms = allreduce_max(float(sum(step_ms)), world)
    value = world * nx * nx * args.steps / (total_ms * 1e-3)

    peak, peak_kind = hbm_peak()
    alg_bytes = nx * nx * BYTES_PER_CELL_STEP * args.steps
    achieved = alg_bytes / (stage_ms * 1e-3) / 1e9
    roofline = {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                "frac": achieved / peak,
                "traffic": measured_traffic(nx, args.precision, args.scheme),
                "traffic_source": "ncu dram__bytes_read.sum + dram__bytes_write.sum per launch",
                "kernel": f"eb2 fused x+y sweep + RK stage ({args.precision})",
                "per_launch_ms": stage_ms / nstage, "peak_kind": peak_kind,
                "alg_bytes_per_launch": nx * nx * BYTES_PER_CELL_STEP / ORDER,
                "stage_share_of_step": stage_ms / sum(step_ms),
                "compute": measured_compute(args.precision, nx * nx, stage_ms / nstage,
                                            local if rank == 0 else None)}

    e2e = None
    if not args.no_e2e:
        host = torch.empty((4, nx + 8, nx + 8), dtype=torch.float64, pin_memory=True).numpy()
        host[...] = state
        k_e2e = max(3, min(args.steps, 50))
        for _ in range(2):
            s.upload(host)
            s.rk_step(ORDER, scheme, s.delta_t(dx, dy), dx, dy)
            s.download(host)
        host[...] = state
        barrier(world)
        t0 = time.perf_counter()
        for _ in range(k_e2e):
            s.upload(host)
            dt = s.delta_t(dx, dy)
            s.rk_step(ORDER, scheme, dt, dx, dy)
            s.download(host)
        e2e_s = allreduce_max(time.perf_counter() - t0, world)
        e2e = {"value": world * nx * nx * k_e2e / e2e_s, "unit": "cell-updates/s",
               "h2d_bytes_per_step": int(host.nbytes), "d2h_bytes_per_step": int(host.nbytes) + 8,
               "steps": k_e2e, "timer": "host wall clock, max over ranks",
               "start": f"t = {T_START}",
               "path": "eb2_upload + eb2_delta_t + eb2_rk_step + eb2_download"}
    s.close()

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        rate, per_step, n, kind, cores = cpu_rate(nx, scheme, 20.0, 40, 3)
        cpu = {"value": rate, "unit": "cell-updates/s", "cores": cores, "kind": kind,
               "sample": f"{n} full SSP-RK3 steps of the {nx}^2 grid ({per_step:.3f} s each)"}
    extra, accuracy = {}, {}
    line = None
    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": "cell-updates/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": total_ms / args.steps, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic", "config": config(args),
            "e2e": e2e, "roofline": roofline, "cpu_baseline": cpu, "clocks": clocks,
            "gpu_launches": launches, "status_flags": st,
            "step_ms_min_median_max": [min(step_ms), float(np.median(step_ms)), max(step_ms)],
            "extra": extra,
        }
    if line is not None and not args.no_extra and world == 1:
        # The extras take minutes.  If the run is stopped by SIGTERM meanwhile,
        # the line is printed with the extras measured so far.
        import signal

        def stop(signum, frame):
            line["extra_incomplete"] = "stopped by signal %d during the extras" % signum
            if accuracy:
                line["accuracy"] = accuracy
            print(json.dumps(line), flush=True)
            os._exit(0)
        signal.signal(signal.SIGTERM, stop)
        run_extras(eb2, local, peak, args.serve_rate, args.serve_requests, extra, accuracy)
        signal.signal(signal.SIGTERM, signal.SIG_DFL)
    if line is not None:
        if accuracy:
            line["accuracy"] = accuracy
        print(json.dumps(line), flush=True)


def main():
    args = parse()
    # the reference arm uses no collective: rank 0 works, the others leave
    world, rank, local = dist_setup(collective=args.impl == "ours")
    try:
        if args.accuracy is not None:
            if rank == 0:
                run_accuracy(args, local)
        elif args.dmr:
            if rank == 0:
                run_dmr(args, local)
        elif args.serve is not None:
            if rank == 0:
                import overheatingproblem_b200 as eb2
                print(json.dumps(serve_stream(eb2, local, args.serve, args.serve_rate, 7)),
                      flush=True)
        elif args.impl == "reference":
            run_reference(args, world, rank)
        else:
            run_ours(args, world, rank, local)
    finally:
        if world > 1 and args.impl == "ours":
            import torch.distributed as dist
            dist.destroy_process_group()


if __name__ == "__main__":
    main()
