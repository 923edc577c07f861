"""Benchmark of the 2D Euler FVM step on B200.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Workload (one step = one SSP-RK3 step of the whole grid, CFL time step from the
device reduction): the four-quadrant Riemann problem on [0,1]^2, 1024 x 1024
cells, gamma 1.4, characteristic WENO5-JS + HLLC + SSP-RK3, CFL 0.5, plain
FP64 drop-in form (bit-identical to the reference).  Inputs are synthetic (the
benchmark's own initial state); nothing is downloaded.

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
            measured copy bandwidth;
  cpu_baseline  the reference built from its own sources (oracle/_ref), all
            host cores, on a bounded sample of the same workload;
  extra     the same device-time measurement for the 4096^2 grid in the FP64
            and mixed-precision forms (HLLC and Roe).
With --impl reference, rank 0 times the reference's CPU implementation on the
same workload and prints the reference line; other ranks exit.
For N > 1 (torchrun) every rank runs an independent replica (weak scaling):
a single solve of this size does not shard in this build.

--nx/--precision/--scheme/--no-e2e/--no-cpu-baseline/--no-extra select a single
measurement (used for profiling runs).
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
    ap.add_argument("--serve-baseline", type=int, default=None,
                    help="time only the first N requests one at a time in FP64 "
                         "(default: the whole stream, the same requests as the server)")
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


def serve_stream(eb2, local, n, rate, seed, baseline_n, reps=3):
    """Batched mixed-precision server vs one-at-a-time plain FP64 solves on the
    same trace: solves/s and latency percentiles (finish - arrival); the server
    side is the median of `reps` replays."""
    import numpy as np

    from overheatingproblem_b200.server import Server
    reqs, arr = stream_trace(n, rate, seed, eb2)
    # The trace is replayed in real time, so how requests meet in batches (and the
    # rate) varies from replay to replay: three replays, the median one reported.
    runs = []
    with Server(device=local, precision=eb2.lib.MIXED, scheme=2,
                hbm_budget=120 * 10**9) as srv:
        for _ in range(reps):
            runs.append(srv.run_trace(reqs, arr))
    runs.sort(key=lambda o: o["makespan"])
    out = runs[len(runs) // 2]
    lat = out["finish"] - arr
    batched = {"solves_per_s": n / out["makespan"], "makespan_s": out["makespan"],
               "p50_latency_s": float(np.percentile(lat, 50)),
               "p99_latency_s": float(np.percentile(lat, 99)), "requests": n,
               "steps": int(out["steps"].sum()),
               "non_physical": int((out["status"] != 0).sum()),
               "replays_solves_per_s": [n / o["makespan"] for o in runs]}
    # one-at-a-time plain FP64 launches: each request on its own context,
    # started when it has arrived and the previous one has finished
    m = n if baseline_n is None else min(baseline_n, n)
    t0 = time.perf_counter()
    fin = np.zeros(m)
    bad = 0
    for i in range(m):
        wait = arr[i] - (time.perf_counter() - t0)
        if wait > 0:
            time.sleep(wait)
        r = reqs[i]
        with eb2.Solver(r.nx, r.ny, device=local, recon=5, characteristic=True, weno_z=False,
                        cfl=r.cfl, precision=eb2.lib.FP64) as s:
            lx, ly, _ = s.init_case(r.test_case, r.q)
            ly = r.ly if r.ly > 0 else ly
            s.run(ORDER, 2, lx / r.nx, ly / r.ny, r.tmax)
            s.download()
            bad += s.status() != 0
        fin[i] = time.perf_counter() - t0
    blat = fin - arr[:m]
    base = {"solves_per_s": m / fin[-1], "makespan_s": float(fin[-1]),
            "p50_latency_s": float(np.percentile(blat, 50)),
            "p99_latency_s": float(np.percentile(blat, 99)), "requests": m,
            "non_physical": int(bad)}
    return {"trace": f"{n} requests, Poisson arrivals at {rate}/s, seed {seed}",
            "batched_mixed": batched, "one_at_a_time_fp64": base,
            "speedup_solves_per_s": batched["solves_per_s"] / base["solves_per_s"]}


def run_accuracy(args, local):
    """FP64 vs mixed on the benchmark problem up to t = T, with checkpoints:
    density/velocity/pressure L1 (mean over cells) and Linf differences.  A
    third run, FP64 from the same initial state with one density value moved
    by one ulp, measures how far the flow itself amplifies a perturbation of
    rounding size (the floor no arithmetic can go below)."""
    import numpy as np
    import torch

    import overheatingproblem_b200 as eb2

    nx, scheme, T = args.nx, SCHEMES[args.scheme], args.accuracy
    marks = [t for t in (0.05, 0.1, 0.2) if t < T] + [T]
    runs = {"fp64": eb2.lib.FP64, "mixed": eb2.lib.MIXED, "fp64_1ulp": eb2.lib.FP64}
    out, prim = {}, {}
    for name, prec in runs.items():
        s = eb2.Solver(nx, nx, device=local, recon=5, characteristic=True, weno_z=False,
                       cfl=0.5, precision=prec)
        lx, ly, _ = s.init_case(eb2.lib.CASE_FOUR_QUADRANT)
        if name == "fp64_1ulp":
            U = s.download()
            c = 4 + nx // 3
            U[0, c, c] = np.nextafter(U[0, c, c], np.inf)
            s.upload(U)
        torch.cuda.synchronize(local)
        el, steps, t = 0.0, 0, 0.0
        prim[name] = []
        for tm in marks:
            t0 = time.perf_counter()
            n, t = s.run(ORDER, scheme, lx / nx, ly / nx, tm, t0=t)
            el += time.perf_counter() - t0
            steps += n
            prim[name].append(s.con_to_pri()[:, 4:-4, 4:-4].copy())
        out[name] = {"steps": steps, "t_final": t, "seconds": el, "status_flags": s.status(),
                     "cell_updates_per_s": nx * nx * steps / el}
        s.close()
    names = ["rho", "u", "v", "p"]

    def diff(other):
        rows = []
        for k, tm in enumerate(marks):
            d = np.abs(prim["fp64"][k] - prim[other][k])
            rows.append({"t": tm, "l1": {q: float(d[i].mean()) for i, q in enumerate(names)},
                         "linf": {q: float(d[i].max()) for i, q in enumerate(names)}})
        return rows

    mixed, ulp = diff("mixed"), diff("fp64_1ulp")
    line = {"accuracy": workload(nx, "mixed", args.scheme) + f" vs FP64, t = {T}",
            "l1": mixed[-1]["l1"], "linf": mixed[-1]["linf"],
            "rel_l1_rho": float(np.abs(prim["fp64"][-1][0] - prim["mixed"][-1][0]).sum() /
                                np.abs(prim["fp64"][-1][0]).sum()),
            "checkpoints": {"mixed_vs_fp64": mixed, "fp64_1ulp_vs_fp64": ulp},
            "note": "checkpoint times clip the CFL step in all three runs alike",
            "runs": out}
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
            "l2": "flushed between timed steps (256 MiB write outside the timed intervals)",
            "parallelism": "replicas"}


def measured_traffic(nx, precision, scheme):
    """DRAM bytes (read + write) per fused-stage launch of this workload, from
    the committed ncu launch-list summary profiles/launches_<precision>_<nx>.md
    (taken with the same bench command), or None when there is none."""
    path = os.path.join(os.path.dirname(os.path.abspath(__file__)), "profiles",
                        f"launches_{precision}_{nx}.md")
    if scheme != "hllc" or not os.path.exists(path):
        return None
    for line in open(path):
        if "k_stage" in line and line.startswith("|"):
            cells = [c.strip() for c in line.strip().strip("|").split("|")]
            return (float(cells[4].split()[0]) + float(cells[5].split()[0])) * 1e6
    return None


def measured_compute(precision):
    """The binding on-chip limit of the stage kernel, from the committed ncu
    summary profiles/stage_<precision>_2048.md (its "now" column): FP64 pipe
    activity for the FP64 form, issue activity for the mixed form (fractions
    of peak), or None."""
    path = os.path.join(os.path.dirname(os.path.abspath(__file__)), "profiles",
                        f"stage_{precision}_2048.md")
    row = "FP64 pipe active" if precision == "fp64" else "issue active"
    if not os.path.exists(path):
        return None
    col = None
    for line in open(path):
        if not line.startswith("|"):
            continue
        cells = [c.strip() for c in line.strip().strip("|").split("|")]
        if cells[0] == "metric":
            col = next((i for i, c in enumerate(cells) if c.startswith("now") or "(now)" in c),
                       None)
        elif col is not None and cells[0].startswith(row) and len(cells) > col:
            try:
                frac = float(cells[col].split()[0]) / 100.0
            except ValueError:
                return None
            return {"limit": "fp64 pipe" if precision == "fp64" else "instruction issue",
                    "active_frac": frac,
                    "source": f"profiles/stage_{precision}_2048.md (ncu, 2048^2 stage)"}
    return None


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
    rate, per_step, n, kind, cores = cpu_rate(args.nx, SCHEMES[args.scheme], 150.0, args.steps,
                                              min(args.warmup, 1))
    line = {
        "metric": METRIC, "value": rate, "unit": "cell-updates/s", "n_gpus": args.gpus,
        "steps": n, "warmup": min(args.warmup, 1), "ms_per_step": per_step * 1e3,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic", "config": config(args), "impl": "reference",
        "cpu_baseline": {"value": rate, "unit": "cell-updates/s", "cores": cores, "kind": kind,
                         "sample": f"{n} full SSP-RK3 steps of the {args.nx}^2 grid"},
        "e2e": {"value": rate, "unit": "cell-updates/s", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


# --------------------------------------------------------------------------- GPU
def measure(eb2, local, nx, precision, scheme, steps, warmup, flush=FLUSH_BYTES):
    """Device time of `steps` steps (after `warmup`), L2 flushed between steps."""
    prec = eb2.lib.FP64 if precision == "fp64" else eb2.lib.MIXED
    s = eb2.Solver(nx, nx, device=local, recon=5, characteristic=True, weno_z=False, cfl=0.5,
                   precision=prec)
    lx, ly, _ = s.init_case(eb2.lib.CASE_FOUR_QUADRANT)
    dx, dy = lx / nx, ly / nx
    if warmup:
        s.bench_steps(ORDER, scheme, dx, dy, warmup, 0)
        s.init_case(eb2.lib.CASE_FOUR_QUADRANT)
    step_ms, stage_ms, nstage, launches = s.bench_steps(ORDER, scheme, dx, dy, steps, flush)
    st = s.status()
    return s, dx, dy, step_ms, stage_ms, nstage, launches, st


def run_ours(args, world, rank, local):
    import numpy as np
    import torch

    import overheatingproblem_b200 as eb2

    nx, scheme = args.nx, SCHEMES[args.scheme]
    torch.cuda.init()
    # warm-up pass (clocks, kernel attributes) outside the timed region
    s, *_ = measure(eb2, local, nx, args.precision, scheme, max(args.warmup, 3), 0, 0)
    s.close()
    torch.cuda.synchronize(local)
    sampler = ClockSampler(physical_gpu(local)) if rank == 0 else None
    barrier(world)
    torch.cuda.synchronize(local)
    s, dx, dy, step_ms, stage_ms, nstage, launches, st = measure(
        eb2, local, nx, args.precision, scheme, args.steps, 0)
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
                "compute": measured_compute(args.precision)}

    e2e = None
    if not args.no_e2e:
        s.init_case(eb2.lib.CASE_FOUR_QUADRANT)
        host = torch.empty((4, nx + 8, nx + 8), dtype=torch.float64, pin_memory=True).numpy()
        s.download(host)
        k_e2e = max(3, min(args.steps, 50))
        for _ in range(2):
            s.upload(host)
            s.rk_step(ORDER, scheme, s.delta_t(dx, dy), dx, dy)
            s.download(host)
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
               "path": "eb2_upload + eb2_delta_t + eb2_rk_step + eb2_download"}
    s.close()

    extra = {}
    if not args.no_extra:
        for tag, (n2, prec, sch, k) in {
                "fp64_4096_hllc": (4096, "fp64", 2, 10),
                "mixed_4096_hllc": (4096, "mixed", 2, 40),
                "mixed_4096_roe": (4096, "mixed", 3, 40),
                "mixed_1024_hllc": (1024, "mixed", 2, 200)}.items():
            s2, _, _, sm, stm, nst, _, st2 = measure(eb2, local, n2, prec, sch, k, 2)
            s2.close()
            tot = allreduce_max(float(sum(sm)), world)
            extra[tag] = {"value": world * n2 * n2 * k / (tot * 1e-3), "unit": "cell-updates/s",
                          "ms_per_step": tot / k, "steps": k, "status_flags": st2,
                          "roofline_frac": n2 * n2 * BYTES_PER_CELL_STEP * k / (stm * 1e-3) / 1e9
                          / peak}
        if rank == 0:
            extra["served_stream"] = serve_stream(eb2, local, 64, args.serve_rate, 7,
                                                  args.serve_baseline)

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        rate, per_step, n, kind, cores = cpu_rate(nx, scheme, 20.0, 40, 1)
        cpu = {"value": rate, "unit": "cell-updates/s", "cores": cores, "kind": kind,
               "sample": f"{n} full SSP-RK3 steps of the {nx}^2 grid ({per_step:.3f} s each)"}
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
                print(json.dumps(serve_stream(eb2, local, args.serve, args.serve_rate, 7,
                                              args.serve_baseline)), flush=True)
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
