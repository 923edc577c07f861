"""The solve server: continuous batching of independent solves.

A result must not depend on what else is in the batch: each request run
alone, run in a mix of uneven sizes and final times, and run by eb2_run on a
context gives the same bits (mixed precision and FP64 forms alike).  Plus
admission by HBM budget, retirement and the request loop."""
from __future__ import annotations

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def fq_states(rng):
    """Four-quadrant states mild enough that the reference scheme stays
    physical (wide random states can drive it into negative pressures)."""
    st = []
    for _ in range(4):
        st += [rng.uniform(0.5, 2.0), rng.uniform(-0.5, 0.5), rng.uniform(-0.5, 0.5),
               rng.uniform(0.5, 2.0)]
    return st


def mix(gpu):
    from overheatingproblem_b200.server import Request
    rng = np.random.default_rng(11)
    L = gpu.lib
    reqs = []
    for k, n in enumerate([64, 128, 96, 48, 160, 64]):
        if k % 2 == 0:
            reqs.append(Request(L.CASE_FOUR_QUADRANT, n, n, q=fq_states(rng),
                                tmax=float(rng.uniform(0.02, 0.06))))
        else:
            reqs.append(Request(L.CASE_WALL_HEATING, n, n, q=[float(rng.uniform(0.5, 2.0))],
                                ly=1.0, tmax=float(rng.uniform(0.02, 0.06))))
    return reqs


def run_alone_ctx(gpu, req, precision, scheme=2):
    """The same solve on a single-solve context (eb2_run)."""
    with gpu.Solver(req.nx, req.ny, precision=precision, recon=5, characteristic=True,
                    weno_z=False, cfl=req.cfl) as s:
        lx, ly, _ = s.init_case(req.test_case, req.q)
        if req.ly > 0:
            ly = req.ly
        if req.lx > 0:
            lx = req.lx
        s.run(3, scheme, lx / req.nx, ly / req.ny, req.tmax)
        return s.download()


# (the FP64 form also with the anti-overheating HLLCHC flux, AR_scheme 22)
@pytest.mark.parametrize("precision,scheme", [("mixed", 2), ("fp64", 2), ("fp64", 22)])
def test_result_same_alone_and_in_the_mix(gpu, precision, scheme):
    from overheatingproblem_b200.server import Server
    prec = gpu.lib.MIXED if precision == "mixed" else gpu.lib.FP64
    reqs = mix(gpu)
    with Server(precision=prec, scheme=scheme) as srv:
        mixed = srv.run_trace(reqs, np.zeros(len(reqs)), keep_results=True)["results"]
    for i, req in enumerate(reqs):
        with Server(precision=prec, scheme=scheme) as srv:
            alone = srv.run_trace([req], [0.0], keep_results=True)["results"][0]
        ctx = run_alone_ctx(gpu, req, prec, scheme)
        g = 4
        a, b, c = (x[:, g:-g, g:-g] for x in (alone, mixed[i], ctx))
        assert np.all(np.isfinite(c)), i
        assert np.array_equal(a.view(np.int64), b.view(np.int64)), i
        assert np.array_equal(a.view(np.int64), c.view(np.int64)), i
        assert np.all(np.isfinite(a))


def test_slot_that_fills_the_gpu_has_its_own_launch(gpu):
    """A mixed slot with more tiles than the GPU holds CTAs (768^2: 1152 tiles
    of 16 x 32) runs as a stage launch of its own beside the batched launch of
    the small slots; its result and theirs stay the bits of single-solve runs."""
    from overheatingproblem_b200.server import Request, Server
    L = gpu.lib
    rng = np.random.default_rng(5)
    reqs = [Request(L.CASE_FOUR_QUADRANT, 768, 768, q=fq_states(rng), tmax=0.02),
            Request(L.CASE_FOUR_QUADRANT, 64, 64, q=fq_states(rng), tmax=0.03),
            Request(L.CASE_WALL_HEATING, 96, 96, q=[1.3], ly=1.0, tmax=0.025)]
    with Server(precision=L.MIXED, scheme=2) as srv:
        got = srv.run_trace(reqs, np.zeros(len(reqs)), keep_results=True)["results"]
    for i, req in enumerate(reqs):
        ctx = run_alone_ctx(gpu, req, L.MIXED)
        a, c = (x[:, 4:-4, 4:-4] for x in (got[i], ctx))
        assert np.all(np.isfinite(c)), i
        assert np.array_equal(a.view(np.int64), c.view(np.int64)), i


def test_reused_slot_with_its_own_launch(gpu):
    """Two large mixed requests of different sizes through one slot, one after
    the other: the second reuses the slot index with a grid and buffers of its
    own, and its launch must follow them (same bits as a single-solve run)."""
    from overheatingproblem_b200.server import Request, Server
    L = gpu.lib
    rng = np.random.default_rng(9)
    reqs = [Request(L.CASE_FOUR_QUADRANT, 768, 768, q=fq_states(rng), tmax=0.01),
            Request(L.CASE_FOUR_QUADRANT, 896, 896, q=fq_states(rng), tmax=0.015)]
    with Server(precision=L.MIXED, scheme=2, max_slots=1) as srv:
        got = srv.run_trace(reqs, np.zeros(len(reqs)), keep_results=True)["results"]
    for i, req in enumerate(reqs):
        ctx = run_alone_ctx(gpu, req, L.MIXED)
        a, c = (x[:, 4:-4, 4:-4] for x in (got[i], ctx))
        assert np.array_equal(a.view(np.int64), c.view(np.int64)), i


def test_admission_by_budget_and_retirement(gpu):
    from overheatingproblem_b200.server import Request, Server
    L = gpu.lib
    one = 3 * 4 * 136 * 136 * 8 + 3 * 296 * 8     # slot bytes of a 128^2 solve
    with Server(precision=L.MIXED, hbm_budget=2 * one + 100) as srv:
        r = Request(L.CASE_FOUR_QUADRANT, 128, 128, tmax=0.01)
        a, b = srv.submit(r), srv.submit(r)
        assert a is not None and b is not None
        assert srv.submit(r) is None                      # budget full
        while srv.active:
            srv.step()
        done = {x[0] for x in srv.finished()}
        assert done == {a, b}
        srv.fetch(a)
        c = srv.submit(r)                                 # memory freed by retirement
        assert c is not None
        while srv.active:
            srv.step()
        assert srv.stats()["hbm_used"] == 2 * one


def test_request_loop_admits_while_running(gpu):
    """Later arrivals are admitted while earlier solves run (their work
    overlaps on the device), and every request finishes."""
    from overheatingproblem_b200.server import Request, Server
    L = gpu.lib
    reqs = [Request(L.CASE_FOUR_QUADRANT, 512, 512, tmax=0.1) for _ in range(6)]
    arrivals = np.arange(len(reqs)) * 0.002
    with Server(precision=gpu.lib.MIXED) as srv:
        out = srv.run_trace(reqs, arrivals)
    admit, finish = out["admit"], out["finish"]
    assert np.all(finish > admit) and np.all(admit >= arrivals - 1e-9)
    # some request was admitted before an earlier one had finished
    order = np.argsort(admit)
    assert any(admit[order[k + 1]] < finish[order[k]] for k in range(len(reqs) - 1))
