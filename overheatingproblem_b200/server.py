"""The solve server (eb2_server_*): continuous batching of independent solves.

    srv = Server(precision=MIXED, scheme=2)
    ids = [srv.submit(Request(CASE_FOUR_QUADRANT, 256, 256, q=states, tmax=0.2))]
    while srv.active: srv.step()
    U = srv.fetch(ids[0])

``Server.run_trace`` replays a whole arrival trace through the native request
loop and returns admission/finish times per request.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass, field

import numpy as np

from . import lib as L

_dp = C.POINTER(C.c_double)
_Req = L.Request


@dataclass
class Request:
    test_case: int
    nx: int
    ny: int
    q: list | None = None
    lx: float = 0.0
    ly: float = 0.0
    tmax: float = 0.0
    cfl: float = 0.5
    meta: dict = field(default_factory=dict)

    def to_c(self) -> _Req:
        r = _Req()
        r.test_case, r.nx, r.ny = self.test_case, self.nx, self.ny
        if self.q is not None:
            r.has_q = 1
            for i, v in enumerate(self.q):
                r.q[i] = float(v)
        r.lx, r.ly, r.tmax, r.cfl = self.lx, self.ly, self.tmax, self.cfl
        return r


class Server:
    def __init__(self, device: int = 0, *, max_slots: int = 1024,
                 hbm_budget: int = 120 * 10**9, precision: int = L.MIXED, scheme: int = 2,
                 characteristic: bool = True, weno_z: bool = False, gamma: float = 1.4):
        self._lib = L.library()
        h = C.c_void_p()
        L.check(self._lib.eb2_server_create(C.byref(h), device, max_slots, int(hbm_budget),
                                            precision, 5, int(characteristic), int(weno_z),
                                            scheme, gamma))
        self._h = h

    def close(self):
        if getattr(self, "_h", None) is not None and self._h.value:
            self._lib.eb2_server_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def submit(self, req: Request) -> int | None:
        """Request id, or None when no slot or budget is free right now."""
        cid = C.c_longlong()
        rc = self._lib.eb2_server_submit(self._h, C.byref(req.to_c()), C.byref(cid))
        if rc == L.EB2_EBUSY:
            return None
        L.check(rc)
        return cid.value

    def step(self, ngraphs: int = 1) -> int:
        nf = C.c_int()
        L.check(self._lib.eb2_server_step(self._h, ngraphs, C.byref(nf)))
        return nf.value

    def finished(self):
        n = C.c_int()
        ids = (C.c_longlong * 4096)()
        tf = (C.c_double * 4096)()
        st = (C.c_longlong * 4096)()
        fl = (C.c_uint * 4096)()
        L.check(self._lib.eb2_server_poll(self._h, ids, tf, st, fl, 4096, C.byref(n)))
        return [(ids[i], tf[i], st[i], fl[i]) for i in range(n.value)]

    def fetch(self, rid: int, shape=None) -> np.ndarray | None:
        out = None if shape is None else np.zeros(shape)
        L.check(self._lib.eb2_server_fetch(self._h, rid, None if out is None else L.dptr(out)))
        return out

    def timing(self) -> dict:
        """Device time of the batch steps so far (s), and the host seconds in
        autotuner trials and in admission, rebuilds and retirement."""
        ms, tune, admin = C.c_double(), C.c_double(), C.c_double()
        L.check(self._lib.eb2_server_timing(self._h, C.byref(ms), C.byref(tune),
                                            C.byref(admin)))
        return {"busy_s": ms.value * 1e-3, "tune_s": tune.value, "admin_s": admin.value}

    def stats(self):
        used, act, gl = C.c_ulonglong(), C.c_int(), C.c_longlong()
        L.check(self._lib.eb2_server_stats(self._h, C.byref(used), C.byref(act), C.byref(gl)))
        return {"hbm_used": used.value, "active": act.value, "graph_launches": gl.value}

    @property
    def active(self) -> int:
        return self.stats()["active"]

    def run_trace(self, reqs: list[Request], arrival_s, keep_results=False):
        """Replay a trace in real time.  keep_results: False, True (every
        request's final state) or a collection of request indices whose final
        states are kept (the others are dropped at retirement)."""
        n = len(reqs)
        arr = (_Req * n)(*[r.to_c() for r in reqs])
        t_arr = np.ascontiguousarray(arrival_s, dtype=np.float64)
        admit = np.zeros(n)
        finish = np.zeros(n)
        steps = (C.c_longlong * max(n, 1))()
        status = (C.c_uint * max(n, 1))()
        span = C.c_double()
        results = None
        res_ptrs = None
        if keep_results is not False:
            keep = set(range(n)) if keep_results is True else set(keep_results)
            results = [np.zeros((4, r.nx + 8, r.ny + 8)) if i in keep else None
                       for i, r in enumerate(reqs)]
            res_ptrs = (_dp * n)(*[L.dptr(a) if a is not None else None for a in results])
        L.check(self._lib.eb2_server_run_trace(self._h, arr, L.dptr(t_arr), n, L.dptr(admit),
                                               L.dptr(finish), steps, status, res_ptrs,
                                               C.byref(span)))
        return {"admit": admit, "finish": finish, "makespan": span.value, "results": results,
                "steps": np.array(steps[:n], dtype=np.int64),
                "status": np.array(status[:n], dtype=np.uint32)}
