"""One device-resident solve: a thin object over an eb2_ctx.

Arrays exchanged with the host are numpy float64 [4, nx+8, ny+8] in the
reference's layout (x index first, y unit stride, 4 ghost layers).
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import lib as L

GC = 4


class Solver:
    def __init__(self, nx: int, ny: int, device: int = 0, *, gamma: float = 1.4,
                 cfl: float = 0.5, recon: int = 5, characteristic: bool = False,
                 weno_z: bool = True, precision: int = L.FP64, source: bool = False,
                 gravity: float = 1.0):
        self._lib = L.library()
        h = C.c_void_p()
        L.check(self._lib.eb2_ctx_create(C.byref(h), int(nx), int(ny), int(device)))
        self._h = h
        self.nx, self.ny = int(nx), int(ny)
        self.rows, self.cols = self.nx + 2 * GC, self.ny + 2 * GC
        self.set_material(gamma, source, gravity, cfl)
        self.set_reconstruction(recon, characteristic, weno_z)
        self.set_precision(precision)

    # -- lifetime ------------------------------------------------------------
    def close(self) -> None:
        if getattr(self, "_h", None) is not None and self._h.value:
            self._lib.eb2_ctx_destroy(self._h)
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

    @property
    def handle(self) -> C.c_void_p:
        return self._h

    # -- settings ------------------------------------------------------------
    def set_material(self, gamma, source=False, gravity=1.0, cfl=0.5):
        self.gamma, self.cfl = gamma, cfl
        L.check(self._lib.eb2_set_material(self._h, gamma, int(bool(source)), gravity, cfl))

    def set_reconstruction(self, recon=5, characteristic=False, weno_z=True):
        L.check(self._lib.eb2_set_reconstruction(self._h, int(recon), int(bool(characteristic)),
                                                 int(bool(weno_z))))

    def set_precision(self, precision):
        L.check(self._lib.eb2_set_precision(self._h, int(precision)))

    def set_positivity_fallback(self, on: bool):
        L.check(self._lib.eb2_set_positivity_fallback(self._h, int(bool(on))))

    def set_bc(self, left, right, bottom, top):
        L.check(self._lib.eb2_set_bc(self._h, left, right, bottom, top))

    def get_bc(self) -> tuple:
        kinds = (C.c_int * 4)()
        L.check(self._lib.eb2_get_bc(self._h, kinds))
        return tuple(kinds)

    def set_bc_states(self, inflow=None, fixed=None):
        a = None if inflow is None else np.ascontiguousarray(inflow, dtype=np.float64)
        b = None if fixed is None else np.ascontiguousarray(fixed, dtype=np.float64)
        L.check(self._lib.eb2_set_bc_states(self._h, None if a is None else L.dptr(a),
                                            None if b is None else L.dptr(b)))

    def set_double_mach(self, on: bool):
        L.check(self._lib.eb2_set_double_mach(self._h, int(bool(on))))

    # -- state -----------------------------------------------------------------
    def zeros(self) -> np.ndarray:
        return np.zeros((4, self.rows, self.cols), dtype=np.float64)

    def init_case(self, case: int, q=None):
        qa = None if q is None else np.ascontiguousarray(q, dtype=np.float64)
        lx, ly, tmax = C.c_double(), C.c_double(), C.c_double()
        L.check(self._lib.eb2_init_case(self._h, int(case), None if qa is None else L.dptr(qa),
                                        C.byref(lx), C.byref(ly), C.byref(tmax)))
        self.lx, self.ly = lx.value, ly.value
        self.dx, self.dy = self.lx / self.nx, self.ly / self.ny
        return lx.value, ly.value, tmax.value

    def upload(self, U: np.ndarray) -> None:
        U = np.ascontiguousarray(U, dtype=np.float64)
        if U.shape != (4, self.rows, self.cols):
            raise ValueError(f"state shape {U.shape} != {(4, self.rows, self.cols)}")
        L.check(self._lib.eb2_upload(self._h, L.dptr(U)))

    def download(self, out: np.ndarray | None = None) -> np.ndarray:
        out = self.zeros() if out is None else out
        L.check(self._lib.eb2_download(self._h, L.dptr(out)))
        return out

    # -- operators ---------------------------------------------------------------
    def bc_apply(self, time: float = 0.0):
        L.check(self._lib.eb2_bc_apply(self._h, time))

    def con_to_pri(self, pri: np.ndarray | None = None) -> np.ndarray:
        pri = self.zeros() if pri is None else pri
        L.check(self._lib.eb2_con_to_pri(self._h, L.dptr(pri)))
        return pri

    def eigen(self, direction: int, pri: np.ndarray):
        el = np.zeros((4, 4, self.rows, self.cols))
        er = np.zeros((4, 4, self.rows, self.cols))
        L.check(self._lib.eb2_eigen(self._h, direction, L.dptr(np.ascontiguousarray(pri)),
                                    L.dptr(el), L.dptr(er)))
        return el, er

    def reconstruct(self, direction: int, dx: float, dy: float):
        ql, qr = self.zeros(), self.zeros()
        L.check(self._lib.eb2_reconstruct(self._h, direction, dx, dy, L.dptr(ql), L.dptr(qr)))
        return ql, qr

    def riemann(self, scheme: int, direction: int, ql, qr, flux=None):
        flux = self.zeros() if flux is None else flux
        L.check(self._lib.eb2_riemann(self._h, scheme, direction, L.dptr(ql), L.dptr(qr),
                                      L.dptr(flux)))
        return flux

    def flux_reconstruction(self, scheme: int, dx: float, dy: float, f=None, g=None):
        f = self.zeros() if f is None else f
        g = self.zeros() if g is None else g
        L.check(self._lib.eb2_flux_reconstruction(self._h, scheme, dx, dy, L.dptr(f), L.dptr(g)))
        return f, g

    def space_discrete(self, dx, dy, f, g, out=None, source=None):
        out = self.zeros() if out is None else out
        src = None if source is None else L.dptr(np.ascontiguousarray(source))
        L.check(self._lib.eb2_space_discrete(self._h, dx, dy, L.dptr(f), L.dptr(g), src,
                                             L.dptr(out)))
        return out

    def delta_t(self, dx: float, dy: float) -> float:
        dt = C.c_double()
        L.check(self._lib.eb2_delta_t(self._h, dx, dy, C.byref(dt)))
        return dt.value

    def wave_speeds(self):
        sx, sy = C.c_double(), C.c_double()
        L.check(self._lib.eb2_wave_speeds(self._h, C.byref(sx), C.byref(sy)))
        return sx.value, sy.value

    def rk_step(self, order: int, scheme: int, dt: float, dx: float, dy: float,
                time: float = 0.0, allow_nonphysical: bool = True) -> int:
        rc = self._lib.eb2_rk_step(self._h, order, scheme, dt, dx, dy, time)
        if rc == L.EB2_ENONPHYS and allow_nonphysical:
            return rc
        L.check(rc)
        return rc

    def run(self, order: int, scheme: int, dx: float, dy: float, tmax: float, n_out: int = 1,
            t0: float = 0.0, on_output=None):
        steps, tf = C.c_longlong(), C.c_double()
        if on_output is None:
            cb = OUTPUT_NONE
        else:
            cb = L.OUTPUT_FN(lambda _u, t, s: on_output(t, s))
        L.check(self._lib.eb2_run(self._h, order, scheme, dx, dy, t0, tmax, n_out, cb, None,
                                  C.byref(steps), C.byref(tf)))
        return steps.value, tf.value

    def advance(self, order: int, scheme: int, dx: float, dy: float, nsteps: int) -> None:
        """Exactly `nsteps` device-loop steps (CFL dt, no clipping)."""
        L.check(self._lib.eb2_advance(self._h, order, scheme, dx, dy, int(nsteps)))

    def bench_steps(self, order: int, scheme: int, dx: float, dy: float, nsteps: int,
                    flush_bytes: int = 0):
        """Per-step device times (ms), summed stage-kernel time (ms), stage
        launches and library launches inside the timed intervals."""
        step_ms = (C.c_float * nsteps)()
        stage_ms, nst, nl = C.c_float(), C.c_int(), C.c_longlong()
        L.check(self._lib.eb2_bench_steps(self._h, order, scheme, dx, dy, int(nsteps),
                                          int(flush_bytes), step_ms, C.byref(stage_ms),
                                          C.byref(nst), C.byref(nl)))
        return list(step_ms), stage_ms.value, nst.value, nl.value

    def set_stream(self, stream_handle: int | None) -> None:
        L.check(self._lib.eb2_set_stream(self._h, stream_handle))

    def status(self) -> int:
        st = C.c_uint()
        L.check(self._lib.eb2_status(self._h, C.byref(st)))
        return st.value

    def clear_status(self):
        L.check(self._lib.eb2_clear_status(self._h))

    def synchronize(self):
        L.check(self._lib.eb2_synchronize(self._h))


OUTPUT_NONE = L.OUTPUT_FN()
