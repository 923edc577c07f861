"""ctypes bindings for the CPU oracle and the reference build.

TEST INFRASTRUCTURE ONLY: imported by tests/, __graft_entry__.smoke() and the
CPU-baseline leg of bench.py, never by the product package.

* ``Oracle``    -- oracle/liboracle.so, the C restatement (euler_oracle.c).
* ``Reference`` -- oracle/_ref/libref.so (the reference as shipped),
  oracle/_ref/libref_wjs.so (its characteristic WENO5 switched to Jiang-Shu
  weights) or oracle/_ref/libref_wjs_dmr.so (that, with the reference's own
  commented-out BC_DoubleMach_2D calls of the RK stages switched on), built
  from the reference's own sources by oracle/Makefile.  They exist only where
  the reference tree was present at build time.

``REFERENCE_TREE`` is the one place that names where the reference's sources
lie (environment variable EB2_REFERENCE_TREE); only build recipes and the
checks that compile the reference's own caller read it.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
GC = 4
REFERENCE_TREE = os.environ.get("EB2_REFERENCE_TREE", "/root/reference")

_VARIANTS = {"": "libref.so", "wjs": "libref_wjs.so", "wjs_dmr": "libref_wjs_dmr.so"}

# BC kinds (include/Boundary_Condition.h:21-27)
OUTFLOW, REFLECT, PERIODIC, INFLOW, FIXED = 0, 1, 2, 3, 4
# cases of orc_init_case
FOUR_QUADRANT, WALL_HEATING, DOUBLE_MACH, PRECISION, NOH_1D, SOD_1D = 1, 2, 3, 4, 5, 6

_dp = C.POINTER(C.c_double)


def _ptr(a: np.ndarray):
    assert a.dtype == np.float64 and a.flags["C_CONTIGUOUS"]
    return a.ctypes.data_as(_dp)


class OrcParams(C.Structure):
    _fields_ = [
        ("nx", C.c_int), ("ny", C.c_int), ("gc", C.c_int),
        ("gamma", C.c_double), ("cfl", C.c_double),
        ("recon", C.c_int), ("characteristic", C.c_int), ("weno_z", C.c_int),
        ("source", C.c_int), ("gravity", C.c_double),
        ("bc", C.c_int * 4), ("dmr", C.c_int),
        ("inflow", C.c_double * 4), ("fixed", (C.c_double * 4) * 4),
    ]


def build(ref: bool = False) -> None:
    targets = ["all"] + (["ref"] if ref else [])
    subprocess.run(["make", "-s", "-C", HERE] + targets, check=True)


class Oracle:
    """The C restatement. Arrays are float64 [4, nx+8, ny+8], C order."""

    def __init__(self, path: str | None = None):
        path = path or os.path.join(HERE, "liboracle.so")
        if not os.path.exists(path):
            build(ref=False)
        lib = C.CDLL(path)
        P = C.POINTER(OrcParams)
        sig = {
            "orc_defaults": (None, [P, C.c_int, C.c_int]),
            "orc_con_to_pri": (None, [P, _dp, _dp]),
            "orc_eigen": (None, [P, C.c_int, _dp, _dp, _dp]),
            "orc_recon": (C.c_int, [P, C.c_int, _dp, _dp, _dp, C.c_double, C.c_double]),
            "orc_riemann": (None, [P, C.c_int, C.c_int, _dp, _dp, _dp]),
            "orc_flux_recon": (C.c_int, [P, C.c_int, _dp, _dp, _dp, C.c_double, C.c_double]),
            "orc_space_item": (None, [P, C.c_double, C.c_double, _dp, _dp, _dp, _dp]),
            "orc_bc": (None, [P, _dp, C.c_double]),
            "orc_source": (None, [P, _dp, _dp]),
            "orc_rk": (C.c_int, [P, C.c_int, C.c_int, _dp, C.c_double, C.c_double,
                                 C.c_double, C.c_double]),
            "orc_dt": (C.c_double, [P, _dp, C.c_double, C.c_double]),
            "orc_wave_speeds": (None, [P, _dp, _dp, _dp]),
            "orc_mesh": (None, [C.c_int, C.c_int, _dp, _dp, C.c_double, C.c_double]),
            "orc_init_case": (C.c_int, [P, C.c_int, _dp, _dp, _dp, _dp, _dp]),
            "orc_run": (C.c_long, [P, C.c_int, C.c_int, _dp, C.c_double, C.c_double,
                                   C.c_double, C.c_int, _dp]),
        }
        for name, (res, args) in sig.items():
            fn = getattr(lib, name)
            fn.restype = res
            fn.argtypes = args
        self.lib = lib

    def params(self, nx: int, ny: int, **kw) -> OrcParams:
        p = OrcParams()
        self.lib.orc_defaults(C.byref(p), nx, ny)
        for k, v in kw.items():
            if k == "bc":
                for s in range(4):
                    p.bc[s] = int(v[s])
            else:
                setattr(p, k, v)
        return p

    @staticmethod
    def shape(p: OrcParams):
        return (4, p.nx + 2 * p.gc, p.ny + 2 * p.gc)

    def zeros(self, p):
        return np.zeros(self.shape(p), dtype=np.float64)

    def init_case(self, p: OrcParams, which: int, q=None):
        U = self.zeros(p)
        lx, ly, tmax = C.c_double(), C.c_double(), C.c_double()
        qa = None if q is None else np.ascontiguousarray(q, dtype=np.float64)
        rc = self.lib.orc_init_case(C.byref(p), which, None if qa is None else _ptr(qa),
                                    _ptr(U), C.byref(lx), C.byref(ly), C.byref(tmax))
        if rc:
            raise ValueError(f"orc_init_case rc={rc}")
        return U, lx.value, ly.value, tmax.value

    def con_to_pri(self, p, U):
        W = self.zeros(p)
        self.lib.orc_con_to_pri(C.byref(p), _ptr(U), _ptr(W))
        return W

    def eigen(self, p, direction, pri):
        rows, cols = p.nx + 2 * p.gc, p.ny + 2 * p.gc
        el = np.zeros((4, 4, rows, cols))
        er = np.zeros((4, 4, rows, cols))
        self.lib.orc_eigen(C.byref(p), direction, _ptr(pri), _ptr(el), _ptr(er))
        return el, er

    def recon(self, p, direction, U, dx, dy):
        ql, qr = self.zeros(p), self.zeros(p)
        rc = self.lib.orc_recon(C.byref(p), direction, _ptr(U), _ptr(ql), _ptr(qr), dx, dy)
        if rc:
            raise ValueError(f"orc_recon rc={rc}")
        return ql, qr

    def riemann(self, p, scheme, direction, ql, qr, flux=None):
        flux = self.zeros(p) if flux is None else flux
        self.lib.orc_riemann(C.byref(p), scheme, direction, _ptr(ql), _ptr(qr), _ptr(flux))
        return flux

    def flux_recon(self, p, scheme, U, dx, dy):
        f, g = self.zeros(p), self.zeros(p)
        rc = self.lib.orc_flux_recon(C.byref(p), scheme, _ptr(U), _ptr(f), _ptr(g), dx, dy)
        if rc:
            raise ValueError(f"orc_flux_recon rc={rc}")
        return f, g

    def space_item(self, p, dx, dy, f, g, s):
        out = self.zeros(p)
        self.lib.orc_space_item(C.byref(p), dx, dy, _ptr(f), _ptr(g), _ptr(s), _ptr(out))
        return out

    def bc(self, p, U, t=0.0):
        self.lib.orc_bc(C.byref(p), _ptr(U), t)
        return U

    def rk(self, p, order, scheme, U, dt, dx, dy, t=0.0):
        rc = self.lib.orc_rk(C.byref(p), order, scheme, _ptr(U), dt, dx, dy, t)
        if rc:
            raise ValueError(f"orc_rk rc={rc}")
        return U

    def dt(self, p, U, dx, dy) -> float:
        return self.lib.orc_dt(C.byref(p), _ptr(U), dx, dy)

    def wave_speeds(self, p, U):
        sx, sy = C.c_double(), C.c_double()
        self.lib.orc_wave_speeds(C.byref(p), _ptr(U), C.byref(sx), C.byref(sy))
        return sx.value, sy.value

    def run(self, p, order, scheme, U, dx, dy, tmax, n_out=1):
        tf = C.c_double()
        n = self.lib.orc_run(C.byref(p), order, scheme, _ptr(U), dx, dy, tmax, n_out,
                             C.byref(tf))
        return n, tf.value


class Reference:
    """The reference compiled from its own sources (oracle/_ref)."""

    def __init__(self, variant: str = ""):
        path = os.path.join(HERE, "_ref", _VARIANTS[variant])
        if not os.path.exists(path):
            raise FileNotFoundError(path)
        self.variant = variant
        lib = C.CDLL(path)
        i, d = C.c_int, C.c_double
        sig = {
            "ref_set_params": (None, [d, d, i, i, i, d]),
            "ref_set_bc": (None, [i, i, i, i]),
            "ref_get_bc": (None, [C.POINTER(C.c_int)]),
            "ref_init": (None, [i, i, i, _dp, _dp, _dp, _dp, _dp, _dp, _dp]),
            "ref_con_to_pri": (None, [i, i, _dp, _dp]),
            "ref_eigen": (None, [i, i, i, _dp, _dp, _dp]),
            "ref_recon": (None, [i, i, i, _dp, _dp, _dp, d, d]),
            "ref_riemann": (None, [i, i, i, i, _dp, _dp, _dp]),
            "ref_flux_recon": (None, [i, i, i, _dp, _dp, _dp, d, d, d]),
            "ref_space_item": (None, [i, i, d, d, _dp, _dp, _dp, _dp]),
            "ref_bc": (None, [i, i, _dp]),
            "ref_bc_dmr": (None, [i, i, _dp, d]),
            "ref_source": (None, [i, i, _dp, _dp]),
            "ref_rk": (None, [i, i, i, i, _dp, d, d, d]),
            "ref_rk_dmr": (None, [i, i, i, i, _dp, d, d, d, d]),
            "ref_dt": (d, [i, i, _dp, d, d]),
            "ref_mesh": (None, [i, i, _dp, _dp, d, d]),
            "ref_read_control": (None, [C.c_char_p, C.POINTER(C.c_int), _dp, C.c_char_p, i]),
            "ref_run": (C.c_long, [i, i, i, i, _dp, d, d, d, i, i, _dp]),
            "ref_num_threads": (i, []),
            "ref_set_threads": (None, [i]),
            "ref_set_time": (None, [d]),
        }
        for n_, (res, args) in sig.items():
            fn = getattr(lib, n_)
            fn.restype = res
            fn.argtypes = args
        self.lib = lib

    @staticmethod
    def available(variant: str = "") -> bool:
        return os.path.exists(os.path.join(HERE, "_ref", _VARIANTS[variant]))

    def configure(self, p: OrcParams):
        self.lib.ref_set_params(p.gamma, p.cfl, p.recon, p.characteristic, p.source, p.gravity)
        self.lib.ref_set_bc(p.bc[0], p.bc[1], p.bc[2], p.bc[3])

    def rk(self, p, order, scheme, U, dt, dx, dy, t=0.0):
        """One RKn_TimeAd step.  In the wjs_dmr build the reference's own RK
        stages fill ghosts with BC_DoubleMach_2D at the global Time = t; in the
        other builds p.dmr selects the composed ref_rk_dmr."""
        self.configure(p)
        rows, cols = U.shape[1], U.shape[2]
        if self.variant == "wjs_dmr":
            self.lib.ref_set_time(t)
            self.lib.ref_rk(order, scheme, rows, cols, _ptr(U), dt, dx, dy)
        elif p.dmr:
            self.lib.ref_rk_dmr(order, scheme, rows, cols, _ptr(U), dt, dx, dy, t)
        else:
            self.lib.ref_rk(order, scheme, rows, cols, _ptr(U), dt, dx, dy)
        return U

    def init(self, test_case: int, nx: int, ny: int):
        """Init_Euler_2D of one of the reference's own TestCase2D values: the
        conserved state, the domain lengths and final time, and the boundary
        kinds the case sets."""
        rows, cols = nx + 2 * GC, ny + 2 * GC
        arrs = [np.zeros((4, rows, cols)) for _ in range(4)]
        lx, ly, tmax = C.c_double(), C.c_double(), C.c_double()
        self.lib.ref_init(test_case, rows, cols, *(_ptr(a) for a in arrs), C.byref(lx),
                          C.byref(ly), C.byref(tmax))
        kinds = (C.c_int * 4)()
        self.lib.ref_get_bc(kinds)
        return arrs[1], lx.value, ly.value, tmax.value, tuple(kinds)

    def dt(self, p, U, dx, dy) -> float:
        self.configure(p)
        return self.lib.ref_dt(U.shape[1], U.shape[2], _ptr(U), dx, dy)

    def riemann(self, p, scheme, direction, ql, qr, flux):
        self.configure(p)
        self.lib.ref_riemann(scheme, direction, ql.shape[1], ql.shape[2], _ptr(ql), _ptr(qr),
                             _ptr(flux))
        return flux

    def run(self, p, order, scheme, U, dx, dy, tmax, n_out=1):
        self.configure(p)
        tf = C.c_double()
        n = self.lib.ref_run(order, scheme, U.shape[1], U.shape[2], _ptr(U), dx, dy, tmax,
                             n_out, int(p.dmr), C.byref(tf))
        return n, tf.value
