"""ctypes binding of libeuler_b200.so (include/euler_b200.h).

The library is loaded from this package directory (it is built in-tree by
``python -m overheatingproblem_b200.build``).  A missing library raises
``ImportError`` at first use; a missing GPU makes ``eb2_ctx_create`` fail with
EB2_ECUDA, which surfaces as :class:`EB2Error`.  Nothing here computes on the
CPU.
"""
from __future__ import annotations

import ctypes as C
import os
import threading

HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_NAME = "libeuler_b200.so"

EB2_OK, EB2_EARG, EB2_ENOMEM, EB2_ECUDA, EB2_ENONPHYS, EB2_EUNSUPPORTED, EB2_EBUSY = range(7)
ST_NONPHYSICAL, ST_NAN_STATE, ST_BAD_DT = 1, 2, 4
FP64, MIXED = 0, 1
BC_OUTFLOW, BC_REFLECTION, BC_PERIODICITY, BC_INFLOW, BC_FIXED_VALUE = range(5)

CASE_PRECISION = 0
CASE_SOD_1D = 1
CASE_IMPACT_WALL_1D = 4
CASE_NOH_1D = 6
CASE_RIEMANN = (7, 8, 9, 10, 11)
CASE_CONTACT_1D, CASE_SHOCK_IMPACT_1D, CASE_DOUBLE_RARE_1D = 2, 3, 5
CASE_TAYLOR_GREEN, CASE_GAUSSIAN_PULSE, CASE_KELVIN_HELMHOLTZ, CASE_RAYLEIGH_TAYLOR = 12, 13, 14, 15
CASE_DOUBLE_MACH = 16
CASE_BLAST_WAVE, CASE_NOH_2D, CASE_ODD_EVEN, CASE_BACKWARD_STEP = 17, 18, 19, 20
CASE_FOUR_QUADRANT = 100
CASE_WALL_HEATING = 101

_dp = C.POINTER(C.c_double)
_vp = C.c_void_p
OUTPUT_FN = C.CFUNCTYPE(None, C.c_void_p, C.c_double, C.c_longlong)


class EB2Error(RuntimeError):
    def __init__(self, code: int, message: str):
        super().__init__(f"[eb2 error {code}] {message}")
        self.code = code


class Control(C.Structure):
    """eb2_control == ControlParams of src/RP_FVM.c:66-82."""
    _fields_ = [
        ("test_case", C.c_int), ("L_nx", C.c_int), ("L_ny", C.c_int),
        ("Time_ADM", C.c_int), ("scheme", C.c_int), ("M_gamma", C.c_double),
        ("Source", C.c_int), ("Gravity", C.c_double), ("CFL", C.c_double),
        ("Tmax", C.c_double), ("Control_Compution", C.c_int), ("Control_output", C.c_int),
        ("Recon_Accur", C.c_int), ("Characteriz", C.c_int), ("output_dir", C.c_char * 256),
    ]


class Request(C.Structure):
    """eb2_request of include/euler_b200.h."""
    _fields_ = [("test_case", C.c_int), ("nx", C.c_int), ("ny", C.c_int), ("has_q", C.c_int),
                ("q", C.c_double * 16), ("lx", C.c_double), ("ly", C.c_double),
                ("tmax", C.c_double), ("cfl", C.c_double)]


class NoallocConfig(C.Structure):
    """eb2_noalloc_config of include/euler_b200.h."""
    _fields_ = [
        ("gamma", C.c_double), ("recon", C.c_int), ("characteristic", C.c_int),
        ("weno_z", C.c_int), ("bc_left", C.c_int), ("bc_right", C.c_int),
        ("bc_bottom", C.c_int), ("bc_top", C.c_int), ("source", C.c_int),
        ("gravity", C.c_double),
    ]


NOALLOC_MAX_CELLS = 262144

# name -> (restype, argtypes); every entry point declared in include/euler_b200.h
SIGNATURES = {
    "eb2_ctx_create": (C.c_int, [C.POINTER(_vp), C.c_int, C.c_int, C.c_int]),
    "eb2_ctx_destroy": (C.c_int, [_vp]),
    "eb2_set_stream": (C.c_int, [_vp, _vp]),
    "eb2_set_material": (C.c_int, [_vp, C.c_double, C.c_int, C.c_double, C.c_double]),
    "eb2_set_reconstruction": (C.c_int, [_vp, C.c_int, C.c_int, C.c_int]),
    "eb2_set_precision": (C.c_int, [_vp, C.c_int]),
    "eb2_set_positivity_fallback": (C.c_int, [_vp, C.c_int]),
    "eb2_set_bc": (C.c_int, [_vp, C.c_int, C.c_int, C.c_int, C.c_int]),
    "eb2_get_bc": (C.c_int, [_vp, C.POINTER(C.c_int)]),
    "eb2_set_bc_states": (C.c_int, [_vp, _dp, _dp]),
    "eb2_set_double_mach": (C.c_int, [_vp, C.c_int]),
    "eb2_init_case": (C.c_int, [_vp, C.c_int, _dp, _dp, _dp, _dp]),
    "eb2_init_case_fields": (C.c_int, [_vp, C.c_int, _dp, _dp, _dp, _dp, _dp, _dp, _dp]),
    "eb2_upload": (C.c_int, [_vp, _dp]),
    "eb2_download": (C.c_int, [_vp, _dp]),
    "eb2_state_device_ptr": (C.c_int, [_vp, C.POINTER(_dp)]),
    "eb2_bc_apply": (C.c_int, [_vp, C.c_double]),
    "eb2_con_to_pri": (C.c_int, [_vp, _dp]),
    "eb2_eigen": (C.c_int, [_vp, C.c_int, _dp, _dp, _dp]),
    "eb2_reconstruct": (C.c_int, [_vp, C.c_int, C.c_double, C.c_double, _dp, _dp]),
    "eb2_riemann": (C.c_int, [_vp, C.c_int, C.c_int, _dp, _dp, _dp]),
    "eb2_flux_reconstruction": (C.c_int, [_vp, C.c_int, C.c_double, C.c_double, _dp, _dp]),
    "eb2_space_discrete": (C.c_int, [_vp, C.c_double, C.c_double, _dp, _dp, _dp, _dp]),
    "eb2_delta_t": (C.c_int, [_vp, C.c_double, C.c_double, _dp]),
    "eb2_wave_speeds": (C.c_int, [_vp, _dp, _dp]),
    "eb2_rk_step": (C.c_int, [_vp, C.c_int, C.c_int, C.c_double, C.c_double, C.c_double,
                              C.c_double]),
    "eb2_run": (C.c_int, [_vp, C.c_int, C.c_int, C.c_double, C.c_double, C.c_double,
                          C.c_double, C.c_int, OUTPUT_FN, _vp, C.POINTER(C.c_longlong), _dp]),
    "eb2_advance": (C.c_int, [_vp, C.c_int, C.c_int, C.c_double, C.c_double, C.c_int]),
    "eb2_bench_steps": (C.c_int, [_vp, C.c_int, C.c_int, C.c_double, C.c_double, C.c_int,
                                  C.c_ulonglong, C.POINTER(C.c_float), C.POINTER(C.c_float),
                                  C.POINTER(C.c_int), C.POINTER(C.c_longlong)]),
    "eb2_server_create": (C.c_int, [C.POINTER(_vp), C.c_int, C.c_int, C.c_ulonglong, C.c_int,
                                    C.c_int, C.c_int, C.c_int, C.c_int, C.c_double]),
    "eb2_server_destroy": (C.c_int, [_vp]),
    "eb2_server_submit": (C.c_int, [_vp, C.POINTER(Request), C.POINTER(C.c_longlong)]),
    "eb2_server_step": (C.c_int, [_vp, C.c_int, C.POINTER(C.c_int)]),
    "eb2_server_timing": (C.c_int, [_vp, C.POINTER(C.c_double), C.POINTER(C.c_double),
                                    C.POINTER(C.c_double)]),
    "eb2_server_poll": (C.c_int, [_vp, C.POINTER(C.c_longlong), _dp, C.POINTER(C.c_longlong),
                                  C.POINTER(C.c_uint), C.c_int, C.POINTER(C.c_int)]),
    "eb2_server_fetch": (C.c_int, [_vp, C.c_longlong, _dp]),
    "eb2_server_stats": (C.c_int, [_vp, C.POINTER(C.c_ulonglong), C.POINTER(C.c_int),
                                   C.POINTER(C.c_longlong)]),
    "eb2_server_run_trace": (C.c_int, [_vp, C.POINTER(Request), _dp, C.c_int, _dp, _dp,
                                       C.POINTER(C.c_longlong), C.POINTER(C.c_uint),
                                       C.POINTER(_dp), _dp]),
    "eb2_rk1_backward_step": (C.c_int, [_vp, C.c_int, C.c_double, C.c_double, C.c_double]),
    "eb2_rk_step_noalloc": (C.c_int, [_vp, C.c_int, C.c_int, C.POINTER(NoallocConfig), C.c_int,
                                      C.c_int, C.c_double, C.c_double, C.c_double, C.c_double,
                                      _vp]),
    "eb2_status": (C.c_int, [_vp, C.POINTER(C.c_uint)]),
    "eb2_clear_status": (C.c_int, [_vp]),
    "eb2_synchronize": (C.c_int, [_vp]),
    "eb2_last_error": (C.c_char_p, []),
    "eb2_version": (C.c_char_p, []),
    "eb2_read_control_file": (C.c_int, [C.c_char_p, C.POINTER(Control)]),
}

_lock = threading.Lock()
_lib = None


def library_path() -> str:
    return os.path.join(HERE, _LIB_NAME)


def library() -> C.CDLL:
    """Load libeuler_b200.so (once) and declare every entry point."""
    global _lib
    with _lock:
        if _lib is None:
            path = library_path()
            if not os.path.exists(path):
                raise ImportError(
                    f"{path} is missing: build it with `python -m overheatingproblem_b200.build` "
                    "(the package has no CPU fallback)")
            lib = C.CDLL(path)
            for name, (res, args) in SIGNATURES.items():
                fn = getattr(lib, name)
                fn.restype = res
                fn.argtypes = args
            _lib = lib
        return _lib


def check(rc: int) -> None:
    if rc != EB2_OK:
        msg = library().eb2_last_error().decode(errors="replace")
        raise EB2Error(rc, msg)


def dptr(a):
    """double* of a C-contiguous float64 numpy array."""
    if a.dtype.name != "float64" or not a.flags["C_CONTIGUOUS"]:
        raise TypeError("expected a C-contiguous float64 array")
    return a.ctypes.data_as(_dp)
