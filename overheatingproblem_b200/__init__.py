"""B200 (sm_100a) implementation of the 2D Euler finite-volume step of
xujf520/OverheatingProblem (src/RP_FVM.c and its headers).

The compute lives in ``libeuler_b200.so`` (CUDA kernels behind the C ABI of
``include/euler_b200.h``); this package is its Python host side:

* :mod:`.lib`    -- ctypes loading of the library; raises if it or a GPU is missing.
* :mod:`.solver` -- :class:`Solver`, one device-resident solve.
* :mod:`.api`    -- the reference's operator API by its own names
  (``Init_Euler_2D``, ``RK3_TimeAd``, ``Get_Delta_T_2D``, ...) on host arrays.
* :mod:`.control`-- ``ReadControlFile`` for the reference's ControlFile.txt.

There is no CPU fallback: every numerical entry point runs on the GPU.
"""
from .lib import EB2Error, library, library_path  # noqa: F401
from .solver import Solver  # noqa: F401

__all__ = ["EB2Error", "Solver", "library", "library_path"]
