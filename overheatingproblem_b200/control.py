"""ControlFile.txt-driven setup: ``ReadControlFile`` of src/RP_FVM.c:382-589,
implemented in C in the library (eb2_read_control_file), and the mapping of
its parameters onto a :class:`~overheatingproblem_b200.Solver`."""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass

from . import lib as L

# TestCase2D enumerators (include/Golbal.h:8-30 of the reference)
TEST_CASE_NAMES = {
    0: "Precision_Test", 1: "1D_Sod_Shocktube", 2: "1D_Contact_Wave", 3: "1D_Shock_Impact",
    4: "1D_Impact_Wall", 5: "1D_Double_Rarefaction", 6: "1D_Noh_Problem",
    7: "2D_Riemann_Case1", 8: "2D_Riemann_Case2", 9: "2D_Riemann_Case3",
    10: "2D_Riemann_Case4", 11: "2D_Riemann_Case5", 12: "Taylor_Green_Vortex",
    13: "Gaussian_Pulse", 14: "Kelvin_Helmholtz", 15: "Rayleigh_Taylor",
    16: "Double_Mach_Reflection", 17: "Blast_Wave", 18: "2D_Noh_Problem",
    19: "Odd_Even_Decoupling", 20: "Backward_Step",
}


@dataclass
class ControlParams:
    """ControlParams, src/RP_FVM.c:66-82."""
    test_case: int
    L_nx: int
    L_ny: int
    Time_ADM: int
    scheme: int
    M_gamma: float
    Source: int
    Gravity: float
    CFL: float
    Tmax: float
    Control_Compution: int
    Control_output: int
    Recon_Accur: int
    Characteriz: int
    output_dir: str


def ReadControlFile(path: str) -> ControlParams:  # noqa: N802 - the reference's name
    c = L.Control()
    L.check(L.library().eb2_read_control_file(path.encode(), C.byref(c)))
    return ControlParams(c.test_case, c.L_nx, c.L_ny, c.Time_ADM, c.scheme, c.M_gamma,
                         c.Source, c.Gravity, c.CFL, c.Tmax, c.Control_Compution,
                         c.Control_output, c.Recon_Accur, c.Characteriz,
                         c.output_dir.decode(errors="replace"))


def solver_options(c: ControlParams, honour_recon_keys: bool = False) -> dict:
    """Reconstruction and time-stepping options implied by a control file.

    The reference parses Recon_Accur and Characteriz but never copies them to
    the globals its kernels read (src/RP_FVM.c:600-605 sets only gamma,
    source, gravity and CFL; include/Golbal.h:58,60 fix WENO5 component-wise).
    The same holds here unless ``honour_recon_keys`` is set."""
    if honour_recon_keys:
        recon, ch = c.Recon_Accur, bool(c.Characteriz)
    else:
        recon, ch = 5, False
    return {"recon": recon, "characteristic": ch, "order": c.Time_ADM, "scheme": c.scheme}
