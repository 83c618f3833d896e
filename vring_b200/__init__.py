"""vring_b200: the RK3 fractional-step core of vring (cylindrical vortex-ring
Navier-Stokes solver) on one B200, behind a C ABI (include/vring_b200.h)
that mirrors the reference's Fortran subroutine surface."""
from .api import (FIELD_ID, LIB_PATH, Ensemble, K2d, Part, Run, UNet, VrError, autotune, declared_symbols, lib,
                  set_tiles, solve_lap_bthom, solve_lap_thom)

__all__ = ["Run", "Part", "Ensemble", "autotune", "set_tiles", "K2d", "UNet", "VrError", "lib", "LIB_PATH", "FIELD_ID", "declared_symbols",
           "solve_lap_thom", "solve_lap_bthom"]
