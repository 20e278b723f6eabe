"""banana_b200: B200-native 3D FLIP/APIC/AFLIP fluid step, pressure PCG and uniform-grid
neighbour search behind the C ABI in include/banana_b200.h."""
from .capi import FlipSolver, load, pcg_solve_7pt  # noqa: F401

__all__ = ["FlipSolver", "load", "pcg_solve_7pt"]
