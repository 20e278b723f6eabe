"""banana_b200: B200-native 3D FLIP/APIC/AFLIP fluid step, pressure PCG and uniform-grid
neighbour search behind the C ABI in include/banana_b200.h."""
from .capi import (BnnError, FlipBatch, FlipSolver, load, pcg_barrier_probe, pcg_solve_7pt,  # noqa: F401
                   scene_bytes_estimate)

__all__ = ["BnnError", "FlipBatch", "FlipSolver", "load", "pcg_barrier_probe", "pcg_solve_7pt", "scene_bytes_estimate"]
