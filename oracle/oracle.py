"""ctypes wrapper of the oracle (TEST INFRASTRUCTURE ONLY).

liboracle.so is the CPU restatement of the reference's FLIP step, PCG solver, grid cell
sort and neighbour search (oracle/flip_oracle.cpp).  Only the tests, the smoke check and
bench.py's CPU-baseline leg load it, as the checker / timed CPU baseline.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
SRC = HERE / "flip_oracle.cpp"
SRCS = [SRC, HERE / "aniso_oracle.cpp"]
LIB = HERE / "liboracle.so"

CXXFLAGS = ["-O3", "-march=x86-64-v3", "-ffp-contract=off", "-fno-fast-math", "-fopenmp", "-fPIC", "-shared",
            "-std=c++20"]


def build(force: bool = False) -> Path:
    """Compile the restatement (no FMA contraction: one rounding per float operation)."""
    if force or not LIB.exists() or any(LIB.stat().st_mtime < f.stat().st_mtime for f in SRCS):
        cmd = ["g++", *CXXFLAGS, "-o", str(LIB), *[str(f) for f in SRCS]]
        res = subprocess.run(cmd, capture_output=True, text=True)
        if res.returncode != 0:
            raise RuntimeError("oracle build failed:\n" + res.stderr)
    return LIB


class OrcParams(C.Structure):
    _fields_ = [
        ("box_min", C.c_float * 3), ("box_max", C.c_float * 3), ("cell_size", C.c_float),
        ("n_expand_cells", C.c_uint32), ("cfl_factor", C.c_float), ("min_timestep", C.c_float),
        ("max_timestep", C.c_float), ("frame_duration", C.c_float), ("pic_flip_ratio", C.c_float),
        ("cg_relative_tolerance", C.c_float), ("max_cg_iteration", C.c_uint32), ("advection_steps", C.c_uint32),
        ("reduce_mode", C.c_int32), ("pcg_mode", C.c_int32), ("preconditioner", C.c_int32),
        ("refine_tolerance", C.c_float), ("refine_inner_tolerance", C.c_float), ("sort_each_step", C.c_int32),
        ("nthreads", C.c_int32), ("solver_kind", C.c_int32), ("apply_gravity", C.c_int32),
        ("correct_position", C.c_int32), ("repulsive_force_stiffness", C.c_float),
        ("ratio_cell_size_p_radius", C.c_float),
    ]


class OrcStepStats(C.Structure):
    _fields_ = [
        ("dt", C.c_double), ("frame_time", C.c_double), ("frame_finished", C.c_uint32),
        ("pcg_iterations", C.c_uint32), ("pcg_residual", C.c_double), ("pcg_success", C.c_uint32),
        ("n_active", C.c_uint32), ("outer_iterations", C.c_uint32), ("zero_phi_cells", C.c_uint32),
        ("t_move", C.c_double), ("t_sort", C.c_double), ("t_p2g", C.c_double), ("t_extrap", C.c_double),
        ("t_sdf", C.c_double), ("t_system", C.c_double), ("t_solve", C.c_double), ("t_update", C.c_double),
        ("t_g2p", C.c_double),
    ]


_lib = None


def lib() -> C.CDLL:
    global _lib
    if _lib is None:
        build()
        L = C.CDLL(str(LIB))
        vp = C.c_void_p
        fp = C.POINTER(C.c_float)
        dp = C.POINTER(C.c_double)
        u32p = C.POINTER(C.c_uint32)
        i32p = C.POINTER(C.c_int32)
        u64p = C.POINTER(C.c_uint64)
        L.orc_set_threads.argtypes = [C.c_int]; L.orc_set_threads.restype = C.c_int
        L.orc_create.argtypes = [C.POINTER(OrcParams), C.c_int]; L.orc_create.restype = vp
        L.orc_destroy.argtypes = [vp]; L.orc_destroy.restype = None
        L.orc_grid_dims.argtypes = [vp, i32p]; L.orc_grid_dims.restype = None
        L.orc_set_particles.argtypes = [vp, fp, fp, C.c_uint32]; L.orc_set_particles.restype = None
        L.orc_get_particles.argtypes = [vp, fp, fp]; L.orc_get_particles.restype = None
        L.orc_get_particles_f64.argtypes = [vp, dp, dp]; L.orc_get_particles_f64.restype = None
        L.orc_get_particle_ids.argtypes = [vp, u32p]; L.orc_get_particle_ids.restype = None
        L.orc_get_grid.argtypes = [vp, C.c_int, fp]; L.orc_get_grid.restype = C.c_int
        L.orc_get_grid_f64.argtypes = [vp, C.c_int, dp]; L.orc_get_grid_f64.restype = C.c_int
        L.orc_set_grid.argtypes = [vp, C.c_int, fp]; L.orc_set_grid.restype = C.c_int
        L.orc_step.argtypes = [vp, C.POINTER(OrcStepStats)]; L.orc_step.restype = C.c_int
        L.orc_p2g_only.argtypes = [vp]; L.orc_p2g_only.restype = C.c_int
        L.orc_system_nnz.argtypes = [vp]; L.orc_system_nnz.restype = C.c_uint32
        L.orc_get_system.argtypes = [vp, u32p, u32p, fp, fp]; L.orc_get_system.restype = None
        L.orc_pcg.argtypes = [C.c_uint32, u32p, u32p, fp, fp, C.c_float, C.c_uint32, C.c_int, C.c_int, C.c_float,
                              dp, u32p, dp, u32p]
        L.orc_pcg.restype = C.c_int
        L.orc_dot_canonical_f32.argtypes = [fp, fp, C.c_uint64]; L.orc_dot_canonical_f32.restype = C.c_double
        L.orc_cell_sort.argtypes = [fp, C.c_uint32, fp, C.c_float, i32p, u32p, u32p, u32p]
        L.orc_cell_sort.restype = C.c_uint32
        L.orc_z_sort.argtypes = [fp, C.c_uint32, C.c_float, u64p, u32p]; L.orc_z_sort.restype = None
        L.orc_neighbors.argtypes = [fp, C.c_uint32, C.c_float, u64p, u32p]; L.orc_neighbors.restype = C.c_uint64
        L.orc_grid_neighbor_list.argtypes = [fp, C.c_uint32, fp, C.c_float, i32p, fp, C.c_float, C.c_int, u32p]
        L.orc_grid_neighbor_list.restype = C.c_uint32
        L.orc_grid_ncells.argtypes = [fp, fp, C.c_float, i32p]; L.orc_grid_ncells.restype = None
        L.orc_interp_face.argtypes = [vp, C.c_int, C.c_double, C.c_double, C.c_double]
        L.orc_interp_face.restype = C.c_double
        L.orc_set_boundaries.argtypes = [vp, vp, C.c_uint32, C.c_int]; L.orc_set_boundaries.restype = C.c_int
        L.orc_aniso_kernels.argtypes = [fp, C.c_uint32, fp, C.c_float, i32p, C.c_float, C.c_float, C.c_float,
                                        C.c_float, C.c_float, C.c_uint32, fp, fp]
        L.orc_aniso_kernels.restype = C.c_uint32
        L.orc_cbrt_newton.argtypes = [C.c_double]; L.orc_cbrt_newton.restype = C.c_double
        L.orc_aniso_kernel_matrix.argtypes = [fp, C.c_float, fp]; L.orc_aniso_kernel_matrix.restype = None
        _lib = L
    return _lib


def _p(a: np.ndarray, t):
    return a.ctypes.data_as(C.POINTER(t))


def set_threads(n: int) -> int:
    return lib().orc_set_threads(int(n))


def make_params(cfg: dict) -> OrcParams:
    p = OrcParams()
    p.box_min[:] = cfg.get("box_min", (0.0, 0.0, 0.0))
    p.box_max[:] = cfg.get("box_max", (1.0, 1.0, 1.0))
    p.cell_size = cfg["cell_size"]
    p.n_expand_cells = cfg.get("n_expand_cells", 2)
    p.cfl_factor = cfg.get("cfl_factor", 1.0)
    p.min_timestep = cfg.get("min_timestep", 1e-6)
    p.max_timestep = cfg.get("max_timestep", np.float32(1.0) / np.float32(30.0))
    p.frame_duration = cfg.get("frame_duration", np.float32(1.0 / 30.0))
    p.pic_flip_ratio = cfg.get("pic_flip_ratio", 0.97)
    p.cg_relative_tolerance = cfg.get("cg_relative_tolerance", 1e-6)
    p.max_cg_iteration = cfg.get("max_cg_iteration", 5000)
    p.advection_steps = cfg.get("advection_steps", 1)
    p.reduce_mode = cfg.get("reduce_mode", 1)
    p.pcg_mode = cfg.get("pcg_mode", 0)
    p.preconditioner = cfg.get("preconditioner", 0)
    p.refine_tolerance = cfg.get("refine_tolerance", 1e-8)
    p.refine_inner_tolerance = cfg.get("refine_inner_tolerance", 1e-3)
    p.sort_each_step = cfg.get("sort_each_step", 1)
    p.nthreads = cfg.get("nthreads", 1)
    p.solver_kind = cfg.get("solver_kind", 0)
    p.apply_gravity = cfg.get("apply_gravity", 1)
    p.correct_position = cfg.get("correct_position", 0)
    p.repulsive_force_stiffness = cfg.get("repulsive_force_stiffness", 50.0)
    p.ratio_cell_size_p_radius = cfg.get("ratio_cell_size_p_radius", 2.0)
    return p


class Oracle:
    """One FLIP solver state in the restatement (float, or double for the FP64 build)."""

    def __init__(self, cfg: dict, use_double: bool = False):
        self.L = lib()
        self.params = make_params(cfg)
        self.h = self.L.orc_create(C.byref(self.params), 1 if use_double else 0)
        g = np.zeros(3, np.int32)
        self.L.orc_grid_dims(self.h, _p(g, C.c_int32))
        self.G = tuple(int(x) for x in g)
        self.n = 0

    def close(self):
        if self.h:
            self.L.orc_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def face_shape(self, d: int):
        G = list(self.G)
        G[d] += 1
        return tuple(G)

    def set_particles(self, pos: np.ndarray, vel: np.ndarray):
        pos = np.ascontiguousarray(pos, np.float32)
        vel = np.ascontiguousarray(vel, np.float32)
        self.n = len(pos)
        self.L.orc_set_particles(self.h, _p(pos, C.c_float), _p(vel, C.c_float), self.n)

    def get_particles(self, f64: bool = False):
        if f64:
            pos = np.zeros((self.n, 3), np.float64)
            vel = np.zeros((self.n, 3), np.float64)
            self.L.orc_get_particles_f64(self.h, _p(pos, C.c_double), _p(vel, C.c_double))
        else:
            pos = np.zeros((self.n, 3), np.float32)
            vel = np.zeros((self.n, 3), np.float32)
            self.L.orc_get_particles(self.h, _p(pos, C.c_float), _p(vel, C.c_float))
        return pos, vel

    def particle_ids(self):
        ids = np.zeros(self.n, np.uint32)
        self.L.orc_get_particle_ids(self.h, _p(ids, C.c_uint32))
        return ids

    def grid(self, which: int, f64: bool = False) -> np.ndarray:
        if which in (0, 1, 2):
            shape = self.face_shape(which)
        elif which in (5, 6, 7):
            shape = self.face_shape(which - 5)
        elif which in (9, 10, 11):
            shape = self.face_shape(which - 9)
        elif which == 12:
            shape = tuple(g + 1 for g in self.G)
        else:
            shape = self.G
        n = int(np.prod(shape))
        if f64:
            out = np.zeros(n, np.float64)
            self.L.orc_get_grid_f64(self.h, which, _p(out, C.c_double))
        else:
            out = np.zeros(n, np.float32)
            self.L.orc_get_grid(self.h, which, _p(out, C.c_float))
        return out.reshape(shape[::-1])  # (z, y, x) numpy view of the (k*Sy+j)*Sx+i layout

    def set_grid(self, which: int, arr: np.ndarray):
        a = np.ascontiguousarray(arr, np.float32).ravel()
        self.L.orc_set_grid(self.h, which, _p(a, C.c_float))

    def interp_face(self, d: int, gx: float, gy: float, gz: float) -> float:
        """velocity component d sampled at grid coordinates (PIC_Solver::getVelocityFromGrid)"""
        return self.L.orc_interp_face(self.h, d, gx, gy, gz)

    def set_boundaries(self, objs, update_grid: bool = True) -> None:
        """Boundary objects (ctypes structures with the bnn_boundary_object layout)"""
        if not objs:
            lib().orc_set_boundaries(self.h, None, 0, 0)
            return
        arr = (type(objs[0]) * len(objs))(*objs)
        lib().orc_set_boundaries(self.h, C.cast(arr, C.c_void_p), len(objs), 1 if update_grid else 0)

    def step(self) -> dict:
        st = OrcStepStats()
        self.L.orc_step(self.h, C.byref(st))
        return {f: getattr(st, f) for f, _ in OrcStepStats._fields_}

    def p2g_only(self) -> None:
        """Sort the particles by cell and run P2G alone (grid fields then hold its result)."""
        self.L.orc_p2g_only(self.h)

    def system(self):
        """(rowStart, colIndex, values, rhs) of the last pressure system"""
        nnz = self.L.orc_system_nnz(self.h)
        act = self.grid(8)
        n = int(act.max()) if act.size else 0
        rs = np.zeros(n + 1, np.uint32)
        ci = np.zeros(nnz, np.uint32)
        va = np.zeros(nnz, np.float32)
        rhs = np.zeros(n, np.float32)
        self.L.orc_get_system(self.h, _p(rs, C.c_uint32), _p(ci, C.c_uint32), _p(va, C.c_float), _p(rhs, C.c_float))
        return rs, ci, va, rhs


def pcg(rowStart, colIndex, vals, rhs, tol, max_iter, mode, precond=0, inner_tol=1e-3):
    """Standalone PCG in the restatement: mode 0 canonical FP32, 1 canonical FP64, 2 refined,
    3 reference-order FP32, 4 reference-order FP64."""
    L = lib()
    n = len(rhs)
    rs = np.ascontiguousarray(rowStart, np.uint32)
    ci = np.ascontiguousarray(colIndex, np.uint32)
    va = np.ascontiguousarray(vals, np.float32)
    b = np.ascontiguousarray(rhs, np.float32)
    x = np.zeros(n, np.float64)
    it = C.c_uint32()
    outer = C.c_uint32()
    res = C.c_double()
    rc = L.orc_pcg(n, _p(rs, C.c_uint32), _p(ci, C.c_uint32), _p(va, C.c_float), _p(b, C.c_float), tol, max_iter,
                   mode, precond, inner_tol, _p(x, C.c_double), C.byref(it), C.byref(res), C.byref(outer))
    return x, {"iterations": it.value, "residual": res.value, "success": rc == 0, "outer": outer.value}


def dot_canonical(a: np.ndarray, b: np.ndarray) -> float:
    a = np.ascontiguousarray(a, np.float32)
    b = np.ascontiguousarray(b, np.float32)
    return lib().orc_dot_canonical_f32(_p(a, C.c_float), _p(b, C.c_float), len(a))


def cell_sort(pos, bmin, cell_size, ncells):
    pos = np.ascontiguousarray(pos, np.float32)
    n = len(pos)
    bm = np.ascontiguousarray(bmin, np.float32)
    nc = np.ascontiguousarray(ncells, np.int32)
    cid = np.zeros(n, np.uint32)
    srt = np.zeros(n, np.uint32)
    start = np.zeros(int(np.prod(nc.astype(np.int64))) + 1, np.uint32)
    oor = lib().orc_cell_sort(_p(pos, C.c_float), n, _p(bm, C.c_float), cell_size, _p(nc, C.c_int32),
                              _p(cid, C.c_uint32), _p(srt, C.c_uint32), _p(start, C.c_uint32))
    return cid, srt, start, oor


def z_sort(pos, radius):
    pos = np.ascontiguousarray(pos, np.float32)
    n = len(pos)
    z = np.zeros(n, np.uint64)
    perm = np.zeros(n, np.uint32)
    lib().orc_z_sort(_p(pos, C.c_float), n, radius, _p(z, C.c_uint64), _p(perm, C.c_uint32))
    return z, perm


def neighbors(pos, radius):
    pos = np.ascontiguousarray(pos, np.float32)
    n = len(pos)
    L = lib()
    total = L.orc_neighbors(_p(pos, C.c_float), n, radius, None, None)
    off = np.zeros(n + 1, np.uint64)
    idx = np.zeros(max(int(total), 1), np.uint32)
    L.orc_neighbors(_p(pos, C.c_float), n, radius, _p(off, C.c_uint64), _p(idx, C.c_uint32))
    return off, idx[: int(total)]


def grid_ncells(bmin, bmax, cell_size):
    out = np.zeros(3, np.int32)
    lib().orc_grid_ncells(_p(np.ascontiguousarray(bmin, np.float32), C.c_float),
                          _p(np.ascontiguousarray(bmax, np.float32), C.c_float), cell_size, _p(out, C.c_int32))
    return tuple(int(x) for x in out)


def grid_neighbor_list(pos, bmin, cell_size, ncells, q, d2=None):
    pos = np.ascontiguousarray(pos, np.float32)
    out = np.zeros(max(len(pos), 1), np.uint32)
    qq = np.ascontiguousarray(q, np.float32)
    n = lib().orc_grid_neighbor_list(_p(pos, C.c_float), len(pos), _p(np.ascontiguousarray(bmin, np.float32), C.c_float),
                                     cell_size, _p(np.ascontiguousarray(ncells, np.int32), C.c_int32),
                                     _p(qq, C.c_float), 0.0 if d2 is None else d2, 0 if d2 is None else 1,
                                     _p(out, C.c_uint32))
    return out[:n]


def aniso_kernels(pos, bmin, cell_size, ncells, particle_radius, kernel_ratio=8.0, spray=0.75, blend=0.5,
                  axis_ratio=8.0, threshold=25):
    """AnisotropicKernelGenerator::computeAniKernels in the canonical order of the cell grid
    (bmin, cell_size, ncells).  Returns (centers n x 3, matrices n x 9 column-major, sprays)."""
    pos = np.ascontiguousarray(pos, np.float32)
    n = len(pos)
    cen = np.zeros((n, 3), np.float32)
    mat = np.zeros((n, 9), np.float32)
    sprays = lib().orc_aniso_kernels(_p(pos, C.c_float), n, _p(np.ascontiguousarray(bmin, np.float32), C.c_float),
                                     float(cell_size), _p(np.ascontiguousarray(ncells, np.int32), C.c_int32),
                                     float(particle_radius), float(kernel_ratio), float(spray), float(blend),
                                     float(axis_ratio), int(threshold), _p(cen, C.c_float), _p(mat, C.c_float))
    return cen, mat, int(sprays)


def cbrt_newton(y: float) -> float:
    return lib().orc_cbrt_newton(float(y))


def aniso_kernel_matrix(cov, axis_ratio=8.0):
    """Kernel matrix (column-major 9) of one covariance matrix (3 x 3)."""
    c = np.ascontiguousarray(np.asarray(cov, np.float32).T.reshape(9))
    out = np.zeros(9, np.float32)
    lib().orc_aniso_kernel_matrix(_p(c, C.c_float), float(axis_ratio), _p(out, C.c_float))
    return out
