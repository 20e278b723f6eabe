"""ctypes binding of libbanana_b200.so (the C ABI declared in include/banana_b200.h).

This is the reference-facing surface the tests and the benchmark drive.  It loads the
in-tree CUDA library and raises if it is missing: there is no CPU path behind it.
"""
from __future__ import annotations

import ctypes as C
import os
from pathlib import Path

import numpy as np

PKG = Path(__file__).resolve().parent
LIB_PATH = Path(os.environ.get("BNN_LIB", str(PKG / "libbanana_b200.so")))

BNN_OK = 0
STATUS = {0: "OK", 1: "INVALID_ARGUMENT", 2: "OUT_OF_MEMORY", 3: "PCG_NOT_CONVERGED", 4: "DEVICE_CHECK",
          5: "TIMEOUT", 6: "CUDA", 7: "NOT_SUPPORTED", 8: "CAPACITY"}
STATUS_CODE = {v: k for k, v in STATUS.items()}
SOLVER_KIND = {"FLIP": 0, "APIC": 1, "AFLIP": 2, "PIC": 3}
PCG_MODE = {"fp32": 0, "fp64": 1, "refined": 2}
# OR-ed into a PCG mode: the single-reduction form of the iteration instead of the default
# PCGSolver::solve_precond step order (include/banana_b200.h BNN_PCG_SINGLE_REDUCTION)
PCG_SINGLE_REDUCTION = 0x10
FIELD = {"u": 0, "v": 1, "w": 2, "phi": 3, "pressure": 4, "old_u": 5, "old_v": 6, "old_w": 7, "active": 8,
         "weight_u": 9, "weight_v": 10, "weight_w": 11, "boundary_sdf": 12}
GEOMETRY = {"box": 0, "sphere": 1}

# Exported symbols of the C ABI (every one is declared in include/banana_b200.h)
EXPORTS = [
    "bnn_flip_create", "bnn_flip_destroy", "bnn_flip_grid_dims", "bnn_flip_set_particles", "bnn_flip_get_particles",
    "bnn_flip_num_particles", "bnn_flip_get_grid", "bnn_flip_step", "bnn_flip_advance_frame",
    "bnn_flip_device_particles", "bnn_flip_step_host", "bnn_flip_stream", "bnn_cell_sort", "bnn_cell_sort_noalloc", "bnn_z_sort", "bnn_neighbors",
    "bnn_pcg_solve_7pt", "bnn_pcg_barrier_probe", "bnn_version", "bnn_last_error", "bnn_launch_count",
    "bnn_flip_device_bytes", "bnn_scene_bytes_estimate", "bnn_flip_set_grid",
    "bnn_batch_create", "bnn_batch_destroy", "bnn_batch_add_scene", "bnn_batch_remove_scene", "bnn_batch_step",
    "bnn_batch_scene_info", "bnn_batch_get_scene", "bnn_batch_memory",
    "bnn_aniso_default_params", "bnn_anisotropic_kernels", "bnn_flip_anisotropic_kernels",
    "bnn_flip_set_boundaries", "bnn_tile_shapes", "bnn_set_tile_shape", "bnn_tile_tuning",
]


class BnnError(RuntimeError):
    def __init__(self, code: int, what: str):
        super().__init__(f"{what} failed: {STATUS.get(code, code)} ({code}) {last_error()}")
        self.code = code


class Params(C.Structure):
    _fields_ = [
        ("box_min", C.c_float * 3), ("box_max", C.c_float * 3), ("cell_size", C.c_float),
        ("n_expand_cells", C.c_uint32), ("cfl_factor", C.c_float), ("min_timestep", C.c_float),
        ("max_timestep", C.c_float), ("frame_duration", C.c_float), ("pic_flip_ratio", C.c_float),
        ("cg_relative_tolerance", C.c_float), ("max_cg_iteration", C.c_uint32), ("advection_steps", C.c_uint32),
        ("solver_kind", C.c_int32), ("pcg_mode", C.c_int32), ("preconditioner", C.c_int32),
        ("refine_tolerance", C.c_float), ("refine_inner_tolerance", C.c_float), ("apply_gravity", C.c_int32),
        ("max_particles", C.c_uint32), ("correct_position", C.c_int32), ("repulsive_force_stiffness", C.c_float),
        ("ratio_cell_size_p_radius", C.c_float),
    ]


class StepStats(C.Structure):
    _fields_ = [
        ("dt", C.c_double), ("frame_time", C.c_double), ("frame_finished", C.c_uint32),
        ("pcg_iterations", C.c_uint32), ("pcg_residual", C.c_double), ("pcg_success", C.c_uint32),
        ("n_active", C.c_uint32), ("outer_iterations", C.c_uint32), ("zero_phi_cells", C.c_uint32),
        ("stage_ms", C.c_float * 10), ("device_flags", C.c_uint32), ("pcg_kernel_ms", C.c_float),
    ]


BATCH_STAGED = 0      # BNN_BATCH_STAGED: one launch per stage over the scenes it takes
BATCH_PER_SCENE = 1   # BNN_BATCH_PER_SCENE: every scene on its own stream
BATCH_NO_GRAPHS = 0x100  # BNN_BATCH_NO_GRAPHS: the staged step without CUDA-graph replay


class BatchParams(C.Structure):
    _fields_ = [("hbm_budget_bytes", C.c_uint64), ("worker_threads", C.c_uint32), ("step_mode", C.c_uint32)]


class BatchStats(C.Structure):
    _fields_ = [("scenes", C.c_uint32), ("failed", C.c_uint32), ("particle_steps", C.c_uint64),
                ("pcg_iterations", C.c_uint64), ("wall_ms", C.c_double), ("max_scene_ms", C.c_double),
                ("staged_scenes", C.c_uint32), ("graph_instantiations", C.c_uint16),
                ("graph_updates", C.c_uint16)]


class PcgStats(C.Structure):
    _fields_ = [("iterations", C.c_uint32), ("outer_iterations", C.c_uint32), ("residual", C.c_double),
                ("success", C.c_uint32), ("ms", C.c_float)]


class BoundaryObject(C.Structure):
    """bnn_boundary_object: a box / sphere the fluid stays inside, with its current
    world-to-object map (rows of a 3x4 affine matrix) and uniform scale."""
    _fields_ = [("geometry", C.c_int32), ("dynamic", C.c_int32), ("box_min", C.c_float * 3),
                ("box_max", C.c_float * 3), ("inv_transform", C.c_float * 12), ("uniform_scale", C.c_float),
                ("transformed", C.c_int32)]


def boundary_object(geometry: str, box_min=(0, 0, 0), box_max=(0, 0, 0), translation=None, axis_angle=None,
                    scale=None, dynamic: bool = False) -> BoundaryObject:
    """A boundary object with GeometryObject's transformation translate * rotate * scale
    (Animation.h:199-231); axis_angle = (ax, ay, az, angle in radians)."""
    o = BoundaryObject()
    o.geometry = GEOMETRY[geometry]
    o.dynamic = 1 if dynamic else 0
    for d in range(3):
        o.box_min[d] = float(box_min[d])
        o.box_max[d] = float(box_max[d])
    transformed = translation is not None or axis_angle is not None or scale is not None
    T = np.eye(4)
    if translation is not None:
        T[:3, 3] = np.asarray(translation, np.float64)
    Rm = np.eye(4)
    if axis_angle is not None and float(axis_angle[3]) != 0.0:
        a = np.asarray(axis_angle[:3], np.float64)
        a = a / np.linalg.norm(a)
        c, sn = np.cos(float(axis_angle[3])), np.sin(float(axis_angle[3]))
        K = np.array([[0, -a[2], a[1]], [a[2], 0, -a[0]], [-a[1], a[0], 0]])
        Rm[:3, :3] = c * np.eye(3) + sn * K + (1 - c) * np.outer(a, a)
    sc = 1.0 if scale is None else float(scale)
    S = np.diag([sc, sc, sc, 1.0])
    inv = np.linalg.inv(T @ Rm @ S)
    M = inv[:3, :4].astype(np.float32).reshape(-1)
    for q in range(12):
        o.inv_transform[q] = float(M[q])
    o.uniform_scale = sc
    o.transformed = 1 if transformed else 0
    return o


class AnisoParams(C.Structure):
    _fields_ = [("particle_radius", C.c_float), ("kernel_ratio", C.c_float), ("default_spray_size", C.c_float),
                ("position_blending", C.c_float), ("axis_ratio", C.c_float), ("neighbor_threshold", C.c_uint32)]


class AnisoStats(C.Structure):
    _fields_ = [("grid_bmin", C.c_float * 3), ("grid_cell_size", C.c_float), ("grid_dims", C.c_int32 * 3),
                ("sprays", C.c_uint32), ("ms", C.c_float)]


STAGES = ["move", "sort", "p2g", "extrapolate", "fluid_sdf", "system", "pcg", "update", "g2p", "step"]

_lib = None


def load() -> C.CDLL:
    """Load the in-tree CUDA library (fails loudly when it has not been built)."""
    global _lib
    if _lib is not None:
        return _lib
    if not LIB_PATH.exists():
        raise RuntimeError(f"{LIB_PATH} is missing: run banana_b200.build.build() first (no CPU fallback exists)")
    L = C.CDLL(str(LIB_PATH))
    vp = C.c_void_p
    fp = C.POINTER(C.c_float)
    dp = C.POINTER(C.c_double)
    u32p = C.POINTER(C.c_uint32)
    i32p = C.POINTER(C.c_int32)
    u64p = C.POINTER(C.c_uint64)
    L.bnn_flip_create.argtypes = [C.POINTER(Params), C.POINTER(vp)]
    L.bnn_flip_destroy.argtypes = [vp]
    L.bnn_flip_grid_dims.argtypes = [vp, i32p]
    L.bnn_flip_set_particles.argtypes = [vp, fp, fp, C.c_uint32]
    L.bnn_flip_get_particles.argtypes = [vp, fp, fp]
    L.bnn_flip_num_particles.argtypes = [vp, u32p]
    L.bnn_flip_get_grid.argtypes = [vp, C.c_int32, fp, C.c_size_t]
    L.bnn_flip_step.argtypes = [vp, C.POINTER(StepStats)]
    L.bnn_flip_advance_frame.argtypes = [vp, u32p]
    L.bnn_flip_device_particles.argtypes = [vp, C.POINTER(fp), C.POINTER(u32p)]
    L.bnn_flip_step_host.argtypes = [vp, fp, fp, C.POINTER(StepStats)]
    L.bnn_flip_stream.argtypes = [vp, C.POINTER(vp)]
    L.bnn_cell_sort.argtypes = [vp, C.c_uint32, fp, C.c_float, i32p, vp, vp, vp, u32p, vp]
    L.bnn_cell_sort_noalloc.argtypes = [vp, C.c_uint32, fp, C.c_float, i32p, vp, vp, vp, u32p, vp]
    L.bnn_z_sort.argtypes = [vp, C.c_uint32, C.c_float, vp, vp, vp]
    L.bnn_neighbors.argtypes = [vp, C.c_uint32, C.c_float, vp, vp, C.c_uint64, u64p, vp]
    L.bnn_pcg_solve_7pt.argtypes = [C.c_uint32, fp, i32p, C.c_float, fp, C.c_float, C.c_uint32, C.c_int32, C.c_float,
                                    dp, C.POINTER(PcgStats)]
    L.bnn_pcg_barrier_probe.argtypes = [C.c_float, i32p, fp]
    L.bnn_flip_device_bytes.argtypes = [vp, u64p]
    L.bnn_flip_set_grid.argtypes = [vp, C.c_int32, fp, C.c_size_t]
    L.bnn_scene_bytes_estimate.argtypes = [C.POINTER(Params), C.c_uint32, u64p]
    L.bnn_batch_create.argtypes = [C.POINTER(BatchParams), C.POINTER(vp)]
    L.bnn_batch_destroy.argtypes = [vp]
    L.bnn_batch_add_scene.argtypes = [vp, C.POINTER(Params), fp, fp, C.c_uint32, u32p]
    L.bnn_batch_remove_scene.argtypes = [vp, C.c_uint32]
    L.bnn_batch_step.argtypes = [vp, C.POINTER(BatchStats)]
    L.bnn_batch_scene_info.argtypes = [vp, C.c_uint32, u32p, u64p, C.POINTER(StepStats)]
    L.bnn_batch_get_scene.argtypes = [vp, C.c_uint32, fp, fp]
    L.bnn_batch_memory.argtypes = [vp, u64p, u64p]
    L.bnn_flip_set_boundaries.argtypes = [vp, C.POINTER(BoundaryObject), C.c_uint32, C.c_int32]
    L.bnn_tile_shapes.argtypes = [i32p, i32p, C.c_int32]
    L.bnn_set_tile_shape.argtypes = [C.c_int32]
    L.bnn_tile_tuning.argtypes = [C.c_char_p, C.c_size_t, C.POINTER(C.c_size_t)]
    L.bnn_aniso_default_params.argtypes = [C.c_float, C.POINTER(AnisoParams)]
    L.bnn_anisotropic_kernels.argtypes = [vp, C.c_uint32, C.POINTER(AnisoParams), vp, vp, C.POINTER(AnisoStats), vp]
    L.bnn_flip_anisotropic_kernels.argtypes = [vp, C.POINTER(AnisoParams), fp, fp, C.POINTER(AnisoStats)]
    L.bnn_launch_count.argtypes = []
    L.bnn_launch_count.restype = C.c_uint64
    L.bnn_version.restype = C.c_char_p
    L.bnn_last_error.restype = C.c_char_p
    for name in EXPORTS:
        if name not in ("bnn_version", "bnn_last_error", "bnn_launch_count"):
            getattr(L, name).restype = C.c_int
    _lib = L
    return L


def tile_shapes() -> list:
    """(tz, yc) of every tile shape of the FLIP P2G + fluid SDF pass (bnn_tile_shapes)."""
    L = load()
    n = int(L.bnn_tile_shapes(None, None, 0))
    tz, yc = (C.c_int32 * n)(), (C.c_int32 * n)()
    L.bnn_tile_shapes(tz, yc, n)
    return [(int(tz[i]), int(yc[i])) for i in range(n)]


def set_tile_shape(shape: int) -> None:
    """Use one tile shape for every launch of the process (-1: tune per launch kind)."""
    L = load()
    check(L.bnn_set_tile_shape(int(shape)), "bnn_set_tile_shape")


def tile_tuning() -> list:
    """The tuner's choices so far, one dict per tuned launch kind (bnn_tile_tuning)."""
    import json
    L = load()
    need = C.c_size_t()
    L.bnn_tile_tuning(None, 0, C.byref(need))
    buf = C.create_string_buffer(int(need.value))
    check(L.bnn_tile_tuning(buf, len(buf), C.byref(need)), "bnn_tile_tuning")
    return [json.loads(line) for line in buf.value.decode().splitlines() if line.strip()]


def launch_count() -> int:
    """Kernels launched by libbanana_b200 so far in this process."""
    return int(load().bnn_launch_count())


def last_error() -> str:
    try:
        return (load().bnn_last_error() or b"").decode()
    except Exception:
        return ""


def check(code: int, what: str) -> None:
    if code != BNN_OK:
        raise BnnError(code, what)


def _p(a: np.ndarray, t):
    return a.ctypes.data_as(C.POINTER(t))


def make_params(cfg: dict) -> Params:
    p = Params()
    p.box_min[:] = cfg.get("box_min", (0.0, 0.0, 0.0))
    p.box_max[:] = cfg.get("box_max", (1.0, 1.0, 1.0))
    p.cell_size = cfg["cell_size"]
    p.n_expand_cells = cfg.get("n_expand_cells", 2)
    p.cfl_factor = cfg.get("cfl_factor", 1.0)
    p.min_timestep = cfg.get("min_timestep", 1e-6)
    p.max_timestep = cfg.get("max_timestep", float(np.float32(1.0) / np.float32(30.0)))
    p.frame_duration = cfg.get("frame_duration", float(np.float32(1.0 / 30.0)))
    p.pic_flip_ratio = cfg.get("pic_flip_ratio", 0.97)
    p.cg_relative_tolerance = cfg.get("cg_relative_tolerance", 1e-6)
    p.max_cg_iteration = cfg.get("max_cg_iteration", 5000)
    p.advection_steps = cfg.get("advection_steps", 1)
    p.solver_kind = cfg.get("solver_kind", 0)
    p.pcg_mode = cfg.get("pcg_mode", 0)
    p.preconditioner = cfg.get("preconditioner", 0)
    p.refine_tolerance = cfg.get("refine_tolerance", 1e-8)
    p.refine_inner_tolerance = cfg.get("refine_inner_tolerance", 1e-2)
    p.apply_gravity = cfg.get("apply_gravity", 1)
    p.max_particles = cfg.get("max_particles", 0)
    p.correct_position = cfg.get("correct_position", 0)
    p.repulsive_force_stiffness = cfg.get("repulsive_force_stiffness", 50.0)
    p.ratio_cell_size_p_radius = cfg.get("ratio_cell_size_p_radius", 2.0)
    return p


class FlipSolver:
    """One device-resident FLIP/APIC/AFLIP scene behind the C ABI."""

    def __init__(self, cfg: dict):
        self.L = load()
        self.cfg = dict(cfg)
        self.params = make_params(cfg)
        h = C.c_void_p()
        check(self.L.bnn_flip_create(C.byref(self.params), C.byref(h)), "bnn_flip_create")
        self.h = h
        g = np.zeros(3, np.int32)
        check(self.L.bnn_flip_grid_dims(self.h, _p(g, C.c_int32)), "bnn_flip_grid_dims")
        self.G = tuple(int(x) for x in g)
        self.n = 0

    def close(self):
        if getattr(self, "h", None):
            self.L.bnn_flip_destroy(self.h)
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
        check(self.L.bnn_flip_set_particles(self.h, _p(pos, C.c_float), _p(vel, C.c_float), self.n),
              "bnn_flip_set_particles")

    def get_particles(self):
        pos = np.zeros((self.n, 3), np.float32)
        vel = np.zeros((self.n, 3), np.float32)
        check(self.L.bnn_flip_get_particles(self.h, _p(pos, C.c_float), _p(vel, C.c_float)), "bnn_flip_get_particles")
        return pos, vel

    def grid(self, field) -> np.ndarray:
        which = FIELD[field] if isinstance(field, str) else int(field)
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
        out = np.zeros(int(np.prod(shape)), np.float32)
        check(self.L.bnn_flip_get_grid(self.h, which, _p(out, C.c_float), out.size), "bnn_flip_get_grid")
        return out.reshape(shape[::-1])

    def step(self, allow_fail: bool = False) -> dict:
        st = StepStats()
        rc = self.L.bnn_flip_step(self.h, C.byref(st))
        d = {f: getattr(st, f) for f, _ in StepStats._fields_ if f != "stage_ms"}
        d["stage_ms"] = dict(zip(STAGES, list(st.stage_ms)))
        d["status"] = rc
        if rc != BNN_OK and not allow_fail:
            raise BnnError(rc, "bnn_flip_step")
        return d

    def step_host(self, pos: np.ndarray, vel: np.ndarray) -> dict:
        st = StepStats()
        check(self.L.bnn_flip_step_host(self.h, _p(pos, C.c_float), _p(vel, C.c_float), C.byref(st)),
              "bnn_flip_step_host")
        d = {f: getattr(st, f) for f, _ in StepStats._fields_ if f != "stage_ms"}
        d["stage_ms"] = dict(zip(STAGES, list(st.stage_ms)))
        return d

    def stream_ptr(self) -> int:
        """cudaStream_t of this handle (all its kernels run on it)"""
        s = C.c_void_p()
        check(self.L.bnn_flip_stream(self.h, C.byref(s)), "bnn_flip_stream")
        return int(s.value or 0)

    def step_host_ptr(self, pos_ptr: int, vel_ptr: int) -> dict:
        """bnn_flip_step_host on raw (pinned) host pointers"""
        st = StepStats()
        check(self.L.bnn_flip_step_host(self.h, C.cast(pos_ptr, C.POINTER(C.c_float)),
                                        C.cast(vel_ptr, C.POINTER(C.c_float)), C.byref(st)), "bnn_flip_step_host")
        d = {f: getattr(st, f) for f, _ in StepStats._fields_ if f != "stage_ms"}
        d["stage_ms"] = dict(zip(STAGES, list(st.stage_ms)))
        return d

    def advance_frame(self) -> int:
        k = C.c_uint32()
        check(self.L.bnn_flip_advance_frame(self.h, C.byref(k)), "bnn_flip_advance_frame")
        return k.value

    def set_boundaries(self, objs, update_grid: bool = True) -> None:
        """Boundary objects besides the domain box (bnn_flip_set_boundaries)"""
        arr = (BoundaryObject * max(len(objs), 1))(*objs)
        check(self.L.bnn_flip_set_boundaries(self.h, arr, len(objs), 1 if update_grid else 0),
              "bnn_flip_set_boundaries")

    def anisotropic_kernels(self, params: dict | None = None):
        """Kernel centres (n x 3) and matrices (n x 9, column-major) of the current
        particles, in the order they were given, plus the pass statistics."""
        cen = np.zeros((self.n, 3), np.float32)
        mat = np.zeros((self.n, 9), np.float32)
        st = AnisoStats()
        prm = aniso_params(**params) if params else None
        check(self.L.bnn_flip_anisotropic_kernels(self.h, C.byref(prm) if prm is not None else None,
                                                  _p(cen, C.c_float), _p(mat, C.c_float), C.byref(st)),
              "bnn_flip_anisotropic_kernels")
        return cen, mat, aniso_stats_dict(st)


def aniso_params(particle_radius: float = 0.0, **kw) -> AnisoParams:
    """AnisotropicKernelGenerator parameters: the reference defaults, overridden by kw"""
    p = AnisoParams()
    check(load().bnn_aniso_default_params(float(particle_radius), C.byref(p)), "bnn_aniso_default_params")
    for k, v in kw.items():
        setattr(p, k, v)
    return p


def aniso_stats_dict(st: AnisoStats) -> dict:
    return {"grid_bmin": list(st.grid_bmin), "grid_cell_size": st.grid_cell_size, "grid_dims": list(st.grid_dims),
            "sprays": st.sprays, "ms": st.ms}


def anisotropic_kernels_dev(pos_ptr: int, n: int, params: AnisoParams, cen_ptr: int, mat_ptr: int,
                            stream: int = 0) -> dict:
    """bnn_anisotropic_kernels on device pointers (AoS float32 points in, centres n x 3 and
    matrices n x 9 out)."""
    st = AnisoStats()
    check(load().bnn_anisotropic_kernels(C.c_void_p(pos_ptr), n, C.byref(params), C.c_void_p(cen_ptr),
                                         C.c_void_p(mat_ptr), C.byref(st), C.c_void_p(stream)),
          "bnn_anisotropic_kernels")
    return aniso_stats_dict(st)


def pcg_solve_7pt(diag, nbr, offdiag, rhs, tol, max_iter, mode="fp32", inner_tol=1e-3):
    L = load()
    n = len(rhs)
    d = np.ascontiguousarray(diag, np.float32)
    nb = np.ascontiguousarray(nbr, np.int32).reshape(-1)
    b = np.ascontiguousarray(rhs, np.float32)
    x = np.zeros(max(n, 1), np.float64)
    st = PcgStats()
    m = PCG_MODE[mode] if isinstance(mode, str) else int(mode)
    rc = L.bnn_pcg_solve_7pt(n, _p(d, C.c_float), _p(nb, C.c_int32), offdiag, _p(b, C.c_float), tol, max_iter, m,
                             inner_tol, _p(x, C.c_double), C.byref(st))
    if rc not in (BNN_OK, 3):
        raise BnnError(rc, "bnn_pcg_solve_7pt")
    return x[:n], {f: getattr(st, f) for f, _ in PcgStats._fields_}


def pcg_barrier_probe(limit_seconds: float = 0.05):
    """Self-test of the bounded PCG barrier wait (bnn_pcg_barrier_probe): one block waits at
    a barrier sized for two until the wait gives up.  Returns (status, elapsed_ms); status
    is STATUS_CODE["TIMEOUT"] when the wait gave up as designed."""
    st = C.c_int32(-1)
    ms = C.c_float(0.0)
    check(load().bnn_pcg_barrier_probe(C.c_float(limit_seconds), C.byref(st), C.byref(ms)), "bnn_pcg_barrier_probe")
    return int(st.value), float(ms.value)


def scene_bytes_estimate(cfg: dict, n: int) -> int:
    """Device bytes a scene with these parameters and n particles is expected to hold."""
    b = C.c_uint64()
    p = make_params(cfg)
    check(load().bnn_scene_bytes_estimate(C.byref(p), int(n), C.byref(b)), "bnn_scene_bytes_estimate")
    return int(b.value)


class FlipBatch:
    """Many independent scenes on one GPU (bnn_batch_*): every scene computes what a lone
    FlipSolver computes; step() advances all of them by one sub-step."""

    def __init__(self, hbm_budget_bytes: int = 0, worker_threads: int = 0, step_mode: int = BATCH_STAGED):
        self.L = load()
        bp = BatchParams(int(hbm_budget_bytes), int(worker_threads), int(step_mode))
        h = C.c_void_p()
        check(self.L.bnn_batch_create(C.byref(bp), C.byref(h)), "bnn_batch_create")
        self.h = h
        self.n = {}

    def close(self):
        if self.h:
            self.L.bnn_batch_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def add_scene(self, cfg: dict, pos, vel) -> int:
        """Admit a scene; raises BnnError(CAPACITY) when it does not fit the budget."""
        pos = np.ascontiguousarray(pos, np.float32)
        vel = np.ascontiguousarray(vel, np.float32)
        p = make_params(cfg)
        sid = C.c_uint32()
        check(self.L.bnn_batch_add_scene(self.h, C.byref(p), _p(pos, C.c_float), _p(vel, C.c_float), len(pos),
                                         C.byref(sid)), "bnn_batch_add_scene")
        self.n[sid.value] = len(pos)
        return int(sid.value)

    def remove_scene(self, sid: int) -> None:
        check(self.L.bnn_batch_remove_scene(self.h, int(sid)), "bnn_batch_remove_scene")
        self.n.pop(sid, None)

    def step(self, allow_fail: bool = False) -> dict:
        st = BatchStats()
        rc = self.L.bnn_batch_step(self.h, C.byref(st))
        if rc != BNN_OK and not allow_fail:
            raise BnnError(rc, "bnn_batch_step")
        return {f: getattr(st, f) for f, _ in BatchStats._fields_}

    def scene_info(self, sid: int) -> dict:
        n = C.c_uint32()
        steps = C.c_uint64()
        st = StepStats()
        rc = self.L.bnn_batch_scene_info(self.h, int(sid), C.byref(n), C.byref(steps), C.byref(st))
        d = {f: getattr(st, f) for f, _ in StepStats._fields_ if f != "stage_ms"}
        d["stage_ms"] = dict(zip(STAGES, list(st.stage_ms)))
        d.update(n=int(n.value), steps=int(steps.value), status=int(rc))
        return d

    def get_scene(self, sid: int):
        n = self.n[sid]
        pos = np.zeros((max(n, 1), 3), np.float32)
        vel = np.zeros((max(n, 1), 3), np.float32)
        check(self.L.bnn_batch_get_scene(self.h, int(sid), _p(pos, C.c_float), _p(vel, C.c_float)),
              "bnn_batch_get_scene")
        return pos[:n], vel[:n]

    def memory(self) -> tuple[int, int]:
        a = C.c_uint64()
        b = C.c_uint64()
        check(self.L.bnn_batch_memory(self.h, C.byref(a), C.byref(b)), "bnn_batch_memory")
        return int(a.value), int(b.value)
