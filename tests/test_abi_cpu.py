"""The C ABI without a GPU: the library loads, exports every function include/banana_b200.h
declares, its struct layouts match the ctypes binding, and argument validation (the
reference's __BNN_REQUIRE checks, Macros.h:225-233) returns status codes before any CUDA
call."""
import ctypes as C
import re
import subprocess
from pathlib import Path

import pytest

from banana_b200 import build as bld
from banana_b200 import capi

ROOT = Path(__file__).resolve().parent.parent
HEADER = ROOT / "include" / "banana_b200.h"


@pytest.fixture(scope="module")
def lib():
    if not bld.LIB.exists():
        bld.build_cuda()
    return capi.load()


def _declared():
    text = HEADER.read_text()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(bnn_[a-z0-9_]+)\s*\(", text)))


def test_every_declared_symbol_is_exported(lib):
    names = _declared()
    assert len(names) >= 15
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing
    assert set(names) == set(capi.EXPORTS)


def test_struct_layouts_match_binding(tmp_path):
    src = tmp_path / "layout.c"
    fields = {"bnn_params": capi.Params, "bnn_step_stats": capi.StepStats, "bnn_pcg_stats": capi.PcgStats,
              "bnn_batch_params": capi.BatchParams, "bnn_batch_stats": capi.BatchStats,
              "bnn_aniso_params": capi.AnisoParams, "bnn_aniso_stats": capi.AnisoStats,
              "bnn_boundary_object": capi.BoundaryObject}
    lines = ['#include <stdio.h>', '#include <stddef.h>', '#include "banana_b200.h"', "int main(void) {"]
    for cname, py in fields.items():
        lines.append(f'printf("{cname} %zu\\n", sizeof({cname}));')
        for f, _ in py._fields_:
            lines.append(f'printf("{cname}.{f} %zu\\n", offsetof({cname}, {f}));')
    lines.append("return 0; }")
    src.write_text("\n".join(lines))
    exe = tmp_path / "layout"
    subprocess.run(["gcc", "-I", str(ROOT / "include"), str(src), "-o", str(exe)], check=True)
    out = dict(l.split() for l in subprocess.run([str(exe)], capture_output=True, text=True, check=True).stdout.split("\n") if l)
    for cname, py in fields.items():
        assert int(out[cname]) == C.sizeof(py), cname
        for f, _ in py._fields_:
            assert int(out[f"{cname}.{f}"]) == getattr(py, f).offset, (cname, f)


def test_validation_needs_no_gpu(lib):
    assert lib.bnn_version().decode().startswith("banana_b200")
    h = C.c_void_p()
    p = capi.make_params({"cell_size": 0.0})
    assert lib.bnn_flip_create(C.byref(p), C.byref(h)) == capi.STATUS_CODE["INVALID_ARGUMENT"]
    p = capi.make_params({"cell_size": 0.1, "solver_kind": 9})
    assert lib.bnn_flip_create(C.byref(p), C.byref(h)) == capi.STATUS_CODE["NOT_SUPPORTED"]
    p = capi.make_params({"cell_size": 0.1, "box_max": (0.0, 1.0, 1.0)})
    assert lib.bnn_flip_create(C.byref(p), C.byref(h)) == capi.STATUS_CODE["INVALID_ARGUMENT"]
    assert lib.bnn_flip_create(None, C.byref(h)) == capi.STATUS_CODE["INVALID_ARGUMENT"]
    assert lib.bnn_flip_step(None, None) == capi.STATUS_CODE["INVALID_ARGUMENT"]
    assert lib.bnn_neighbors(None, 5, C.c_float(0.1), None, None, 0, None, None) == capi.STATUS_CODE["INVALID_ARGUMENT"]
    assert lib.bnn_cell_sort_noalloc(None, 1 << 21, None, C.c_float(1.0), None, None, None, None, None, None) \
        == capi.STATUS_CODE["INVALID_ARGUMENT"]
    # anisotropic kernels: the reference defaults (AniKernelGenerator.h:41-45,51), and the
    # argument checks that come before any CUDA call
    ap = capi.aniso_params(0.5)
    assert (ap.kernel_ratio, ap.default_spray_size, ap.position_blending, ap.axis_ratio, ap.neighbor_threshold) == \
        (8.0, 0.75, 0.5, 8.0, 25)
    assert lib.bnn_anisotropic_kernels(None, 4, C.byref(ap), None, None, None, None) == \
        capi.STATUS_CODE["INVALID_ARGUMENT"]
    bad = capi.aniso_params(0.0)
    assert lib.bnn_anisotropic_kernels(None, 0, C.byref(bad), None, None, None, None) == \
        capi.STATUS_CODE["INVALID_ARGUMENT"]
    assert lib.bnn_flip_anisotropic_kernels(None, None, None, None, None) == capi.STATUS_CODE["INVALID_ARGUMENT"]
    assert lib.bnn_flip_set_boundaries(None, None, 0, 1) == capi.STATUS_CODE["INVALID_ARGUMENT"]
    st, ms = C.c_int32(0), C.c_float(0.0)
    for lim in (0.0, -1.0, 10.5, float("nan")):
        assert lib.bnn_pcg_barrier_probe(lim, C.byref(st), C.byref(ms)) == capi.STATUS_CODE["INVALID_ARGUMENT"]
    assert lib.bnn_pcg_barrier_probe(0.05, None, None) == capi.STATUS_CODE["INVALID_ARGUMENT"]


def test_missing_library_fails_loudly(monkeypatch, tmp_path):
    monkeypatch.setattr(capi, "_lib", None)
    monkeypatch.setattr(capi, "LIB_PATH", tmp_path / "nope.so")
    with pytest.raises(RuntimeError, match="no CPU fallback"):
        capi.load()


def test_tile_shape_entry_points(lib):
    """bnn_tile_shapes / bnn_set_tile_shape / bnn_tile_tuning need no GPU: the shape table,
    range checks, and the (empty) tuning table with its size protocol."""
    shapes = capi.tile_shapes()
    assert len(shapes) == 6 and shapes[0] == (6, 8) and len(set(shapes)) == 6
    assert lib.bnn_set_tile_shape(len(shapes)) == capi.STATUS_CODE["INVALID_ARGUMENT"]
    assert lib.bnn_set_tile_shape(-2) == capi.STATUS_CODE["INVALID_ARGUMENT"]
    assert lib.bnn_set_tile_shape(2) == 0 and lib.bnn_set_tile_shape(-1) == 0
    need = C.c_size_t()
    assert lib.bnn_tile_tuning(None, 0, C.byref(need)) == capi.STATUS_CODE["CAPACITY"]
    assert need.value >= 1
    assert capi.tile_tuning() == []


def test_batch_mode_validation_needs_no_gpu(lib):
    """bnn_batch_create rejects an unknown step mode before any CUDA call."""
    h = C.c_void_p()
    for mode in (2, 0x200, capi.BATCH_PER_SCENE | 0x400):
        bp = capi.BatchParams(0, 1, mode)
        assert lib.bnn_batch_create(C.byref(bp), C.byref(h)) == capi.STATUS_CODE["INVALID_ARGUMENT"]
