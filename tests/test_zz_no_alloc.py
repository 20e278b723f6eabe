"""The allocation-free cell sort (bnn_cell_sort_noalloc).

Who needs it: code that cannot call cudaMalloc when it needs a sort -- work recorded
while a CUDA graph is being captured (allocation is not capturable), host callbacks and
allocator hooks, or an application that has reserved all device memory beforehand.  The
entry point keeps its scratch in a fixed array inside the library instead.

It must return exactly what the allocating bnn_cell_sort returns (integer work, so the
bar is bit equality), also on a second call in a row (the shared scratch array keeps the
previous call's contents), and it must refuse sizes beyond its fixed limits.  This file
is collected last so a failure here cannot hide failures elsewhere.
"""
import ctypes as C

import numpy as np
import pytest
import torch

from banana_b200 import scenes

pytestmark = pytest.mark.gpu

CAPACITY = 8  # BNN_ERR_CAPACITY


def _sort(L, fn, pts, bmin, cell, nc):
    n = len(pts)
    p = torch.from_numpy(np.ascontiguousarray(pts, np.float32)).cuda()
    cid = torch.zeros(max(n, 1), dtype=torch.int32, device="cuda")
    srt = torch.zeros(max(n, 1), dtype=torch.int32, device="cuda")
    start = torch.zeros(int(np.prod(nc.astype(np.int64))) + 1, dtype=torch.int32, device="cuda")
    oor = C.c_uint32()
    rc = getattr(L, fn)(C.c_void_p(p.data_ptr()), n, bmin.ctypes.data_as(C.POINTER(C.c_float)), cell,
                        nc.ctypes.data_as(C.POINTER(C.c_int32)), C.c_void_p(cid.data_ptr()),
                        C.c_void_p(srt.data_ptr()), C.c_void_p(start.data_ptr()), C.byref(oor), None)
    torch.cuda.synchronize()
    return rc, cid.cpu().numpy()[:n], srt.cpu().numpy()[:n], start.cpu().numpy(), oor.value


def test_noalloc_matches_allocating_sort_twice(bnn):
    L = bnn.load()
    cases = [
        (scenes.point_cloud(300_000, seed=5), np.zeros(3, np.float32), np.float32(0.01), np.array([100, 100, 100], np.int32)),
        # second call: different size and grid; points partly outside the grid are clamped
        (scenes.point_cloud(120_000, seed=9) * np.float32(1.2) - np.float32(0.1), np.zeros(3, np.float32),
         np.float32(1.0 / 64), np.array([64, 64, 64], np.int32)),
    ]
    for pts, bmin, cell, nc in cases:
        ref = _sort(L, "bnn_cell_sort", pts, bmin, cell, nc)
        got = _sort(L, "bnn_cell_sort_noalloc", pts, bmin, cell, nc)
        assert ref[0] == 0 and got[0] == 0
        for a, b in zip(ref[1:4], got[1:4]):
            assert np.array_equal(a, b)
        assert ref[4] == got[4]


def test_noalloc_rejects_oversize(bnn):
    L = bnn.load()
    pts = np.zeros((1_048_577, 3), np.float32)
    rc = _sort(L, "bnn_cell_sort_noalloc", pts, np.zeros(3, np.float32), np.float32(0.5),
               np.array([4, 4, 4], np.int32))[0]
    assert rc == CAPACITY
    rc = _sort(L, "bnn_cell_sort_noalloc", pts[:10], np.zeros(3, np.float32), np.float32(0.001),
               np.array([200, 200, 200], np.int32))[0]
    assert rc == CAPACITY
