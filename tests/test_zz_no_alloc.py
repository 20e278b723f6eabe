"""The allocation-free cell sort (bnn_cell_sort_noalloc).

Who needs it: code that cannot call cudaMalloc when it needs a sort -- an application
whose own pool allocator already holds all device memory (another cudaMalloc would fail
or take memory the pool counts on), or a latency-bound loop in which cudaMalloc /
cudaFree would synchronise the device and stall the work on other streams.  The entry
point keeps its scratch in a fixed array inside the library instead.

It must return exactly what the allocating bnn_cell_sort returns (integer work, so the
bar is bit equality), also on a second call in a row (the shared scratch array keeps the
previous call's contents), it must not change the device's free memory, and it must
refuse sizes beyond its fixed limits.  This file is collected last so a failure here
cannot hide failures elsewhere.
"""
import ctypes as C

import numpy as np
import pytest
import torch

from banana_b200 import scenes

pytestmark = pytest.mark.gpu

CAPACITY = 8  # BNN_ERR_CAPACITY


def _buffers(pts, nc):
    n = len(pts)
    p = torch.from_numpy(np.ascontiguousarray(pts, np.float32)).cuda()
    cid = torch.zeros(max(n, 1), dtype=torch.int32, device="cuda")
    srt = torch.zeros(max(n, 1), dtype=torch.int32, device="cuda")
    start = torch.zeros(int(np.prod(nc.astype(np.int64))) + 1, dtype=torch.int32, device="cuda")
    return p, cid, srt, start


def _call(L, fn, bufs, n, bmin, cell, nc):
    p, cid, srt, start = bufs
    oor = C.c_uint32()
    rc = getattr(L, fn)(C.c_void_p(p.data_ptr()), n, bmin.ctypes.data_as(C.POINTER(C.c_float)), cell,
                        nc.ctypes.data_as(C.POINTER(C.c_int32)), C.c_void_p(cid.data_ptr()),
                        C.c_void_p(srt.data_ptr()), C.c_void_p(start.data_ptr()), C.byref(oor), None)
    torch.cuda.synchronize()
    return rc, oor.value


def _sort(L, fn, pts, bmin, cell, nc):
    n = len(pts)
    bufs = _buffers(pts, nc)
    rc, oor = _call(L, fn, bufs, n, bmin, cell, nc)
    _, cid, srt, start = bufs
    return rc, cid.cpu().numpy()[:n], srt.cpu().numpy()[:n], start.cpu().numpy(), oor


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


def test_noalloc_allocates_no_device_memory(bnn):
    """After a first call (which resolves the scratch array's address), further calls
    leave the device's free memory exactly where it was."""
    L = bnn.load()
    pts = scenes.point_cloud(200_000, seed=3)
    bmin, cell, nc = np.zeros(3, np.float32), np.float32(0.01), np.array([100, 100, 100], np.int32)
    bufs = _buffers(pts, nc)
    assert _call(L, "bnn_cell_sort_noalloc", bufs, len(pts), bmin, cell, nc)[0] == 0
    free0 = torch.cuda.mem_get_info()[0]
    for _ in range(3):
        assert _call(L, "bnn_cell_sort_noalloc", bufs, len(pts), bmin, cell, nc)[0] == 0
    assert torch.cuda.mem_get_info()[0] == free0


def test_noalloc_rejects_oversize(bnn):
    L = bnn.load()
    pts = np.zeros((1_048_577, 3), np.float32)
    rc = _sort(L, "bnn_cell_sort_noalloc", pts, np.zeros(3, np.float32), np.float32(0.5),
               np.array([4, 4, 4], np.int32))[0]
    assert rc == CAPACITY
    rc = _sort(L, "bnn_cell_sort_noalloc", pts[:10], np.zeros(3, np.float32), np.float32(0.001),
               np.array([200, 200, 200], np.int32))[0]
    assert rc == CAPACITY
