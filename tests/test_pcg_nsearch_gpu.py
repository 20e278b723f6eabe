"""Standalone PCG, cell sort, z-sort and neighbour search through the C ABI, against the
oracle (restatements of PCGSolver.cpp, Grid.cpp and NeighborSearch.cpp)."""
import ctypes as C

import numpy as np
import pytest
import torch

from banana_b200 import scenes

pytestmark = pytest.mark.gpu


def _system(oracle_mod, n=32, steps=3):
    cfg = scenes.dam_break_params(n)
    pos, vel = scenes.dam_break(n)
    o = oracle_mod.Oracle(cfg)
    o.set_particles(pos, vel)
    for _ in range(steps):
        o.step()
    rs, ci, va, rhs = o.system()
    nrow = len(rhs)
    diag = np.zeros(nrow, np.float32)
    nbr = -np.ones((nrow, 6), np.int32)
    off = None
    for r in range(nrow):
        cols = ci[rs[r]:rs[r + 1]]
        vals = va[rs[r]:rs[r + 1]]
        lo = [c for c in cols if c < r]
        hi = [c for c in cols if c > r]
        for c, v in zip(cols, vals):
            if c == r:
                diag[r] = v
            else:
                off = v
        nbr[r, 3 - len(lo):3] = lo
        nbr[r, 3:3 + len(hi)] = hi
    return (rs, ci, va, rhs), diag, nbr, off


SINGLE = 0x10  # BNN_PCG_SINGLE_REDUCTION: both inner products in one reduction


@pytest.mark.parametrize("form", [0, SINGLE], ids=["two_reductions", "single_reduction"])
@pytest.mark.parametrize("mode,omode", [("fp32", 0), ("fp64", 1), ("refined", 2)])
def test_pcg_7pt_matches_oracle(bnn, oracle_mod, mode, omode, form):
    (rs, ci, va, rhs), diag, nbr, off = _system(oracle_mod)
    tol = 1e-8 if mode == "refined" else 1e-6
    m = bnn.capi.PCG_MODE[mode] | form
    x, st = bnn.pcg_solve_7pt(diag, nbr, off, rhs, tol, 5000, mode=m, inner_tol=1e-3)
    xo, so = oracle_mod.pcg(rs, ci, va, rhs, tol, 5000, omode | form, inner_tol=1e-3)
    assert st["success"] == 1 and so["success"]
    assert st["iterations"] == so["iterations"]
    if mode == "fp32":
        assert np.array_equal(x.astype(np.float32), xo.astype(np.float32))
    else:
        assert np.array_equal(x, xo)


def test_refined_reaches_1e8_fp64_checked(bnn, oracle_mod):
    """Refined FP32 PCG: max|b - A x| (FP64) < 1e-8 max|b|"""
    (rs, ci, va, rhs), diag, nbr, off = _system(oracle_mod, n=32, steps=4)
    x, st = bnn.pcg_solve_7pt(diag, nbr, off, rhs, 1e-8, 5000, mode="refined", inner_tol=1e-3)
    n = len(rhs)
    ax = np.zeros(n)
    for r in range(n):
        for j in range(rs[r], rs[r + 1]):
            ax[r] += float(va[j]) * x[ci[j]]
    res = np.abs(rhs.astype(np.float64) - ax).max()
    assert res < 1e-8 * np.abs(rhs).max()


def _box_system(nx=40, ny=36, nz=30, holes=0.08, seed=5):
    """A 7-point system on a box of cells with random holes (air cells), rows in cell
    order and neighbours in their direction slots (-z,-y,-x,+x,+y,+z): the layout of a
    grid, which the solver packs into 16-byte row records.  Returns the slot layout, the
    same system with each row's neighbours listed compactly (the general layout), and the
    CSR form for the oracle."""
    rng = np.random.default_rng(seed)
    act = rng.random((nz, ny, nx)) > holes
    row = -np.ones((nz, ny, nx), np.int64)
    row[act] = np.arange(int(act.sum()))
    n = int(act.sum())
    dt = np.float32(1.0 / 30)
    nbr = -np.ones((n, 6), np.int32)
    k, j, i = np.nonzero(act)
    r = row[k, j, i]
    for slot, (dk, dj, di) in enumerate([(-1, 0, 0), (0, -1, 0), (0, 0, -1), (0, 0, 1), (0, 1, 0), (1, 0, 0)]):
        kk, jj, ii = k + dk, j + dj, i + di
        ok = (kk >= 0) & (kk < nz) & (jj >= 0) & (jj < ny) & (ii >= 0) & (ii < nx)
        nb = np.full(n, -1, np.int64)
        nb[ok] = row[kk[ok], jj[ok], ii[ok]]
        nbr[r, slot] = nb
    cnt = (nbr >= 0).sum(1)
    diag = (cnt * dt + (6 - cnt) * dt / np.float32(0.5)).astype(np.float32)
    rhs = (rng.standard_normal(n) * 1e-3).astype(np.float32)
    compact = -np.ones_like(nbr)
    rs, ci, va = [0], [], []
    for q in range(n):
        lo = [c for c in nbr[q, :3] if c >= 0]
        hi = [c for c in nbr[q, 3:] if c >= 0]
        compact[q, 3 - len(lo):3] = lo
        compact[q, 3:3 + len(hi)] = hi
        for c in lo:
            ci.append(c); va.append(-dt)
        ci.append(q); va.append(diag[q])
        for c in hi:
            ci.append(c); va.append(-dt)
        rs.append(len(ci))
    return nbr, compact, diag, -dt, rhs, (np.array(rs), np.array(ci), np.array(va, np.float32))


@pytest.mark.parametrize("form", [0, SINGLE], ids=["two_reductions", "single_reduction"])
@pytest.mark.parametrize("mode,omode", [("fp32", 0), ("fp64", 1), ("refined", 2)])
def test_pcg_7pt_grid_rows_packed_matches_oracle(bnn, oracle_mod, mode, omode, form):
    """Grid-ordered rows take the packed-record solve (x neighbours by warp shuffle); the
    compact layout of the same system takes the general one.  Both equal the oracle, in
    either step order."""
    nbr, compact, diag, off, rhs, (rs, ci, va) = _box_system()
    tol = 1e-8 if mode == "refined" else 1e-6
    xo, so = oracle_mod.pcg(rs, ci, va, rhs, tol, 5000, omode | form, inner_tol=1e-3)
    assert so["success"]
    for layout in (nbr, compact):
        x, st = bnn.pcg_solve_7pt(diag, layout, off, rhs, tol, 5000, mode=bnn.capi.PCG_MODE[mode] | form,
                                  inner_tol=1e-3)
        assert st["success"] == 1
        assert st["iterations"] == so["iterations"]
        if mode == "fp32":
            assert np.array_equal(x.astype(np.float32), xo.astype(np.float32))
        else:
            assert np.array_equal(x, xo)


def _slot_system(nbr, seed):
    """Diagonal (every missing neighbour counted as a face to air, so the matrix is
    strictly diagonally dominant), right-hand side and CSR (columns in slot order, the
    solver's summation order) of a system given as slot neighbours."""
    rng = np.random.default_rng(seed)
    n = len(nbr)
    dt = np.float32(1.0 / 30)
    cnt = (nbr >= 0).sum(1)
    diag = (cnt * dt + (6 - cnt) * dt / np.float32(0.5)).astype(np.float32)
    rhs = (rng.standard_normal(n) * 1e-3).astype(np.float32)
    rs, ci, va = [0], [], []
    for q in range(n):
        for c in nbr[q, :3]:
            if c >= 0:
                ci.append(c); va.append(-dt)
        ci.append(q); va.append(diag[q])
        for c in nbr[q, 3:]:
            if c >= 0:
                ci.append(c); va.append(-dt)
        rs.append(len(ci))
    return diag, -dt, rhs, (np.array(rs), np.array(ci), np.array(va, np.float32))


def _grid_slots(act):
    """Slot neighbours (-z,-y,-x,+x,+y,+z) of the active cells of a (z, y, x) mask, rows
    in cell order."""
    nz, ny, nx = act.shape
    row = -np.ones(act.shape, np.int64)
    row[act] = np.arange(int(act.sum()))
    k, j, i = np.nonzero(act)
    r = row[k, j, i]
    nbr = -np.ones((int(act.sum()), 6), np.int32)
    for slot, (dk, dj, di) in enumerate([(-1, 0, 0), (0, -1, 0), (0, 0, -1), (0, 0, 1), (0, 1, 0), (1, 0, 0)]):
        kk, jj, ii = k + dk, j + dj, i + di
        ok = (kk >= 0) & (kk < nz) & (jj >= 0) & (jj < ny) & (ii >= 0) & (ii < nx)
        nb = np.full(len(r), -1, np.int64)
        nb[ok] = row[kk[ok], jj[ok], ii[ok]]
        nbr[r, slot] = nb
    return nbr


def _layout_system(kind):
    """Grid-row systems of unusual shape for the packed-record solve: 'box' (a box of
    cells with holes), 'wide_rows' (z layers of 120 then 2000 cells along x: y neighbours
    up to ~2000 rows away) and 'unordered_z' (x chains whose z partners are shuffled in
    blocks of 16 rows: valid grid rows whose -z / +z neighbours are not in row order)."""
    rng = np.random.default_rng(21)
    if kind == "box":
        nbr = _grid_slots(rng.random((30, 36, 40)) > 0.08)
    elif kind == "wide_rows":
        act = rng.random((6, 6, 2000)) > 0.08
        act[:3, :, 120:] = False
        nbr = _grid_slots(act)
    else:
        half = 6 * 2048
        n = 2 * half
        nbr = -np.ones((n, 6), np.int32)
        r = np.arange(n)
        chain = (r % 64) != 0  # x chains of 64 rows
        nbr[chain, 2] = r[chain] - 1
        nxt = np.roll(chain, -1) & (r < n - 1)
        nbr[nxt, 3] = r[nxt] + 1
        perm = np.arange(half).reshape(-1, 16)
        for b in perm:
            rng.shuffle(b)
        perm = perm.ravel()
        nbr[np.arange(half), 5] = half + perm
        nbr[half + perm, 0] = np.arange(half)
    return (nbr,) + _slot_system(nbr, 22)


@pytest.mark.parametrize("kind", ["box", "wide_rows", "unordered_z"])
@pytest.mark.parametrize("mode,omode", [("fp32", 0), ("fp64", 1), ("refined", 2)])
def test_pcg_grid_row_layouts_match_oracle(bnn, oracle_mod, kind, mode, omode):
    """Grid rows whose y neighbours lie far away, or whose z partners are out of row order,
    still take the packed-record solve (its x neighbours by warp shuffle, the others by row
    distance) and equal the oracle bit for bit."""
    nbr, diag, off, rhs, (rs, ci, va) = _layout_system(kind)
    tol = 1e-8 if mode == "refined" else 1e-6
    xo, so = oracle_mod.pcg(rs, ci, va, rhs, tol, 5000, omode, inner_tol=1e-3)
    assert so["success"]
    x, st = bnn.pcg_solve_7pt(diag, nbr, off, rhs, tol, 5000, mode=bnn.capi.PCG_MODE[mode], inner_tol=1e-3)
    assert st["success"] == 1 and st["iterations"] == so["iterations"]
    if mode == "fp32":
        assert np.array_equal(x.astype(np.float32), xo.astype(np.float32))
    else:
        assert np.array_equal(x, xo)


def test_barrier_wait_gives_up_and_device_stays_usable(bnn, oracle_mod):
    """A block waiting at a barrier that nothing completes (sized for two blocks, one
    launched) gives up after its limit and reports a timeout; the device then solves a
    system as before."""
    from banana_b200 import capi
    status, ms = bnn.pcg_barrier_probe(0.05)
    assert status == capi.STATUS_CODE["TIMEOUT"]
    assert 50.0 <= ms < 5000.0, ms
    nbr, _, diag, off, rhs, (rs, ci, va) = _box_system(12, 10, 8)
    xo, so = oracle_mod.pcg(rs, ci, va, rhs, 1e-6, 5000, 0)
    x, st = bnn.pcg_solve_7pt(diag, nbr, off, rhs, 1e-6, 5000)
    assert st["success"] == 1 and st["iterations"] == so["iterations"]
    assert np.array_equal(x.astype(np.float32), xo.astype(np.float32))


def test_pcg_7pt_rejects_bad_neighbour_index(bnn):
    nbr, _, diag, off, rhs, _ = _box_system(8, 8, 8)
    bad = nbr.copy()
    bad[5, 4] = len(rhs)  # one past the last row
    with pytest.raises(bnn.BnnError):
        bnn.pcg_solve_7pt(diag, bad, off, rhs, 1e-6, 100)


def _dev(a):
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


def test_cell_sort_bitexact(bnn, oracle_mod):
    pts = scenes.point_cloud(200_000, seed=7)
    bmin = np.zeros(3, np.float32)
    nc = np.array([100, 100, 100], np.int32)
    cid, srt, start, oor = oracle_mod.cell_sort(pts, bmin, np.float32(0.01), nc)
    L = bnn.load()
    p = _dev(pts)
    n = len(pts)
    gc = torch.zeros(n, dtype=torch.int32, device="cuda")
    gs = torch.zeros(n, dtype=torch.int32, device="cuda")
    gst = torch.zeros(int(nc.prod()) + 1, dtype=torch.int32, device="cuda")
    o = C.c_uint32()
    rc = L.bnn_cell_sort(C.c_void_p(p.data_ptr()), n, bmin.ctypes.data_as(C.POINTER(C.c_float)), 0.01,
                         nc.ctypes.data_as(C.POINTER(C.c_int32)), C.c_void_p(gc.data_ptr()), C.c_void_p(gs.data_ptr()),
                         C.c_void_p(gst.data_ptr()), C.byref(o), None)
    torch.cuda.synchronize()
    assert rc == 0
    assert o.value == oor
    assert np.array_equal(gc.cpu().numpy().view(np.uint32), cid)
    assert np.array_equal(gs.cpu().numpy().view(np.uint32), srt)
    assert np.array_equal(gst.cpu().numpy().view(np.uint32), start)


@pytest.mark.parametrize("nc,cell", [((3, 5, 7), 0.34), ((17, 33, 41), 1 / 16.5), ((129, 130, 131), 1 / 128)],
                         ids=["105_cells", "23001_cells", "2196870_cells"])
def test_cell_sort_grid_sizes_bitexact(bnn, oracle_mod, nc, cell):
    """Cell starts (the exclusive prefix sum of the cell counts, total last) on grids of one
    scan tile, of a few tiles with a ragged end, and of many tiles"""
    pts = scenes.point_cloud(150_000, seed=11)
    bmin = np.zeros(3, np.float32)
    nc = np.array(nc, np.int32)
    cid, srt, start, oor = oracle_mod.cell_sort(pts, bmin, np.float32(cell), nc)
    L = bnn.load()
    p = _dev(pts)
    n = len(pts)
    gc = torch.zeros(n, dtype=torch.int32, device="cuda")
    gs = torch.zeros(n, dtype=torch.int32, device="cuda")
    gst = torch.full((int(nc.prod()) + 1,), -1, dtype=torch.int32, device="cuda")
    o = C.c_uint32()
    rc = L.bnn_cell_sort(C.c_void_p(p.data_ptr()), n, bmin.ctypes.data_as(C.POINTER(C.c_float)), float(np.float32(cell)),
                         nc.ctypes.data_as(C.POINTER(C.c_int32)), C.c_void_p(gc.data_ptr()), C.c_void_p(gs.data_ptr()),
                         C.c_void_p(gst.data_ptr()), C.byref(o), None)
    torch.cuda.synchronize()
    assert rc == 0
    assert o.value == oor
    assert np.array_equal(gc.cpu().numpy().view(np.uint32), cid)
    assert np.array_equal(gs.cpu().numpy().view(np.uint32), srt)
    assert np.array_equal(gst.cpu().numpy().view(np.uint32), start)


def test_z_sort_bitexact(bnn, oracle_mod):
    pts = scenes.point_cloud(100_000, seed=3)
    z, perm = oracle_mod.z_sort(pts, np.float32(0.01))
    L = bnn.load()
    p = _dev(pts)
    n = len(pts)
    gz = torch.zeros(n, dtype=torch.int64, device="cuda")
    gp = torch.zeros(n, dtype=torch.int32, device="cuda")
    rc = L.bnn_z_sort(C.c_void_p(p.data_ptr()), n, 0.01, C.c_void_p(gz.data_ptr()), C.c_void_p(gp.data_ptr()), None)
    assert rc == 0
    assert np.array_equal(gz.cpu().numpy().view(np.uint64), z)
    assert np.array_equal(gp.cpu().numpy().view(np.uint32), perm)


def _lists(off, idx, n):
    return [np.sort(idx[off[i]:off[i + 1]]) for i in range(n)]


@pytest.mark.parametrize("n,seed", [(30_000, 7), (60_000, 1)])
def test_neighbors_set_equal(bnn, oracle_mod, n, seed):
    pts = scenes.point_cloud(n, seed=seed)
    r = np.float32(0.01)
    off_o, idx_o = oracle_mod.neighbors(pts, r)
    L = bnn.load()
    p = _dev(pts)
    goff = torch.zeros(n + 1, dtype=torch.int64, device="cuda")
    cap = int(off_o[-1]) + 16
    gidx = torch.zeros(max(cap, 1), dtype=torch.int32, device="cuda")
    tot = C.c_uint64()
    rc = L.bnn_neighbors(C.c_void_p(p.data_ptr()), n, r, C.c_void_p(goff.data_ptr()), C.c_void_p(gidx.data_ptr()),
                         cap, C.byref(tot), None)
    assert rc == 0
    assert tot.value == off_o[-1]
    go = goff.cpu().numpy().view(np.uint64)
    gi = gidx.cpu().numpy().view(np.uint32)[: tot.value]
    assert np.array_equal(go, off_o)
    # set equality per point (the reference's list order depends on its thread schedule)
    owner = np.repeat(np.arange(n), np.diff(go).astype(np.int64))
    a = np.lexsort((gi, owner))
    assert np.array_equal(gi[a], idx_o)


def test_neighbors_capacity_error(bnn):
    pts = scenes.point_cloud(5_000, seed=2)
    L = bnn.load()
    p = _dev(pts)
    goff = torch.zeros(len(pts) + 1, dtype=torch.int64, device="cuda")
    gidx = torch.zeros(4, dtype=torch.int32, device="cuda")
    tot = C.c_uint64()
    rc = L.bnn_neighbors(C.c_void_p(p.data_ptr()), len(pts), 0.05, C.c_void_p(goff.data_ptr()),
                         C.c_void_p(gidx.data_ptr()), 4, C.byref(tot), None)
    assert rc == 8 and tot.value > 4
