"""CPU checks of the oracle (the restatement the GPU parity tests compare against).

1. Known answers from the reference's own tests: the Grid unit test
   (BananaCore/Banana/Grid/_Grid.Test.hpp:29-57) and the Morton encode tables
   (NeighborSearch/Morton/Morton3D_LUTs.h), both extracted into tests/golden/ by the
   scripts beside them.
2. The reference's neighbour-search test method (_NeighborSearch.Test.hpp:119-212): the
   hash-grid search, the Grid search and brute force must agree as sets.
3. Analytic checks of the FLIP pieces that have no reference golden vectors.
"""
import json
from pathlib import Path

import numpy as np
import pytest

from banana_b200 import scenes

GOLDEN = Path(__file__).resolve().parent / "golden"


# ---------------------------------------------------------------------------------- 1
def test_grid_known_answers(oracle_mod):
    ka = json.loads((GOLDEN / "grid_known_answers.json").read_text())
    g = ka["grid"]
    bmin = np.array(g["bmin"], np.float32)
    nc = oracle_mod.grid_ncells(g["bmin"], g["bmax"], np.float32(g["cell_size"]))
    assert list(nc) == ka["ncells"]
    ncv = np.array(nc, np.int32)
    # Grid::getValidCellIdx = nearest valid cell of the truncated cell index
    pos = np.array([ka["valid_cell_idx"]["pos"]], np.float32)
    cid, srt, start, oor = oracle_mod.cell_sort(pos, bmin, np.float32(g["cell_size"]), ncv)
    e = ka["valid_cell_idx"]["expect"]
    assert int(cid[0]) == (e[2] * nc[1] + e[1]) * nc[0] + e[0]
    assert oor == 1  # the z coordinate was outside and got clamped
    # isValidCell / getNearestValidCellIdx are integer range tests
    for c in ka["is_valid_cell"]:
        assert all(0 <= c["cell"][d] < nc[d] for d in range(3)) == c["valid"]
    nv = ka["nearest_valid_cell"]
    assert [min(max(nv["cell"][d], 0), nc[d] - 1) for d in range(3)] == nv["expect"]
    # collectIndexToCells + getNeighborList(ppos, list) (cell span 1, no distance test)
    parts = np.array(ka["neighbor_list"]["particles"], np.float32)
    q = parts[ka["neighbor_list"]["query"]]
    lst = oracle_mod.grid_neighbor_list(parts, bmin, np.float32(g["cell_size"]), ncv, q)
    assert len(lst) == ka["neighbor_list"]["expect_size"]


def _morton_lut(x, y, z, lut):
    ans = 0
    for i in range(8, 0, -1):
        sh = (i - 1) * 8
        ans = ((ans << 24) | (lut["z"][(z >> sh) & 255] | lut["y"][(y >> sh) & 255] | lut["x"][(x >> sh) & 255]))
        ans &= (1 << 64) - 1
    return ans


def test_morton_matches_reference_tables(oracle_mod):
    lut = json.loads((GOLDEN / "morton3d_lut.json").read_text())
    pts = scenes.point_cloud(2000, seed=3)
    r = np.float32(0.01)
    z, perm = oracle_mod.z_sort(pts, r)
    inv = np.float32(1.0 / float(r))
    for p in range(0, 2000, 37):
        k = []
        for d in range(3):
            t = np.float32(pts[p, d] - np.float32(1.2345))
            v = np.float32(inv * t)
            k.append(int(v) if t >= 0 else int(v) - 1)
        c = [kk + 2147483647 for kk in k]
        assert int(z[p]) == _morton_lut(c[0], c[1], c[2], lut)
    # z_sort order: by z-value, ties in input order
    zz = z[perm]
    assert np.all(zz[1:] >= zz[:-1])
    tie = zz[1:] == zz[:-1]
    assert np.all(perm[1:][tie] > perm[:-1][tie])


# ---------------------------------------------------------------------------------- 2
def _brute(pts, r):
    r2 = np.float32(r) * np.float32(r)
    out = []
    for i in range(len(pts)):
        d = (pts[i][None, :] - pts).astype(np.float32)
        l2 = (d[:, 0] * d[:, 0] + d[:, 1] * d[:, 1]) + d[:, 2] * d[:, 2]
        m = np.nonzero(l2 < r2)[0]
        out.append(np.sort(m[m != i]))
    return out


@pytest.mark.parametrize("seed", [1, 2])
def test_neighbor_search_three_ways_agree(oracle_mod, seed):
    pts = scenes.point_cloud(3000, seed=seed)
    r = np.float32(0.05)
    off, idx = oracle_mod.neighbors(pts, r)
    ns = [idx[off[i]:off[i + 1]] for i in range(len(pts))]
    bf = _brute(pts, r)
    nc = np.array([20, 20, 20], np.int32)
    for i in range(0, len(pts), 7):
        assert np.array_equal(ns[i], bf[i])
        grid = np.sort(oracle_mod.grid_neighbor_list(pts, np.zeros(3, np.float32), r, nc, pts[i], d2=r * r))
        assert np.array_equal(grid, bf[i])  # no coincident points, so 0 < d2 and d2 < r2 agree


def test_cell_sort_is_stable_by_cell(oracle_mod):
    pts = scenes.point_cloud(20000, seed=4)
    cid, srt, start, oor = oracle_mod.cell_sort(pts, np.zeros(3, np.float32), np.float32(0.05),
                                                np.array([20, 20, 20], np.int32))
    assert oor == 0
    order = np.lexsort((np.arange(len(pts)), cid))
    assert np.array_equal(srt, order)
    assert np.array_equal(start, np.concatenate([[0], np.cumsum(np.bincount(cid, minlength=8000))]))


# ---------------------------------------------------------------------------------- 3
def test_trilinear_reproduces_linear_fields(oracle_mod):
    cfg = scenes.dam_break_params(8)
    o = oracle_mod.Oracle(cfg)
    G = o.G
    for d in range(3):
        shp = o.face_shape(d)
        k, j, i = np.meshgrid(np.arange(shp[2]), np.arange(shp[1]), np.arange(shp[0]), indexing="ij")
        # face positions in grid coordinates: index + 0.5 off the component axis
        fx = i + (0.0 if d == 0 else 0.5)
        fy = j + (0.0 if d == 1 else 0.5)
        fz = k + (0.0 if d == 2 else 0.5)
        field = (0.5 + 0.25 * fx - 0.125 * fy + 0.0625 * fz).astype(np.float32)
        o.set_grid(d, field)
        rng = np.random.default_rng(d)
        for _ in range(50):
            g = rng.uniform(1.0, G[0] - 2.0, 3)
            v = o.interp_face(d, *g)
            assert abs(v - (0.5 + 0.25 * g[0] - 0.125 * g[1] + 0.0625 * g[2])) < 1e-5


def _run(oracle_mod, n, steps, **over):
    cfg = scenes.dam_break_params(n, **over)
    pos, vel = scenes.dam_break(n)
    o = oracle_mod.Oracle(cfg, use_double=over.pop("use_double", False) if "use_double" in over else False)
    o.set_particles(pos, vel)
    stats = [o.step() for _ in range(steps)]
    return o, stats


def test_pressure_operator_symmetric_positive_diagonal(oracle_mod):
    o, _ = _run(oracle_mod, 16, 3)
    rs, ci, va, rhs = o.system()
    n = len(rhs)
    ent = {}
    for r in range(n):
        cols = ci[rs[r]:rs[r + 1]]
        assert np.all(np.diff(cols.astype(np.int64)) > 0)  # column-sorted rows
        for c, v in zip(cols, va[rs[r]:rs[r + 1]]):
            ent[(r, int(c))] = float(v)
    for (r, c), v in ent.items():
        if r == c:
            assert v > 0
        else:
            assert ent[(c, r)] == v  # exactly symmetric: both sides are -w*dt of the shared face


@pytest.mark.parametrize("mode,tol", [(1, 1e-9), (0, 1e-4), (2, 1e-9), (4, 1e-9), (3, 1e-4)])
def test_pcg_manufactured_solution(oracle_mod, mode, tol):
    o, _ = _run(oracle_mod, 16, 3)
    rs, ci, va, _ = o.system()
    n = len(rs) - 1
    xs = np.random.default_rng(0).standard_normal(n)
    b = np.zeros(n)
    for r in range(n):
        for j in range(rs[r], rs[r + 1]):
            b[r] += float(va[j]) * xs[ci[j]]
    b32 = b.astype(np.float32)
    ctol = 1e-8 if mode in (1, 2, 4) else 1e-6
    x, st = oracle_mod.pcg(rs, ci, va, b32, ctol, 5000, mode, inner_tol=1e-3)
    assert st["success"]
    # compare against the exact solution of the float32-rounded right-hand side
    assert np.abs(x - xs).max() / np.abs(xs).max() < max(tol, 1e-5 if mode in (0, 3) else tol) * 1e3


def test_timed_mode_matches_deterministic_within_rounding(oracle_mod):
    a, _ = _run(oracle_mod, 20, 3)
    b, _ = _run(oracle_mod, 20, 3, nthreads=4, reduce_mode=0)
    scale = max(float(np.abs(a.grid(w)).max()) for w in (0, 1, 2))
    for w in (0, 1, 2):
        ga, gb = a.grid(w), b.grid(w)
        assert np.abs(ga - gb).max() <= 1e-5 * scale


def test_fp64_build_close_to_fp32(oracle_mod):
    a, sa = _run(oracle_mod, 16, 4)
    cfg = scenes.dam_break_params(16)
    pos, vel = scenes.dam_break(16)
    d = oracle_mod.Oracle(cfg, use_double=True)
    d.set_particles(pos, vel)
    for _ in range(4):
        d.step()
    pa, _ = a.get_particles()
    pd, _ = d.get_particles(f64=True)
    assert np.abs(pa - pd).max() < 1e-4 / 16


def test_pcg_zero_rhs_converges_immediately(oracle_mod):
    o, st = _run(oracle_mod, 12, 1)
    assert st[0]["pcg_iterations"] == 0 and st[0]["pcg_success"] == 1  # uniform free fall: div u = 0


def test_seeder_counts_and_cells():
    pos, vel = scenes.dam_break(64)
    assert len(pos) == 25 * 38 * 25 * 8 == 190_000
    assert scenes.dam_break_cells(256) == (102, 153, 102)
    assert 102 * 153 * 102 * 8 == 12_734_496
    dx = 1.0 / 64
    cell = np.floor(pos.astype(np.float64) / dx).astype(np.int64)
    counts = np.bincount((cell[:, 2] * 38 + cell[:, 1]) * 25 + cell[:, 0])
    assert np.all(counts == 8)
    assert np.all(vel == 0)
    p2, _ = scenes.dam_break(64)
    assert np.array_equal(pos, p2)


def test_point_cloud_inside_unit_cube():
    pts = scenes.point_cloud(40000, seed=7)
    assert pts.shape == (40000, 3)
    assert np.all(pts >= 0) and np.all(pts < 1)


def test_p2g_of_uniform_velocity_reproduces_it(oracle_mod):
    """P2G of particles that all carry the same velocity gives that velocity on every valid
    face (sum w v / sum w; equal up to the rounding of the two float sums of ~60 terms,
    a few ulps)."""
    cfg = scenes.dam_break_params(16)
    pos, _ = scenes.dam_break(16)
    v0 = np.array([0.75, -1.25, 0.5], np.float32)
    vel = np.tile(v0, (len(pos), 1))
    o = oracle_mod.Oracle(cfg)
    o.set_particles(pos, vel)
    o.p2g_only()
    for d in range(3):
        u = o.grid(d)
        nz = u[u != 0]
        assert nz.size > 100
        assert np.abs(nz - v0[d]).max() <= 1e-5 * abs(v0[d])


def test_floor_layer_falls_freely_under_static_box_semantics(oracle_mod):
    """A layer covering the whole floor.  With a static box the reference never computes a
    boundary SDF (PIC_Solver.cpp:105-114), so every face weight is 1 and the walls are not
    part of the pressure solve: the projection leaves the uniform gravity field alone (it is
    divergence free), every particle falls with exactly -g t and no sideways motion, and
    only the particle box projection keeps the fluid inside the domain."""
    n = 16
    cfg = scenes.dam_break_params(n)
    pos, vel = scenes.dam_break(n, block=(1.0, 0.25, 1.0))
    o = oracle_mod.Oracle(cfg)
    o.set_particles(pos, vel)
    t = 0.0
    for _ in range(10):
        t += o.step()["dt"]
    p, v = o.get_particles()
    g_t = 9.81 * t
    assert np.abs(v[:, 1] + g_t).max() < 1e-5 * g_t
    assert np.abs(v[:, [0, 2]]).max() < 1e-5 * g_t
    assert p.min() >= 0.0 and p.max() <= 1.0


def test_position_correction_pushes_close_particles_apart(oracle_mod):
    """Two particles closer than the spring radius (2 r / sqrt(3), r = cell / 2) in a still,
    gravity-free box are pushed apart symmetrically by correctParticlePositions; the rest of
    the step does not move them (zero velocity, no gravity)."""
    n = 16
    cfg = scenes.dam_break_params(n, correct_position=1, apply_gravity=0)
    dx = 1.0 / n
    c = np.array([0.5, 0.5, 0.5])
    d = 0.2 * dx
    pos = np.array([c - [d / 2, 0, 0], c + [d / 2, 0, 0]], np.float32)
    vel = np.zeros_like(pos)
    o = oracle_mod.Oracle(cfg)
    o.set_particles(pos, vel)
    o.step()
    p, _ = o.get_particles()
    gap = p[1, 0] - p[0, 0]
    assert gap > d * 1.01
    assert abs((p[0, 0] + p[1, 0]) / 2 - c[0]) < 1e-6
    assert np.abs(p[:, 1:] - pos[:, 1:]).max() < 1e-6
