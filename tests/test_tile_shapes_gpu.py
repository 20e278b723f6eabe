"""Tile shapes of the FLIP P2G + fluid SDF pass: every shape gives the same bits (lone
scenes and the staged batch), and the tuner records a choice per launch kind: the fastest
shape it timed, or the default when none beats it by 3%."""
import numpy as np
import pytest

from banana_b200 import scenes

pytestmark = pytest.mark.gpu


@pytest.fixture
def shapes(bnn):
    out = bnn.capi.tile_shapes()
    yield out
    bnn.capi.set_tile_shape(-1)


def _run_lone(bnn, cfg, pos, vel, steps):
    s = bnn.FlipSolver(cfg)
    s.set_particles(pos, vel)
    for _ in range(steps):
        s.step()
    p, v = s.get_particles()
    u = s.grid("u")
    phi = s.grid("phi")
    s.close()
    return p, v, u, phi


def test_every_shape_gives_the_same_step(bnn, shapes):
    assert len(shapes) >= 2 and shapes[0] == (6, 8)
    n = 40
    cfg = scenes.dam_break_params(n)
    pos, vel = scenes.dam_break(n)
    ref = None
    for k in range(len(shapes)):
        bnn.capi.set_tile_shape(k)
        out = _run_lone(bnn, cfg, pos, vel, 4)
        if ref is None:
            ref = out
            continue
        for a, b, what in zip(ref, out, ("pos", "vel", "u", "phi")):
            assert np.array_equal(a, b), (shapes[k], what)


def test_every_shape_gives_the_same_batch(bnn, shapes):
    specs = [{"res": (40, 24, 32), "block_frac": (0.5, 0.5, 0.4), "seed": 21},
             {"res": (16, 40, 24), "block_frac": (0.6, 0.3, 0.6), "seed": 22},
             {"res": (24, 24, 48), "block_frac": (0.4, 0.6, 0.4), "seed": 23}]
    ref = None
    for k in range(len(shapes)):
        bnn.capi.set_tile_shape(k)
        b = bnn.FlipBatch(worker_threads=1)
        ids = [b.add_scene(*scenes.batch_scene(sp)) for sp in specs]
        for _ in range(3):
            assert b.step()["staged_scenes"] == len(specs)
        out = [b.get_scene(i) for i in ids]
        b.close()
        if ref is None:
            ref = out
            continue
        for q, ((pa, va), (pb, vb)) in enumerate(zip(ref, out)):
            assert np.array_equal(pa, pb) and np.array_equal(va, vb), (shapes[k], q)


def test_tuner_records_the_fastest_shape(bnn, shapes):
    bnn.capi.set_tile_shape(-1)
    n = 36  # a resolution bucket no other test uses
    cfg = scenes.dam_break_params(n)
    pos, vel = scenes.dam_break(n)
    tuned = _run_lone(bnn, cfg, pos, vel, 2)
    bnn.capi.set_tile_shape(0)
    fixed = _run_lone(bnn, cfg, pos, vel, 2)
    for a, b in zip(tuned, fixed):
        assert np.array_equal(a, b)
    g = n + 4
    want = [-(-(g + 1) // 32) * 32 - 1] * 3
    rows = [r for r in bnn.capi.tile_tuning() if r["kind"] == "scene" and r["cells_per_axis_le"] == want]
    assert len(rows) == 1, bnn.capi.tile_tuning()
    r = rows[0]
    assert len(r["us"]) == len(shapes) and all(t > 0 for t in r["us"])
    assert (r["tz"], r["yc"]) == shapes[r["shape"]]
    # the fastest shape, unless it is within 3% of the default's time
    if r["shape"] == 0:
        assert min(r["us"]) >= 0.97 * r["us"][0] * (1 - 1e-6)
    else:
        assert r["us"][r["shape"]] == min(r["us"]) and r["us"][r["shape"]] < 0.97 * r["us"][0]
