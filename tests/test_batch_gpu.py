"""Scene batches (bnn_batch_*): every scene of a batch computes exactly what a lone
solver handle computes -- in the staged step (one launch per stage over all the scenes it
takes) and in the per-scene step (worker threads, each scene on its own stream) -- scenes
come and go between steps, and admission honours the budget."""
import numpy as np
import pytest

from banana_b200 import scenes

pytestmark = pytest.mark.gpu

SPECS = [
    {"res": (24, 32, 16), "block_frac": (0.5, 0.4, 0.6), "seed": 1},
    {"res": (16, 16, 16), "block_frac": (0.3, 0.6, 0.5), "seed": 2},
    {"res": (32, 24, 24), "block_frac": (0.4, 0.5, 0.3), "seed": 3},
    {"res": (20, 20, 28), "block_frac": (0.6, 0.3, 0.4), "seed": 4},
]


def _lone(bnn, spec, steps, **over):
    cfg, pos, vel = scenes.batch_scene(spec, **over)
    s = bnn.FlipSolver(cfg)
    s.set_particles(pos, vel)
    for _ in range(steps):
        s.step()
    out = s.get_particles()
    s.close()
    return out


@pytest.mark.parametrize("mode", ["staged", "staged_no_graphs", "per_scene"])
def test_batch_scenes_equal_lone_solvers(bnn, mode):
    staged = mode.startswith("staged")
    step_mode = {"staged": bnn.capi.BATCH_STAGED, "per_scene": bnn.capi.BATCH_PER_SCENE,
                 "staged_no_graphs": bnn.capi.BATCH_STAGED | bnn.capi.BATCH_NO_GRAPHS}[mode]
    b = bnn.FlipBatch(worker_threads=3, step_mode=step_mode)
    ids = {}
    for q in range(3):
        cfg, pos, vel = scenes.batch_scene(SPECS[q])
        ids[q] = b.add_scene(cfg, pos, vel)
    graphs = []
    for _ in range(5):
        st = b.step()
        assert st["scenes"] == 3 and st["failed"] == 0
        assert st["staged_scenes"] == (3 if staged else 0)
        graphs.append((st["graph_instantiations"], st["graph_updates"]))
    if mode == "staged":
        # both segments built once (the first step tunes the tile shape outside a capture),
        # then replayed while the scenes stay the same
        assert sum(i for i, _ in graphs) == 2 and graphs[-1] == (0, 0)
    else:
        assert graphs == [(0, 0)] * 5
    for q in range(3):
        pg, vg = b.get_scene(ids[q])
        pl, vl = _lone(bnn, SPECS[q], 5)
        assert np.array_equal(pg, pl) and np.array_equal(vg, vl), q
        assert b.scene_info(ids[q])["steps"] == 5
    # scenes leave and join between steps
    b.remove_scene(ids[1])
    cfg, pos, vel = scenes.batch_scene(SPECS[3])
    ids[3] = b.add_scene(cfg, pos, vel)
    for k in range(3):
        st = b.step()
        assert st["scenes"] == 3
        if mode == "staged" and k == 0:
            # other scenes, other launch shapes: the segments are captured again
            assert st["graph_instantiations"] + st["graph_updates"] >= 1
    for q, steps in ((0, 8), (2, 8), (3, 3)):
        pg, _ = b.get_scene(ids[q])
        pl, _ = _lone(bnn, SPECS[q], steps)
        assert np.array_equal(pg, pl), q
    admitted, held = b.memory()
    assert admitted > 0 and held > 0
    b.close()


def test_batch_admission_budget(bnn):
    cfg, pos, vel = scenes.batch_scene(SPECS[0])
    est = bnn.scene_bytes_estimate(cfg, len(pos))
    b = bnn.FlipBatch(hbm_budget_bytes=int(est * 1.5))
    b.add_scene(cfg, pos, vel)
    with pytest.raises(bnn.BnnError) as e:
        b.add_scene(cfg, pos, vel)
    assert e.value.code == 8  # BNN_ERR_CAPACITY
    b.close()


def test_staged_batch_mixed_sizes_and_kinds(bnn):
    """Scenes of uneven sizes (one with more cells than one 2048 x 2048 scan level holds)
    beside a scene the staged step does not take (plain FP32 PCG): each equals its lone run."""
    specs = [{"res": (40, 24, 56), "block_frac": (0.5, 0.5, 0.4), "seed": 11},
             {"res": (16, 48, 16), "block_frac": (0.6, 0.3, 0.6), "seed": 12},
             {"res": (168, 160, 160), "block_frac": (0.2, 0.2, 0.2), "seed": 13},
             {"res": (24, 24, 24), "block_frac": (0.4, 0.6, 0.4), "seed": 14},
             {"res": (32, 16, 40), "block_frac": (0.3, 0.5, 0.5), "seed": 15}]
    over = [{}, {}, {}, {"pcg_mode": 0}, {}]
    steps = 4
    b = bnn.FlipBatch(worker_threads=2)
    ids = []
    for spec, o in zip(specs, over):
        cfg, pos, vel = scenes.batch_scene(spec, **o)
        ids.append(b.add_scene(cfg, pos, vel))
    for _ in range(steps):
        st = b.step()
        assert st["failed"] == 0 and st["staged_scenes"] == 4
    for sid, spec, o in zip(ids, specs, over):
        pg, vg = b.get_scene(sid)
        pl, vl = _lone(bnn, spec, steps, **o)
        assert np.array_equal(pg, pl) and np.array_equal(vg, vl), spec
        info = b.scene_info(sid)
        assert info["steps"] == steps and info["pcg_success"] == 1
    b.close()
