"""Scene batches (bnn_batch_*): every scene of a batch computes exactly what a lone
solver handle computes (scenes are stepped concurrently from worker threads, each on its
own stream), scenes come and go between steps, and admission honours the budget."""
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


def _lone(bnn, spec, steps):
    cfg, pos, vel = scenes.batch_scene(spec)
    s = bnn.FlipSolver(cfg)
    s.set_particles(pos, vel)
    for _ in range(steps):
        s.step()
    return s.get_particles()


def test_batch_scenes_equal_lone_solvers(bnn):
    b = bnn.FlipBatch(worker_threads=3)
    ids = {}
    for q in range(3):
        cfg, pos, vel = scenes.batch_scene(SPECS[q])
        ids[q] = b.add_scene(cfg, pos, vel)
    for _ in range(5):
        st = b.step()
        assert st["scenes"] == 3 and st["failed"] == 0
    for q in range(3):
        pg, vg = b.get_scene(ids[q])
        pl, vl = _lone(bnn, SPECS[q], 5)
        assert np.array_equal(pg, pl) and np.array_equal(vg, vl), q
        assert b.scene_info(ids[q])["steps"] == 5
    # scenes leave and join between steps
    b.remove_scene(ids[1])
    cfg, pos, vel = scenes.batch_scene(SPECS[3])
    ids[3] = b.add_scene(cfg, pos, vel)
    for _ in range(3):
        st = b.step()
        assert st["scenes"] == 3
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
