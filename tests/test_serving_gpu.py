"""Continuous batching on the GPU: requests admitted mid-run under a small HBM budget (so
some wait for memory) each end bit for bit where the same scene run alone ends."""
import numpy as np
import pytest

from banana_b200 import scenes
from banana_b200.serving import Request, SceneServer

pytestmark = pytest.mark.gpu


def test_served_requests_equal_lone_runs(bnn):
    specs = [{"res": (24, 20, 24), "block_frac": (0.4, 0.5, 0.4), "seed": 3},
             {"res": (16, 24, 16), "block_frac": (0.5, 0.4, 0.6), "seed": 4},
             {"res": (20, 20, 20), "block_frac": (0.3, 0.6, 0.3), "seed": 5},
             {"res": (28, 16, 20), "block_frac": (0.6, 0.3, 0.5), "seed": 6}]
    steps = [6, 4, 5, 3]
    built = [scenes.batch_scene(s) for s in specs]
    est = [bnn.capi.scene_bytes_estimate(cfg, len(pos)) for cfg, pos, _ in built]
    # room for the two largest at once, not for all four: later requests wait for memory
    budget = sorted(est)[-1] + sorted(est)[-2] + 1
    batch = bnn.FlipBatch(hbm_budget_bytes=budget, worker_threads=2)

    # the server's clock advances 10 ms per batch step, so arrivals meet the same running
    # set whatever the GPU's speed: requests 2 and 3 arrive while 0 and 1 still run
    now = [0.0]

    class Ticking:
        def __getattr__(self, name):
            return getattr(batch, name)

        def step(self):
            now[0] += 0.01
            return batch.step()

    srv = SceneServer(Ticking(), clock=lambda: now[0])
    reqs = [Request(k, cfg, pos, vel, steps[k], arrival=0.0 if k < 2 else 0.01 * k)
            for k, (cfg, pos, vel) in enumerate(built)]
    results = {r.rid: r for r in srv.run(reqs, time_limit=120.0)}
    batch.close()
    assert sorted(results) == [0, 1, 2, 3]
    assert srv.stats.waits_for_memory >= 1
    for k, (cfg, pos, vel) in enumerate(built):
        lone = bnn.FlipSolver(cfg)
        lone.set_particles(pos, vel)
        for _ in range(steps[k]):
            lone.step()
        p, v = lone.get_particles()
        lone.close()
        assert results[k].steps == steps[k]
        assert np.array_equal(results[k].pos, p) and np.array_equal(results[k].vel, v), k
