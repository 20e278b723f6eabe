"""Host-side pieces of the batch and serving workloads, without a GPU: the seeded scene
and request generators, and the admission estimate (pure host arithmetic in the C ABI)."""
import math

import numpy as np
import pytest

from banana_b200 import build as bld
from banana_b200 import capi, scenes


@pytest.fixture(scope="module")
def lib():
    if not bld.LIB.exists():
        bld.build_cuda()
    return capi.load()


def test_batch_specs_are_seeded_and_in_range():
    a = scenes.batch_scene_specs()
    b = scenes.batch_scene_specs()
    assert a == b and len(a) == 256
    for s in a:
        assert all(r in (32, 48, 64, 96, 128) for r in s["res"])
        assert all(0.2 <= f <= 0.6 for f in s["block_frac"])
    # every resolution appears on every axis
    for ax in range(3):
        assert {s["res"][ax] for s in a} == {32, 48, 64, 96, 128}


def test_batch_scene_particles_fill_the_block():
    s = {"res": (32, 48, 64), "block_frac": (0.5, 0.25, 0.4), "seed": 9}
    cfg, pos, vel = scenes.batch_scene(s)
    dx = 1.0 / 64
    assert cfg["box_max"] == (0.5, 0.75, 1.0)
    cells = [int(math.floor(f * r + 1e-9)) for f, r in zip(s["block_frac"], s["res"])]
    assert len(pos) == 8 * cells[0] * cells[1] * cells[2]
    for a in range(3):
        assert pos[:, a].min() >= 0 and pos[:, a].max() < cells[a] * dx
    assert np.all(vel == 0)


def test_serve_requests_poisson_and_log_uniform():
    r = scenes.serve_requests(4000)
    t = np.array([q["t"] for q in r])
    gaps = np.diff(np.concatenate([[0.0], t]))
    assert np.all(gaps > 0)
    assert abs(gaps.mean() - 1 / 20) < 0.1 / 20          # mean inter-arrival 1/lambda
    assert abs(gaps.std() / gaps.mean() - 1) < 0.1      # exponential: cv = 1
    n = np.array([q["res"][0] for q in r])
    assert n.min() >= 32 and n.max() <= 192
    ln = np.log(n)
    assert abs(np.median(ln) - 0.5 * (math.log(32) + math.log(192))) < 0.1
    assert scenes.serve_requests(10) == scenes.serve_requests(10)


def test_admission_estimate_scales(lib):
    cfg = scenes.dam_break_params(64)
    a = capi.scene_bytes_estimate(cfg, 190_000)
    b = capi.scene_bytes_estimate(cfg, 380_000)
    assert b > a > 0
    big = capi.scene_bytes_estimate(scenes.dam_break_params(256), 12_734_496)
    assert 2e9 < big < 8e9
    fp64 = capi.scene_bytes_estimate(dict(cfg, pcg_mode=1), 190_000)
    assert fp64 > a
