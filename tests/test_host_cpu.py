"""The C++ host side without a GPU: the scene reader and the seeded particle sampler of
FLIP_GPU_Solver produce exactly the particles of banana_b200.scenes.dam_break."""
import subprocess

import numpy as np
import pytest

from banana_b200 import build as bld
from banana_b200 import scenes
from tests.host_scene import dam_break_scene, read_particles


@pytest.fixture(scope="module")
def driver():
    if not bld.LIB.exists():
        bld.build_cuda()
    exe = bld.build_host()
    assert exe is not None and exe.exists()
    return exe


@pytest.mark.parametrize("n", [24, 64])
def test_scene_sampler_matches_python_seeder(driver, tmp_path, n):
    scene = tmp_path / "dam.json"
    scene.write_text(dam_break_scene(n))
    out = tmp_path / "p.f32"
    subprocess.run([str(driver), str(scene), "--sample-only", str(out)], check=True, timeout=60)
    pos, vel = read_particles(out)
    pp, vv = scenes.dam_break(n)
    assert np.array_equal(pos, pp)
    assert np.array_equal(vel, vv)


def test_unknown_solver_is_refused(driver, tmp_path):
    scene = tmp_path / "x.json"
    scene.write_text(dam_break_scene(16, solver="SPH_3DSolver"))
    r = subprocess.run([str(driver), str(scene)], capture_output=True, text=True, timeout=60)
    assert r.returncode == 1 and "not supported" in r.stderr
