"""The C++ drop-in (FLIP_GPU_Solver through the bnn_flip_run driver: factory by scene
name, loadScene, doFrameSimulation per frame) computes the same frames as the solver
driven from Python, and the same as the oracle."""
import subprocess

import numpy as np
import pytest

from banana_b200 import build as bld
from banana_b200 import scenes
from tests.host_scene import dam_break_scene, read_particles

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("solver,kind", [("FLIP_GPU_3DSolver", 0), ("APIC_GPU_3DSolver", 1)])
def test_driver_frames_match_python_and_oracle(bnn, oracle_mod, tmp_path, solver, kind):
    exe = bld.build_host()
    n = 20
    scene = tmp_path / "dam.json"
    scene.write_text(dam_break_scene(n, frames=2, solver=solver))
    out = tmp_path / "out.f32"
    r = subprocess.run([str(exe), str(scene), "--out", str(out)], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr
    lines = [l for l in r.stdout.splitlines() if l.startswith("{\"frame\"")]
    assert len(lines) == 2
    pos, vel = read_particles(out)

    cfg = scenes.dam_break_params(n, solver_kind=kind)
    p0, v0 = scenes.dam_break(n)
    s = bnn.FlipSolver(cfg)
    s.set_particles(p0, v0)
    for _ in range(2):
        s.advance_frame()
    pp, vp = s.get_particles()
    assert np.array_equal(pos, pp) and np.array_equal(vel, vp)

    o = oracle_mod.Oracle(cfg)
    o.set_particles(p0, v0)
    for _ in range(2):
        while not o.step()["frame_finished"]:
            pass
    po, vo = o.get_particles()
    assert np.array_equal(pos, po) and np.array_equal(vel, vo)
