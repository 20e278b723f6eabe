"""The C++ drop-in (FLIP_GPU_Solver through the bnn_flip_run driver: factory by scene
name, loadScene, doFrameSimulation per frame) computes the same frames as the solver
driven from Python, and the same as the oracle."""
import subprocess

import numpy as np
import pytest

from banana_b200 import build as bld
from banana_b200 import scenes
from oracle import bnn_reader
from tests.bnn_format import matrix_values, read_bnn, values
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


def test_memory_state_resume_and_bnn_frames(bnn, tmp_path):
    """SaveMemoryState / LoadMemoryState (PIC_Solver.cpp:158-232): a run that stops after
    frame 2 and a second run resuming from its state file reach frame 3 with exactly the
    particles of one straight 3-frame run.  The .bnn frame files hold the frame's particles
    (16-bit compressed positions, within one quantisation step)."""
    exe = bld.build_host()
    n = 16
    data = tmp_path / "data"
    common = {"DataPath": str(data), "FramePerState": 2, "OptionalSavingData": ["ParticleVelocity", "ObjectIndex"]}

    def run(name, frames, **g):
        sc = tmp_path / f"{name}.json"
        sc.write_text(dam_break_scene(n, frames=frames, **dict(common, **g)))
        out = tmp_path / f"{name}.f32"
        r = subprocess.run([str(exe), str(sc), "--out", str(out)], capture_output=True, text=True, timeout=300)
        assert r.returncode == 0, r.stderr
        return read_particles(out), r.stdout

    (p3, v3), _ = run("straight", 3, SaveFrameData=True, FrameDataFolder="straight")
    (p2, _), _ = run("first", 2, SaveMemoryState=True, MemoryStateDataFolder="state")
    assert (data / "state" / "frame.0002.bnn").exists()
    (pr, vr), out = run("resume", 3, LoadMemoryState=True, MemoryStateDataFolder="state")
    assert '"resumed_after_frame": 2' in out
    assert np.array_equal(pr, p3) and np.array_equal(vr, v3)

    cnt, attrs, _ = read_bnn(data / "straight" / "frame.0003.bnn")
    assert cnt == len(p3)
    dec, lo, hi, _ = values(attrs["particle_position"])
    assert np.abs(dec - p3).max() <= (hi - lo).max() / 65535 * 1.01
    assert attrs["particle_radius"]["type"] == "real"
    assert list(values(attrs["object_index"])) == [0] * cnt
    st_n, st, _ = read_bnn(data / "state" / "frame.0002.bnn")
    assert np.array_equal(values(st["particle_position"]).reshape(-1, 3), p2)
    assert list(values(st["grid_resolution"])) == [n + 4] * 3
    # the same files through the restatement of the reference's own reader
    rn, rfixed, rpart = bnn_reader.read(data / "straight" / "frame.0003.bnn")
    assert rn == cnt
    assert np.array_equal(bnn_reader.particle_attribute(rn, rpart, "particle_position"), dec)
    assert list(bnn_reader.particle_attribute(rn, rpart, "object_index")) == [0] * cnt
    sn, sfixed, spart = bnn_reader.read(data / "state" / "frame.0002.bnn")
    assert np.array_equal(bnn_reader.particle_attribute(sn, spart, "particle_position"), p2)
    assert list(bnn_reader.fixed_attribute(sfixed, "grid_resolution")) == [n + 4] * 3


def test_anikernel_frame_output(bnn, tmp_path):
    """OptionalSavingData "AniKernel" (PIC_Solver.cpp:248-252): the frame file's positions
    are the anisotropic kernel centres and "anisotropic_kernel" holds the 3x3 matrices
    (16-bit compressed with one range for all entries), as the solver API computes them."""
    exe = bld.build_host()
    n = 16
    data = tmp_path / "data"
    sc = tmp_path / "ani.json"
    sc.write_text(dam_break_scene(n, frames=1, DataPath=str(data), SaveFrameData=True, FrameDataFolder="ani",
                                  OptionalSavingData=["AniKernel"]))
    r = subprocess.run([str(exe), str(sc)], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr
    cnt, attrs, order = read_bnn(data / "ani" / "frame.0001.bnn")
    assert order == ["particle_radius", "anisotropic_kernel", "particle_position"]
    assert attrs["anisotropic_kernel"]["count"] == 9 and attrs["anisotropic_kernel"]["bytes"] == 8 + 18 * cnt

    cfg = scenes.dam_break_params(n)
    p0, v0 = scenes.dam_break(n)
    s = bnn.FlipSolver(cfg)
    s.set_particles(p0, v0)
    s.advance_frame()
    cen, mat, st = s.anisotropic_kernels()
    assert cnt == len(cen)
    dec, lo, hi, _ = values(attrs["particle_position"])
    assert np.abs(dec - cen).max() <= (hi - lo).max() / 65535 * 1.01
    K, klo, khi, _ = matrix_values(attrs["anisotropic_kernel"])
    assert klo == mat.min() and khi == mat.max()
    assert np.abs(K - mat).max() <= (khi - klo) / 65535 * 1.01
    # the reference's reader (restated) decodes the same kernels
    rn, _, rpart = bnn_reader.read(data / "ani" / "frame.0001.bnn")
    assert np.array_equal(bnn_reader.particle_attribute(rn, rpart, "anisotropic_kernel", matrix_dim=3), K)
    assert np.array_equal(bnn_reader.particle_attribute(rn, rpart, "particle_position"), dec)


def test_driver_boundary_objects(bnn, tmp_path):
    """AdditionalBoundaryObjects through the C++ driver: a static box equal to the domain
    box changes nothing (the CSG union of two equal boxes is the box), and a box container
    rotating about z (linear keyframes, moved before every sub-step after frame 1, the
    boundary SDF recomputed each time) keeps the fluid inside it."""
    import json
    exe = bld.build_host()
    n = 20

    def run(name, objects, frames):
        sc = json.loads(dam_break_scene(n, frames=frames))
        sc["AdditionalBoundaryObjects"] = objects
        path = tmp_path / f"{name}.json"
        path.write_text(json.dumps(sc))
        out = tmp_path / f"{name}.f32"
        r = subprocess.run([str(exe), str(path), "--out", str(out)], capture_output=True, text=True, timeout=300)
        assert r.returncode == 0, r.stderr
        return read_particles(out), r.stdout

    (p0, v0), _ = run("plain", [], 2)
    (p1, v1), _ = run("same", [{"GeometryType": "Box", "BoxMin": [0, 0, 0], "BoxMax": [1, 1, 1]}], 2)
    assert np.array_equal(p0, p1) and np.array_equal(v0, v1)

    rot = {"GeometryType": "Box", "BoxMin": [-0.45, -0.45, -0.45], "BoxMax": [0.45, 0.45, 0.45],
           "Translation": [0.5, 0.5, 0.5],
           "Animation": {"CubicInterpolationRotation": False,
                         "KeyFrames": [{"Frame": 1, "Translation": [0.5, 0.5, 0.5], "RotationAxisAngle": [0, 0, 1, 0]},
                                       {"Frame": 4, "Translation": [0.5, 0.5, 0.5], "RotationAxisAngle": [0, 0, 1, 30]}]}}
    (p2, v2), out = run("rot", [rot], 4)
    assert out.count('"frame"') == 4
    assert np.isfinite(p2).all() and np.isfinite(v2).all()
    # at the end of frame 4 the box has turned by 30 * (3 + fraction) / 3 degrees at most:
    # every particle lies inside the box turned by the angle of the last sub-step, to a cell
    ang = np.radians(30.0)
    c, s = np.cos(ang), np.sin(ang)
    q = p2.astype(np.float64) - 0.5
    local = np.stack([c * q[:, 0] + s * q[:, 1], -s * q[:, 0] + c * q[:, 1], q[:, 2]], 1)
    assert np.all(np.abs(local) <= 0.45 + 2.0 / n)


def test_reference_scene_through_the_drop_in(bnn, tmp_path):
    """The reference's own FLIP3D_2DamBreak scene (Applications/QtApps/ParticleSimulation/
    Scenes, with only "Solver" changed to FLIP_GPU_3DSolver; tests/golden/scenes) through the
    factory, loadScene and doFrameSimulation: two box generators, position correction,
    two advection steps, frame files written under the scene's own DataPath (relative to
    the working directory here) and readable by the reference's reader."""
    import json
    from pathlib import Path
    exe = bld.build_host()
    scene = Path(__file__).resolve().parent / "golden" / "scenes" / "FLIP3D_2DamBreak.json"
    sc = json.loads(scene.read_text())
    assert sc["GlobalParameters"]["Solver"] == "FLIP_GPU_3DSolver"
    out = tmp_path / "p.f32"
    r = subprocess.run([str(exe), str(scene), "--frames", "2", "--out", str(out)], capture_output=True, text=True,
                       timeout=600, cwd=tmp_path)
    assert r.returncode == 0, r.stderr[-2000:]
    head = json.loads(r.stdout.splitlines()[0])
    assert head["solver"] == "FLIP_GPU_3DSolver"
    frames = [json.loads(l) for l in r.stdout.splitlines()[1:] if l.startswith("{")]
    assert [f["frame"] for f in frames] == [1, 2] and all(f["substeps"] >= 1 for f in frames)
    pos, vel = read_particles(out)
    assert len(pos) == head["particles"] > 0
    lo = np.array(sc["SimulationParameters"]["SimulationDomainBox"]["BoxMin"], np.float32)
    hi = np.array(sc["SimulationParameters"]["SimulationDomainBox"]["BoxMax"], np.float32)
    # the box projection (BoundaryObject::constrainToBoundary, BoundaryObject.cpp:72-90)
    # moves a particle along a finite-difference gradient (GeometryObjects.cpp:37-85), which
    # near the box's edges and corners can leave it a little outside: allow one particle
    # radius (cell size / RatioCellSizePRadius)
    radius = sc["SimulationParameters"]["CellSize"] / 2.0
    excursion = float(max((lo - pos).max(), (pos - hi).max(), 0.0))
    assert excursion <= radius, excursion
    assert np.all(np.isfinite(vel))
    g = sc["GlobalParameters"]
    frame = tmp_path / g["DataPath"] / g["FrameDataFolder"] / "frame.0002.bnn"
    n, fixed, part = bnn_reader.read(frame)
    assert n == len(pos)
    # the scene asks for "anisotropic_kernel" and "object_index", but the reference's
    # saveFrameData tests the names "AniKernel" and "ObjectIndex" (PIC_Solver.cpp:240-255),
    # so, as there, the frame holds the particle radius and positions only
    assert sorted(fixed) == ["particle_radius"] and sorted(part) == ["particle_position"]
    p = bnn_reader.particle_attribute(n, part, "particle_position")
    assert np.abs(p - pos).max() <= (pos.max(0) - pos.min(0)).max() / 65535 * 1.01
