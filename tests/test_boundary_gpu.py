"""Boundary objects beyond the domain box (bnn_flip_set_boundaries) against the oracle.

Static objects only constrain the particles (the reference computes no boundary SDF for
static scenes); a dynamic object turns on the grid side: boundary SDF on the nodes, face
weights, the solid part of the fluid SDF, the weighted pressure system (per-face
off-diagonals in the PCG) and constrainGridVelocity.  The boundary is reset at the start
of every frame with the object's new transformation, as PIC_Solver::advanceScene does.
Every particle and grid field must agree bit for bit.
"""
import numpy as np
import pytest

from banana_b200 import capi, scenes

pytestmark = pytest.mark.gpu

_FIELDS = ("u", "v", "w", "phi", "pressure", "old_u", "old_v", "old_w")


def _sphere():
    return capi.boundary_object("sphere", translation=(0.5, 0.5, 0.5), scale=0.8)


def _rotating_box(frame):
    return capi.boundary_object("box", (-0.45, -0.45, -0.45), (0.45, 0.45, 0.45), translation=(0.5, 0.5, 0.5),
                                axis_angle=(0.0, 0.0, 1.0, 0.1 * frame), dynamic=True)


def _moving_sphere(frame):
    return capi.boundary_object("sphere", translation=(0.5 + 0.02 * frame, 0.55, 0.5), scale=0.62, dynamic=True)


def _pair(bnn, oracle_mod, n, **over):
    cfg = scenes.dam_break_params(n, **over)
    pos, vel = scenes.dam_break(n)
    g = bnn.FlipSolver(cfg)
    g.set_particles(pos, vel)
    o = oracle_mod.Oracle(cfg)
    o.set_particles(pos, vel)
    return g, o


def _same(a, b, what):
    a = np.asarray(a)
    b = np.asarray(b)
    if not np.array_equal(a, b):
        d = np.abs(a.astype(np.float64) - b.astype(np.float64))
        raise AssertionError(f"{what}: {int((d > 0).sum())} values differ, max {np.nanmax(d)}")


def _check(g, o, tag, fields=_FIELDS):
    for f in fields:
        _same(g.grid(f), o.grid(capi.FIELD[f]), f"{tag} {f}")
    pg, vg = g.get_particles()
    po, vo = o.get_particles()
    _same(pg, po, f"{tag} positions")
    _same(vg, vo, f"{tag} velocities")


def _run_frames(g, o, frames, objects):
    for f in range(frames):
        objs = objects(f)
        g.set_boundaries(objs)
        o.set_boundaries(objs)
        if any(ob.dynamic for ob in objs):
            for fld in ("weight_u", "weight_v", "weight_w", "boundary_sdf"):
                _same(g.grid(fld), o.grid(capi.FIELD[fld]), f"frame {f} {fld}")
        for s in range(40):
            sg = g.step()
            so = o.step()
            assert sg["dt"] == so["dt"] and sg["n_active"] == so["n_active"], (f, s)
            assert sg["pcg_iterations"] == so["pcg_iterations"] and sg["pcg_success"] == 1, (f, s)
            _check(g, o, f"frame {f} step {s}")
            if sg["frame_finished"]:
                break


def test_static_objects_constrain_particles_only(bnn, oracle_mod):
    g, o = _pair(bnn, oracle_mod, 24)
    _run_frames(g, o, 2, lambda f: [_sphere()])
    # static objects leave the grid side alone (weights 1, no boundary SDF)
    assert np.all(g.grid("weight_u") == 1.0) and np.all(g.grid("boundary_sdf") == 0.0)
    # one projection per sub-step against the union's SDF: particles end on or near the
    # sphere, within a cell where its wall meets the box's
    p, _ = g.get_particles()
    assert np.all(np.linalg.norm(p - 0.5, axis=1) <= 0.8 + 1.0 / 24)


def test_dynamic_box_flip(bnn, oracle_mod):
    g, o = _pair(bnn, oracle_mod, 24)
    _run_frames(g, o, 3, lambda f: [_sphere(), _rotating_box(f)])
    w = g.grid("weight_u")
    assert w.min() == 0.0 and 0.0 < w[(w > 0) & (w < 1)].size


@pytest.mark.parametrize("kind", [1, 2, 3])
def test_dynamic_sphere_variants(bnn, oracle_mod, kind):
    """APIC, AFLIP and PIC with a moving sphere container"""
    g, o = _pair(bnn, oracle_mod, 20, solver_kind=kind)
    _run_frames(g, o, 2, lambda f: [_moving_sphere(f)])


@pytest.mark.parametrize("mode", [1, 2])
def test_dynamic_boundary_fp64_and_refined(bnn, oracle_mod, mode):
    """FP64 and refined solves read the per-face off-diagonals too"""
    g, o = _pair(bnn, oracle_mod, 20, pcg_mode=mode)
    _run_frames(g, o, 1, lambda f: [_moving_sphere(f)])


def test_clearing_boundaries_restores_the_box(bnn):
    cfg = scenes.dam_break_params(20)
    pos, vel = scenes.dam_break(20)
    a = bnn.FlipSolver(cfg)
    b = bnn.FlipSolver(cfg)
    a.set_particles(pos, vel)
    b.set_particles(pos, vel)
    b.set_boundaries([_moving_sphere(0)])
    b.set_boundaries([])
    for _ in range(4):
        a.step()
        b.step()
    pa, va = a.get_particles()
    pb, vb = b.get_particles()
    _same(pb, pa, "positions")
    _same(vb, va, "velocities")
