"""Edge cases of the sub-step against the oracle: no particles, a single particle,
particles that start on or outside the domain box (the box projection brings them in),
and cells crowded with hundreds of particles.
Every particle and grid field must agree bit for bit after every sub-step."""
import numpy as np
import pytest

from banana_b200 import capi, scenes

pytestmark = pytest.mark.gpu

_FIELDS = ("u", "v", "w", "phi", "pressure", "old_u", "old_v", "old_w")


def _run(bnn, oracle_mod, pos, vel, steps, n=16):
    cfg = scenes.dam_break_params(n)
    g = bnn.FlipSolver(cfg)
    o = oracle_mod.Oracle(cfg)
    g.set_particles(pos, vel)
    o.set_particles(pos, vel)
    for s in range(steps):
        sg = g.step()
        so = o.step()
        assert sg["dt"] == so["dt"] and sg["n_active"] == so["n_active"], s
        assert sg["pcg_iterations"] == so["pcg_iterations"], s
        for f in _FIELDS:
            a, b = g.grid(f), o.grid(capi.FIELD[f])
            assert np.array_equal(a, b), (s, f, float(np.abs(a - b).max()))
        if len(pos):
            pg, vg = g.get_particles()
            po, vo = o.get_particles()
            assert np.array_equal(pg, po) and np.array_equal(vg, vo), s
    return g


def test_no_particles(bnn, oracle_mod):
    z = np.zeros((0, 3), np.float32)
    g = _run(bnn, oracle_mod, z, z, 3)
    st = g.step()
    assert st["n_active"] == 0 and st["pcg_success"] == 1


def test_single_particle(bnn, oracle_mod):
    pos = np.array([[0.31, 0.52, 0.47]], np.float32)
    vel = np.array([[0.2, 0.0, -0.1]], np.float32)
    _run(bnn, oracle_mod, pos, vel, 6)


def test_particles_on_and_outside_the_box(bnn, oracle_mod):
    """The dam block plus particles exactly on the walls and a little outside them (inside
    the 2-cell padding): the first advection projects them back into the box"""
    pos, vel = scenes.dam_break(16)
    extra = np.array([[0.0, 0.5, 0.5], [1.0, 0.25, 0.75], [0.5, 0.0, 0.5], [0.5, 1.0, 0.5],
                      [-0.05, 0.3, 0.3], [0.4, -0.06, 0.2], [1.07, 0.9, 0.1], [0.2, 0.2, 1.1]], np.float32)
    p = np.concatenate([pos, extra]).astype(np.float32)
    v = np.concatenate([vel, np.zeros_like(extra)]).astype(np.float32)
    g = _run(bnn, oracle_mod, p, v, 4)
    pg, _ = g.get_particles()
    assert np.all(pg >= 0.0) and np.all(pg <= 1.0)


def test_crowded_cells(bnn, oracle_mod):
    """Hundreds of particles in a few cells (the cell sort's large-bucket path), among the
    dam block"""
    pos, vel = scenes.dam_break(16)
    rng = np.random.default_rng(3)
    pile = (np.array([0.71, 0.2, 0.63]) + rng.uniform(0, 0.02, size=(400, 3))).astype(np.float32)
    pile2 = (np.array([0.3, 0.8, 0.8]) + rng.uniform(0, 0.05, size=(2500, 3))).astype(np.float32)
    p = np.concatenate([pos, pile, pile2]).astype(np.float32)
    v = np.concatenate([vel, np.zeros_like(pile), np.zeros_like(pile2)]).astype(np.float32)
    _run(bnn, oracle_mod, p, v, 4)
