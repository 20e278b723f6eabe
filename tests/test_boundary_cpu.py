"""Boundary objects in the oracle: analytic checks of the boundary SDF, the face weights
(computeCellWeights with Batty's fraction_inside of the four face corners), and the
particle projection, with no GPU."""
import numpy as np

from banana_b200 import capi, scenes
from oracle import oracle as O


def _oracle(n=20):
    cfg = scenes.dam_break_params(n)
    o = O.Oracle(cfg)
    pos, vel = scenes.dam_break(n)
    o.set_particles(pos, vel)
    return o, cfg


def test_node_sdf_and_weights_of_an_axis_aligned_container():
    o, cfg = _oracle(20)
    dx = cfg["cell_size"]
    lo, hi = 0.225, 0.775           # walls half way between grid nodes
    o.set_boundaries([capi.boundary_object("box", (lo, lo, lo), (hi, hi, hi), dynamic=True)])
    G = o.G
    sdf = o.grid(12)                # (z, y, x) nodes
    x = -2 * dx + np.arange(G[0] + 1) * dx
    X, Y, Z = np.meshgrid(x, x, x, indexing="ij")
    inner = np.minimum.reduce([X - lo, hi - X, Y - lo, hi - Y, Z - lo, hi - Z]).transpose(2, 1, 0)
    # inside the container the SDF is the distance to the nearest wall (positive)
    inside = inner > 0
    np.testing.assert_allclose(sdf[inside], np.minimum(inner[inside], 1.0), atol=1e-6)
    assert np.all(sdf[~inside] <= 1e-7)
    wu = o.grid(9)                  # (z, y, x) of the u faces
    # a u face at x inside, spanning y/z cells that straddle a wall half way: weight 1/2
    i = int(round((0.5 + 2 * dx) / dx))
    j = int((lo + 2 * dx) / dx)     # the cell containing the lower y wall
    k = int(round((0.5 + 2 * dx) / dx))
    assert abs(wu[k, j, i] - 0.5) < 1e-5
    assert wu[k, j + 3, i] == 1.0 and wu[k, 1, i] == 0.0
    assert wu.min() == 0.0 and wu.max() == 1.0


def test_static_objects_leave_the_grid_alone_and_project_particles():
    o, cfg = _oracle(20)
    o.set_boundaries([capi.boundary_object("sphere", translation=(0.5, 0.5, 0.5), scale=0.6)])
    assert np.all(o.grid(9) == 1.0) and np.all(o.grid(12) == 0.0)
    o.step()
    p, _ = o.get_particles()
    # the dam block's corner lies outside the sphere: every particle was projected in
    assert np.all(np.linalg.norm(p.astype(np.float64) - 0.5, axis=1) <= 0.6 + 1e-5)


def test_transform_of_a_rotated_box_matches_the_analytic_distance():
    # box rotated 90 degrees about z maps x <-> y: the SDF at a node equals the unrotated
    # box's with the coordinates swapped
    o, cfg = _oracle(20)
    ob = capi.boundary_object("box", (-0.3, -0.1, -0.2), (0.3, 0.1, 0.2), translation=(0.5, 0.5, 0.5),
                              axis_angle=(0, 0, 1, np.pi / 2), dynamic=True)
    o.set_boundaries([ob])
    dx = cfg["cell_size"]
    sdf = o.grid(12)
    x = -2 * dx + np.arange(o.G[0] + 1) * dx
    X, Y, Z = np.meshgrid(x, x, x, indexing="ij")
    # rotated: half extents 0.1 along x, 0.3 along y, 0.2 along z
    inner = np.minimum.reduce([0.1 - np.abs(X - 0.5), 0.3 - np.abs(Y - 0.5), 0.2 - np.abs(Z - 0.5)])
    inner = inner.transpose(2, 1, 0)
    inside = inner > 1e-4
    np.testing.assert_allclose(sdf[inside], inner[inside], atol=2e-6)
