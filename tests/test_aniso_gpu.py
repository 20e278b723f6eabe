"""Anisotropic kernels on the GPU (bnn_flip_anisotropic_kernels / bnn_anisotropic_kernels)
against the oracle's restatement of AnisotropicKernelGenerator::computeAniKernels
(Simulation/SurfaceReconstruction/AniKernelGenerator.cpp:53-101).

Both sum every particle's neighbours in the canonical order of the same cell grid and use
only correctly rounded operations, so centres and kernel matrices must agree bit for bit.
At the 128^3 dam-break size the checks are the size-independent properties of the output.
"""
import numpy as np
import pytest
import torch

from banana_b200 import capi, scenes
from tests.test_aniso_cpu import _cloud

pytestmark = pytest.mark.gpu


def _eq(a, b, what):
    a = np.asarray(a)
    b = np.asarray(b)
    assert a.shape == b.shape
    if not np.array_equal(a, b):
        d = np.abs(a.astype(np.float64) - b.astype(np.float64))
        bad = np.argwhere(d > 0)
        raise AssertionError(f"{what}: {len(bad)} values differ, max {np.nanmax(d)}, first at {bad[0]}")


def _oracle_for(oracle_mod, pos, st, radius, **kw):
    return oracle_mod.aniso_kernels(pos, st["grid_bmin"], np.float32(st["grid_cell_size"]), st["grid_dims"], radius,
                                    **kw)


@pytest.mark.parametrize("steps", [0, 3])
def test_solver_particles_bitexact(bnn, oracle_mod, steps):
    cfg = scenes.dam_break_params(32)
    pos, vel = scenes.dam_break(32)
    g = bnn.FlipSolver(cfg)
    g.set_particles(pos, vel)
    for _ in range(steps):
        g.step()
    cen, mat, st = g.anisotropic_kernels()
    p, _ = g.get_particles()
    radius = np.float32(np.float32(cfg["cell_size"]) / np.float32(cfg.get("ratio_cell_size_p_radius", 2.0)))
    oc, om, osp = _oracle_for(oracle_mod, p, st, radius)
    assert st["sprays"] == osp
    _eq(cen, oc, "centres")
    _eq(mat, om, "kernel matrices")
    # the pass leaves the particles where they were (it only re-sorts them)
    p2, _ = g.get_particles()
    _eq(p2, p, "positions after the pass")


def test_solver_steps_unchanged_by_the_pass(bnn):
    """Frame output in the middle of a run does not change the run (each sub-step sorts by
    (cell, id) again)"""
    cfg = scenes.dam_break_params(24)
    pos, vel = scenes.dam_break(24)
    a = bnn.FlipSolver(cfg)
    b = bnn.FlipSolver(cfg)
    a.set_particles(pos, vel)
    b.set_particles(pos, vel)
    for s in range(4):
        a.step()
        b.step()
        if s == 1:
            b.anisotropic_kernels()
    pa, va = a.get_particles()
    pb, vb = b.get_particles()
    _eq(pb, pa, "positions")
    _eq(vb, va, "velocities")


@pytest.mark.parametrize("params", [{}, {"neighbor_threshold": 5, "position_blending": 0.9, "axis_ratio": 4.0},
                                    {"kernel_ratio": 4.0, "default_spray_size": 0.5}])
def test_standalone_points_bitexact(bnn, oracle_mod, params):
    pos = _cloud(11)
    radius = np.float32(1.0 / 64.0)
    prm = capi.aniso_params(radius, **params)
    n = len(pos)
    dp = torch.from_numpy(pos).cuda()
    dc = torch.zeros((n, 3), dtype=torch.float32, device="cuda")
    dm = torch.zeros((n, 9), dtype=torch.float32, device="cuda")
    st = capi.anisotropic_kernels_dev(dp.data_ptr(), n, prm, dc.data_ptr(), dm.data_ptr())
    torch.cuda.synchronize()
    kw = {k: v for k, v in params.items()}
    kw = {"threshold" if k == "neighbor_threshold" else
          "blend" if k == "position_blending" else
          "spray" if k == "default_spray_size" else k: v for k, v in kw.items()}
    oc, om, osp = _oracle_for(oracle_mod, pos, st, radius, **kw)
    assert st["sprays"] == osp
    assert np.allclose(st["grid_bmin"], pos.min(0))
    _eq(dc.cpu().numpy(), oc, "centres")
    _eq(dm.cpu().numpy(), om, "kernel matrices")


def test_standalone_edge_cases(bnn):
    radius = np.float32(0.01)
    prm = capi.aniso_params(radius)
    z = torch.zeros(3, dtype=torch.float32, device="cuda")
    # no points
    capi.anisotropic_kernels_dev(z.data_ptr(), 0, prm, z.data_ptr(), z.data_ptr())
    # a single point: a spray point, centre = the point
    one = torch.tensor([[0.3, 0.4, 0.5]], dtype=torch.float32, device="cuda")
    c = torch.zeros((1, 3), dtype=torch.float32, device="cuda")
    m = torch.zeros((1, 9), dtype=torch.float32, device="cuda")
    st = capi.anisotropic_kernels_dev(one.data_ptr(), 1, prm, c.data_ptr(), m.data_ptr())
    assert st["sprays"] == 1
    assert torch.equal(c, one)
    assert torch.equal(m.cpu(), torch.tensor([[0.75, 0, 0, 0, 0.75, 0, 0, 0, 0.75]], dtype=torch.float32))
    # invalid parameters and non-finite coordinates are refused
    with pytest.raises(capi.BnnError):
        capi.anisotropic_kernels_dev(one.data_ptr(), 1, capi.aniso_params(0.0), c.data_ptr(), m.data_ptr())
    bad = torch.tensor([[0.3, float("nan"), 0.5], [0.1, 0.1, 0.1]], dtype=torch.float32, device="cuda")
    c2 = torch.zeros((2, 3), dtype=torch.float32, device="cuda")
    m2 = torch.zeros((2, 9), dtype=torch.float32, device="cuda")
    with pytest.raises(capi.BnnError):
        capi.anisotropic_kernels_dev(bad.data_ptr(), 2, prm, c2.data_ptr(), m2.data_ptr())


def test_dam_break_128_properties(bnn):
    """At 128^3 (1.6M particles): every non-spray kernel has determinant 1, is symmetric to
    rounding and has eigenvalue ratios within axisRatio; centres stay within the kernel
    radius of their particle."""
    cfg = scenes.dam_break_params(128)
    pos, vel = scenes.dam_break(128)
    g = bnn.FlipSolver(cfg)
    g.set_particles(pos, vel)
    g.step()
    cen, mat, st = g.anisotropic_kernels()
    p, _ = g.get_particles()
    r = 8.0 * cfg["cell_size"] / 2.0
    assert np.all(np.linalg.norm(cen.astype(np.float64) - p, axis=1) < r)
    K = mat.reshape(-1, 3, 3).astype(np.float64)
    spray = np.all(K == np.diag([0.75] * 3)[None], axis=(1, 2))
    assert spray.sum() == st["sprays"]
    Kn = K[~spray]
    assert len(Kn) > 0.9 * len(K)
    assert np.abs(np.linalg.det(Kn) - 1.0).max() < 1e-4
    assert np.abs(Kn - Kn.transpose(0, 2, 1)).max() < 1e-5 * np.abs(Kn).max()
    w = np.linalg.eigvalsh(0.5 * (Kn + Kn.transpose(0, 2, 1)))
    assert (w[:, 2] / w[:, 0]).max() < 8.0 * (1 + 1e-4)
    assert w.min() > 0
