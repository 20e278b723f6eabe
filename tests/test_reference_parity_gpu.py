"""Parity of the CUDA path with the reference's own arithmetic, at the sizes of the benchmark
configurations.

The bit-exact tests (test_flip_parity_gpu.py and others) hold the CUDA path to the
oracle's canonical mode, which sums the PCG's dot products in FP64 in the kernels' fixed
chunk order.  Here the CUDA path is held to the oracle in reference mode: FP32 accumulators
summed serially left to right (PCGSolver::solve_precond, PCGSolver.cpp:143-199, with
ParallelBLAS::dotProduct, ParallelBLAS.h:40-48, on one thread), and P2G summed in
particle-array order (FLIP_Solver::mapParticles2Grid, FLIP_Solver.cpp:57-95, on one
thread, particles never re-sorted), i.e. what the reference computes on one TBB thread.

Tolerances are the spec's: grid velocities and pressure within 1e-5 relative, particle
positions within 1e-4 dx after 100 steps.  Relative means against the flow's top speed
(the largest |u|, |v|, |w| of the reference run at that step): with the reference's static
box the walls act only through the particle projection (the boundary SDF is never computed
for a static scene, PIC_Solver.cpp:105-114), so the block falls freely and u, w and the
pressure stay rounding noise around 0 in both runs, and a per-field relative error would
divide noise by noise.  The pressure is measured by the velocity change it makes,
dt * max|delta p| (the update is u -= dt * (p_c - p_l) / theta, PIC_Solver.cpp:911-981),
against the same top speed.
"""
import ctypes as C
import os

import numpy as np
import pytest
import torch

from banana_b200 import scenes

pytestmark = pytest.mark.gpu

TOL_GRID = 1e-5      # grid velocities and pressure, relative to the top speed
TOL_POS_DX = 1e-4    # particle positions, in cells


def _errors(sg, g, o, f64=False):
    """max errors of u, v, w (over the top speed), the pressure (dt * |dp| over the top
    speed) and the step size (relative) between the GPU solver g and the oracle o"""
    ref = {w: o.grid(w, f64=True) if f64 else o.grid(w).astype(np.float64) for w in (0, 1, 2, 4)}
    top = max(float(np.abs(ref[w]).max()) for w in (0, 1, 2))
    e = {}
    for name, w in (("u", 0), ("v", 1), ("w", 2)):
        e[name] = float(np.abs(g.grid(w).astype(np.float64) - ref[w]).max()) / top
    e["pressure"] = sg["dt"] * float(np.abs(g.grid(4).astype(np.float64) - ref[4]).max()) / top
    return e


def test_config1_against_reference_order_100_steps(bnn, oracle_mod):
    """64^3 dam break (190,000 particles), FP32 Jacobi PCG to 1e-6, 100 sub-steps."""
    n = 64
    dx = 1.0 / n
    pos, vel = scenes.dam_break(n)
    g = bnn.FlipSolver(scenes.dam_break_params(n))
    g.set_particles(pos, vel)
    o = oracle_mod.Oracle(scenes.dam_break_params(n, reduce_mode=0, nthreads=1, sort_each_step=0))
    o.set_particles(pos, vel)
    worst = {}
    tg = to = 0.0
    for step in range(100):
        sg = g.step()
        so = o.step()
        assert sg["pcg_success"] == so["pcg_success"] == 1, step
        # the simulated time: a sub-step at a frame's end is the rest of the frame
        # (PIC_Solver.cpp:284-290), a small difference of larger numbers, so single step
        # sizes there differ relatively more than the velocities they come from
        tg += sg["dt"]
        to += so["dt"]
        assert abs(tg - to) <= TOL_GRID * to, (step, tg, to)
        e = _errors(sg, g, o)
        for k, v in e.items():
            worst[k] = max(worst.get(k, 0.0), v)
            assert v <= TOL_GRID, f"step {step}: {k} error {v:.3e} over the top speed"
    pg, _ = g.get_particles()
    po, _ = o.get_particles()
    pos_err = float(np.abs(pg.astype(np.float64) - po).max()) / dx
    print("worst grid errors over 100 steps:", worst, "position error / dx:", pos_err)
    assert pos_err <= TOL_POS_DX


@pytest.mark.slow
def test_config2_first_10_steps(bnn, oracle_mod):
    """256^3 dam break (12,734,496 particles): the FP64-PCG and the refined (FP32 inner,
    FP64 outer to 1e-8) GPU runs against the FP64 build of the oracle in reference order
    (RealType = double, the reference's DOUBLE_PRECISION build, Setup.h:50-59) over the
    first 10 sub-steps, and the FP64-PCG run bit for bit against the oracle's canonical
    mode."""
    n = 256
    dx = 1.0 / n
    pos, vel = scenes.dam_break(n)
    threads = os.cpu_count() or 1
    oracle_mod.set_threads(threads)
    # every stage of the canonical mode is deterministic on any number of threads
    tol = dict(cg_relative_tolerance=1e-8, nthreads=threads)
    runs = {"fp64": bnn.FlipSolver(scenes.dam_break_params(n, pcg_mode=1, **tol)),
            "refined": bnn.FlipSolver(scenes.dam_break_params(n, pcg_mode=2))}
    for s in runs.values():
        s.set_particles(pos, vel)
    can = oracle_mod.Oracle(scenes.dam_break_params(n, pcg_mode=1, **tol))
    can.set_particles(pos, vel)
    d64 = oracle_mod.Oracle(scenes.dam_break_params(n, reduce_mode=0, sort_each_step=0, pcg_mode=1, **tol),
                            use_double=True)
    d64.set_particles(pos, vel)
    for step in range(10):
        sc = can.step()
        sd = d64.step()
        st = {k: s.step() for k, s in runs.items()}
        # FP64 PCG: bit equality with the canonical oracle
        assert st["fp64"]["dt"] == sc["dt"] and st["fp64"]["pcg_iterations"] == sc["pcg_iterations"], step
        for w in (0, 1, 2, 3, 4):
            assert np.array_equal(runs["fp64"].grid(w), can.grid(w)), (step, w)
        pg, vg = runs["fp64"].get_particles()
        pc, vc = can.get_particles()
        assert np.array_equal(pg, pc) and np.array_equal(vg, vc), step
        # both runs against the FP64 reference build
        po, _ = d64.get_particles(f64=True)
        for name, s in runs.items():
            assert st[name]["pcg_success"] == 1, (step, name)
            assert abs(st[name]["frame_time"] - sd["frame_time"]) <= TOL_GRID * sd["frame_time"], (step, name)
            e = _errors(st[name], s, d64, f64=True)
            for k, v in e.items():
                assert v <= TOL_GRID, f"step {step} {name}: {k} error {v:.3e} over the top speed"
            p, _ = s.get_particles()
            assert float(np.abs(p.astype(np.float64) - po).max()) / dx <= TOL_POS_DX, (step, name)
    for s in runs.values():
        s.close()
    can.close()
    d64.close()


def _dev(a):
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


@pytest.mark.slow
def test_config3_4m_points(bnn, oracle_mod):
    """4M points (half uniform, half from 16 Gaussian blobs, seed 7), cell = radius = 0.01:
    cell ids, sorted index and cell offsets bit for bit; neighbour lists equal (each list
    sorted ascending on both sides, so the flat arrays must match)."""
    oracle_mod.set_threads(os.cpu_count() or 1)
    pts = scenes.point_cloud(4_000_000, seed=7)
    n = len(pts)
    bmin = np.zeros(3, np.float32)
    nc = np.array([100, 100, 100], np.int32)
    cid, srt, start, oor = oracle_mod.cell_sort(pts, bmin, np.float32(0.01), nc)
    L = bnn.load()
    p = _dev(pts)
    gc = torch.zeros(n, dtype=torch.int32, device="cuda")
    gs = torch.zeros(n, dtype=torch.int32, device="cuda")
    gst = torch.zeros(int(nc.prod()) + 1, dtype=torch.int32, device="cuda")
    o = C.c_uint32()
    rc = L.bnn_cell_sort(C.c_void_p(p.data_ptr()), n, bmin.ctypes.data_as(C.POINTER(C.c_float)), 0.01,
                         nc.ctypes.data_as(C.POINTER(C.c_int32)), C.c_void_p(gc.data_ptr()), C.c_void_p(gs.data_ptr()),
                         C.c_void_p(gst.data_ptr()), C.byref(o), None)
    torch.cuda.synchronize()
    assert rc == 0 and o.value == oor
    assert np.array_equal(gc.cpu().numpy().view(np.uint32), cid)
    assert np.array_equal(gs.cpu().numpy().view(np.uint32), srt)
    assert np.array_equal(gst.cpu().numpy().view(np.uint32), start)
    del gc, gs, gst
    off_o, idx_o = oracle_mod.neighbors(pts, np.float32(0.01))
    cap = int(off_o[-1])
    goff = torch.zeros(n + 1, dtype=torch.int64, device="cuda")
    gidx = torch.zeros(cap, dtype=torch.int32, device="cuda")
    tot = C.c_uint64()
    rc = L.bnn_neighbors(C.c_void_p(p.data_ptr()), n, 0.01, C.c_void_p(goff.data_ptr()), C.c_void_p(gidx.data_ptr()),
                         cap, C.byref(tot), None)
    assert rc == 0 and tot.value == off_o[-1]
    assert np.array_equal(goff.cpu().numpy().view(np.uint64), off_o)
    # set equality per point: sort every GPU list (key = point << 32 | neighbour) and
    # compare with the oracle's lists, which are ascending
    counts = torch.diff(goff)
    owner = torch.repeat_interleave(torch.arange(n, device="cuda", dtype=torch.int64), counts)
    key = (owner << 32) | (gidx.to(torch.int64) & 0xffffffff)
    del owner, gidx
    key = torch.sort(key).values
    got = (key & 0xffffffff).to(torch.int32)
    del key
    assert np.array_equal(got.cpu().numpy().view(np.uint32), idx_o)
