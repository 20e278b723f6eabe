"""Deterministic scene seeders for the dam-break and point-cloud workloads.

The reference's ParticleGenerator jitters with a process-global, default-seeded MT RNG and
appends from inside a parallel loop (Simulation/SimulationObjects/ParticleGenerator.cpp:
97-114, BananaCore/Banana/Utils/NumberHelpers.h:155-258), so its particle sets are not
reproducible.  These seeders replace it with a counter-based generator (SplitMix64 over
(seed, stream, counter)), so the same seed gives the same particles on every machine and
both the CUDA path and the oracle start from identical inputs.

Dam break: every grid cell lying entirely inside the fluid block [0,ex]x[0,ey]x[0,ez] of
the unit-cube domain gets `ppc` particles, each uniform inside its cell.  Particles are
listed cell by cell (z, then y, then x major-to-minor), `ppc` per cell.
"""
from __future__ import annotations

import math

import numpy as np

_GOLDEN = np.uint64(0x9E3779B97F4A7C15)
_M1 = np.uint64(0xBF58476D1CE4E5B9)
_M2 = np.uint64(0x94D049BB133111EB)


def splitmix64(x: np.ndarray) -> np.ndarray:
    """SplitMix64 finaliser of x (uint64 array), vectorised."""
    with np.errstate(over="ignore"):
        z = x.astype(np.uint64) + _GOLDEN
        z = (z ^ (z >> np.uint64(30))) * _M1
        z = (z ^ (z >> np.uint64(27))) * _M2
        return z ^ (z >> np.uint64(31))


def uniform01(seed: int, stream: int, counter: np.ndarray) -> np.ndarray:
    """Float64 in [0,1) with 53 random bits from (seed, stream, counter)."""
    with np.errstate(over="ignore"):
        key = splitmix64(np.uint64(seed) * _GOLDEN + np.uint64(stream) * np.uint64(0xD1B54A32D192ED03))
        bits = splitmix64(counter.astype(np.uint64) ^ key)
    return (bits >> np.uint64(11)).astype(np.float64) * (1.0 / 9007199254740992.0)


def dam_break_cells(n: int, block=(0.4, 0.6, 0.4)) -> tuple[int, int, int]:
    """Cells of an n^3 unit-cube grid lying fully inside the block (per axis)."""
    return tuple(int(math.floor(e * n + 1e-9)) for e in block)


def dam_break(n: int, block=(0.4, 0.6, 0.4), ppc: int = 8, seed: int = 42, domain_len=(1.0, 1.0, 1.0),
              cell_size: float | None = None):
    """Positions / velocities (float32, (N,3)) of the dam-break fluid block.

    n is the fluid-domain resolution (cells per unit length unless cell_size is given);
    block extents are in world units measured from the domain origin.
    """
    dx = (1.0 / n) if cell_size is None else float(cell_size)
    nx, ny, nz = (int(math.floor(e / dx + 1e-9)) for e in block)
    ncell = nx * ny * nz
    if ncell == 0:
        return np.zeros((0, 3), np.float32), np.zeros((0, 3), np.float32)
    cell = np.arange(ncell, dtype=np.int64)
    ci = cell % nx
    cj = (cell // nx) % ny
    ck = cell // (nx * ny)
    s = np.arange(ppc, dtype=np.int64)
    lin = (cell[:, None] * ppc + s[None, :]).ravel()
    pos = np.empty((ncell * ppc, 3), np.float32)
    for a, c in enumerate((ci, cj, ck)):
        u = uniform01(seed, a, lin)
        cc = np.repeat(c, ppc).astype(np.float64)
        p = ((cc + u) * dx).astype(np.float32)
        # rounding to float32 may land a sample on the next cell's face: keep it inside
        hi = ((cc + 1.0) * dx).astype(np.float32)
        pos[:, a] = np.where(p >= hi, np.nextafter(hi, np.float32(0)), p)
    vel = np.zeros_like(pos)
    return pos, vel


def dam_break_params(n: int, **over) -> dict:
    """Scene parameters of the dam break on an n^3 grid of the unit cube (config keys of
    the reference's scene JSON, see include/banana_b200.h bnn_params)."""
    p = dict(box_min=(0.0, 0.0, 0.0), box_max=(1.0, 1.0, 1.0), cell_size=float(np.float32(1.0 / n)),
             n_expand_cells=2, cfl_factor=1.0, min_timestep=1e-6, max_timestep=float(np.float32(1.0) / np.float32(30.0)),
             frame_duration=float(np.float32(1.0 / 30.0)), pic_flip_ratio=0.97, cg_relative_tolerance=1e-6,
             max_cg_iteration=5000, advection_steps=1, solver_kind=0, pcg_mode=0, preconditioner=0,
             refine_tolerance=1e-8, refine_inner_tolerance=1e-2, apply_gravity=1, correct_position=0,
             repulsive_force_stiffness=50.0, ratio_cell_size_p_radius=2.0)
    p.update(over)
    return p


def point_cloud(n_total: int = 4_000_000, n_blobs: int = 16, sigma: float = 0.03, seed: int = 7):
    """Config-3 point set: half uniform in [0,1)^3, half from `n_blobs` isotropic
    Gaussians (centres uniform in [0.1,0.9]^3).  A Gaussian sample outside [0,1)^3 is
    redrawn from the next counter until it lands inside.  float32 (N,3), uniform points
    first, then blob 0, blob 1, ..."""
    n_uni = n_total // 2
    n_g = n_total - n_uni
    per = n_g // n_blobs
    counts = [per + (1 if b < n_g - per * n_blobs else 0) for b in range(n_blobs)]
    pts = np.empty((n_total, 3), np.float32)
    idx = np.arange(n_uni, dtype=np.int64)
    for a in range(3):
        pts[:n_uni, a] = uniform01(seed, 10 + a, idx).astype(np.float32)
    cidx = np.arange(n_blobs, dtype=np.int64)
    centres = np.stack([0.1 + 0.8 * uniform01(seed, 20 + a, cidx) for a in range(3)], axis=1)
    o = n_uni
    for b in range(n_blobs):
        m = counts[b]
        out = np.empty((m, 3), np.float32)
        todo = np.arange(m, dtype=np.int64)
        attempt = 0
        while todo.size:
            ctr = (np.int64(b) << 40) + (np.int64(attempt) << 32) + todo
            # Box-Muller: three normals from two pairs of uniforms
            u1 = uniform01(seed, 100, ctr)
            u2 = uniform01(seed, 101, ctr)
            u3 = uniform01(seed, 102, ctr)
            u4 = uniform01(seed, 103, ctr)
            r1 = np.sqrt(-2.0 * np.log1p(-u1))
            r2 = np.sqrt(-2.0 * np.log1p(-u3))
            z = np.stack([r1 * np.cos(2 * np.pi * u2), r1 * np.sin(2 * np.pi * u2), r2 * np.cos(2 * np.pi * u4)], 1)
            p = (centres[b][None, :] + sigma * z).astype(np.float32)
            ok = np.all((p >= 0.0) & (p < 1.0), axis=1)
            out[todo[ok]] = p[ok]
            todo = todo[~ok]
            attempt += 1
        pts[o:o + m] = out
        o += m
    return pts


def batch_scene_specs(n_scenes: int = 256, seed: int = 11, choices=(32, 48, 64, 96, 128)):
    """Config-4 scene list: per-axis resolutions drawn from `choices`, block extents
    uniform in [0.2, 0.6] of the domain per axis.  The cell size is 1/64 for every scene,
    so an axis with N cells is N/64 long."""
    specs = []
    for s in range(n_scenes):
        r = uniform01(seed, 1, np.arange(s * 8, s * 8 + 8, dtype=np.int64))
        res = tuple(int(choices[min(int(r[a] * len(choices)), len(choices) - 1)]) for a in range(3))
        frac = tuple(float(0.2 + 0.4 * r[3 + a]) for a in range(3))
        specs.append({"res": res, "block_frac": frac, "seed": seed * 100003 + s})
    return specs


def batch_scene(spec: dict, ppc: int = 8, pcg_mode: int = 2, **over):
    """Parameters and particles of one batch scene (batch_scene_specs / serve_requests):
    domain [0, res/64] per axis with cell size 1/64, a dam-break block of block_frac of
    the domain anchored at the origin, `ppc` particles per cell, FP32 PCG refined to a
    1e-6 relative residual (FP64-checked), as the batch and serving configurations ask.
    The inner FP32 solves stop at 1e-3 of their start residual: two outer rounds reach
    1e-6 (measured on the 256-scene batch: 1e-2 1.33, 1e-3 1.39, 3e-4 1.28, 1e-4 1.19 G
    particle-steps/s)."""
    dx = 1.0 / 64.0
    res = spec["res"]
    ext = tuple(r * dx for r in res)
    block = tuple(f * e for f, e in zip(spec["block_frac"], ext))
    over = dict({"refine_tolerance": 1e-6, "refine_inner_tolerance": 1e-3}, **over)
    cfg = dam_break_params(64, box_max=ext, pcg_mode=pcg_mode, **over)
    pos, vel = dam_break(64, block=block, ppc=ppc, seed=spec["seed"], cell_size=dx)
    return cfg, pos, vel


def serve_requests(n_requests: int, rate: float = 20.0, seed: int = 13, n_min: int = 32, n_max: int = 192):
    """Request stream of the serving workload: Poisson arrivals (exponential gaps, mean
    1/rate seconds), each a cubic scene whose resolution is log-uniform in
    [n_min, n_max] (rounded), block extents uniform in [0.2, 0.6] of the domain."""
    reqs = []
    t = 0.0
    for q in range(n_requests):
        r = uniform01(seed, 2, np.arange(q * 8, q * 8 + 8, dtype=np.int64))
        t += -math.log1p(-r[0]) / rate
        n = int(round(math.exp(math.log(n_min) + r[1] * (math.log(n_max) - math.log(n_min)))))
        frac = tuple(float(0.2 + 0.4 * r[2 + a]) for a in range(3))
        reqs.append({"t": t, "res": (n, n, n), "block_frac": frac, "seed": seed * 100003 + q})
    return reqs
