"""Host-side plumbing for several GPUs: independent scenes are the unit of work.

A single scene does not shard (its pressure solve needs global reductions every PCG
iteration), so one process per GPU owns whole scenes.  Scenes are spread by estimated
bytes moved per sub-step with a longest-first greedy assignment, which keeps every
rank's share within a few percent of the mean for the batched dam-break mix.  The only
collective is the max-over-ranks of a timing (or any other scalar) for reporting.
"""
from __future__ import annotations

from typing import Sequence


def scene_bytes_per_step(res: Sequence[int], n_particles: int) -> float:
    """Estimated device bytes moved per FLIP sub-step of one scene (particles: sort,
    P2G, SDF and G2P; faces: P2G, extrapolation, projection, G2P; cells: SDF, system)."""
    G = [r + 4 for r in res]
    C = G[0] * G[1] * G[2]
    F = (G[0] + 1) * G[1] * G[2] + G[0] * (G[1] + 1) * G[2] + G[0] * G[1] * (G[2] + 1)
    return n_particles * (72 + 24 + 12 + 48) + F * 45.0 + C * 24.0


def shard_scenes(costs: Sequence[float], world: int) -> list[list[int]]:
    """Deterministic longest-first greedy partition of scene indices over `world` ranks."""
    order = sorted(range(len(costs)), key=lambda i: (-costs[i], i))
    load = [0.0] * world
    parts: list[list[int]] = [[] for _ in range(world)]
    for i in order:
        r = min(range(world), key=lambda k: (load[k], k))
        parts[r].append(i)
        load[r] += costs[i]
    for p in parts:
        p.sort()
    return parts


def max_over_ranks(value: float) -> float:
    """Max of a scalar over all ranks of the default process group (identity without one)."""
    import torch
    import torch.distributed as dist
    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size() == 1:
        return float(value)
    dev = "cuda" if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor([float(value)], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())
