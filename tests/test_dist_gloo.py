"""Two ranks over gloo on CPU: scene sharding covers every scene exactly once with a
balanced load, and the max-over-ranks timing reduction the benchmark uses."""
import os
import socket

import numpy as np
import torch.multiprocessing as mp

from banana_b200 import dist as bd
from banana_b200 import scenes


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, q):
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=__import__("datetime").timedelta(seconds=60))
    specs = scenes.batch_scene_specs(256, seed=11)
    costs = []
    for s in specs:
        nx, ny, nz = s["res"]
        cells = [int(np.floor(f * r + 1e-9)) for f, r in zip(s["block_frac"], s["res"])]
        costs.append(bd.scene_bytes_per_step(s["res"], 8 * cells[0] * cells[1] * cells[2]))
    mine = bd.shard_scenes(costs, world)[rank]
    got = [None] * world
    dist.all_gather_object(got, mine)
    m = bd.max_over_ranks(10.0 + rank)
    dist.destroy_process_group()
    q.put((rank, got, m, [costs[i] for i in mine], sum(costs)))


def test_two_rank_sharding_and_max():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = [q.get(timeout=120) for _ in procs]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    res.sort()
    parts = res[0][1]
    assert parts == res[1][1]
    allidx = sorted(i for p in parts for i in p)
    assert allidx == list(range(256))
    assert res[0][2] == res[1][2] == 11.0
    loads = [sum(r[3]) for r in res]
    assert max(loads) / min(loads) < 1.05
