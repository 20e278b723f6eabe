"""Host logic of the serving loop (banana_b200.serving.SceneServer) against a fake scene
batch: arrival-order admission against a byte budget, waiting for memory, re-batching
every step, retirement after each request's sub-steps."""
import numpy as np
import pytest

from banana_b200.serving import CAPACITY, Request, SceneServer


class _Full(Exception):
    code = CAPACITY


class FakeBatch:
    """Admits scenes while the sum of their particle counts fits `budget`."""

    def __init__(self, budget):
        self.budget = budget
        self.scenes = {}
        self.next = 0
        self.log = []

    def add_scene(self, cfg, pos, vel):
        used = sum(len(p) for p, _, _ in self.scenes.values())
        if used + len(pos) > self.budget:
            raise _Full()
        sid = self.next
        self.next += 1
        self.scenes[sid] = [pos.copy(), vel.copy(), 0]
        self.log.append(("add", cfg["rid"]))
        return sid

    def step(self):
        ps = 0
        for s in self.scenes.values():
            s[0] += 1.0
            s[2] += 1
            ps += len(s[0])
        return {"wall_ms": 1.0, "particle_steps": ps}

    def scene_info(self, sid):
        s = self.scenes[sid]
        return {"steps": s[2], "n": len(s[0])}

    def get_scene(self, sid):
        return self.scenes[sid][0], self.scenes[sid][1]

    def remove_scene(self, sid):
        self.log.append(("remove", sid))
        del self.scenes[sid]


class Clock:
    def __init__(self):
        self.t = 0.0

    def __call__(self):
        return self.t


def _req(rid, n, steps, arrival):
    return Request(rid, {"rid": rid}, np.zeros((n, 3), np.float32), np.zeros((n, 3), np.float32), steps, arrival)


def test_admission_in_arrival_order_with_wait_for_memory():
    clk = Clock()
    b = FakeBatch(budget=100)
    srv = SceneServer(b, clock=clk)
    # 60 + 50 do not fit together: request 1 waits for request 0; request 2 (small) must
    # not overtake it
    for r in (_req(0, 60, 3, 0.0), _req(1, 50, 2, 0.0), _req(2, 10, 1, 0.0)):
        srv.submit(r)
    srv.t0 = 0.0
    done = []
    for _ in range(10):
        done += srv.step()
        clk.t += 0.1
    # admitted in arrival order (2 joined 1 once 0 had left); 2 finishes first (1 sub-step)
    assert [e for e in b.log if e[0] == "add"] == [("add", 0), ("add", 1), ("add", 2)]
    assert [r.rid for r in done] == [0, 2, 1]
    assert srv.stats.waits_for_memory >= 1
    r0, r2, r1 = done
    assert r0.steps == 3 and r1.steps == 2 and r2.steps == 1
    # each result is that scene's own state after its own sub-steps
    assert np.all(r0.pos == 3.0) and np.all(r1.pos == 2.0) and np.all(r2.pos == 1.0)
    assert r1.admitted >= r0.finished - 1e-12 and r1.wait > 0


def test_requests_join_when_they_arrive():
    clk = Clock()
    b = FakeBatch(budget=1000)
    srv = SceneServer(b, clock=clk)
    srv.submit(_req(0, 10, 5, 0.0))
    srv.submit(_req(1, 10, 2, 0.25))
    srv.t0 = 0.0
    running = []
    done = []
    for _ in range(6):
        done += srv.step()
        running.append(len(srv.running))
        clk.t += 0.1
    assert running[:3] == [1, 1, 1] and 2 in running
    assert [r.rid for r in done] == [1, 0] or [r.rid for r in done] == [0, 1]
    s = srv.stats.summary(done, 0.6)
    assert s["completed"] == 2 and s["step_latency_ms"]["p50"] == 1.0 and s["max_running"] == 2


def test_request_too_large_alone_fails():
    clk = Clock()
    srv = SceneServer(FakeBatch(budget=5), clock=clk)
    srv.submit(_req(0, 10, 1, 0.0))
    srv.t0 = 0.0
    with pytest.raises(RuntimeError):
        srv.step()
