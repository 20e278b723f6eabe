"""Online serving of fluid scenes: continuous batching over one GPU's scene batch.

The reference runs one scene per ParticleSolver object and has no serving layer
(Simulation/ParticleSolvers/ParticleSolver.h:39-105; its Simulator drives one solver on one
thread, Applications/QtApps/ParticleSimulation/Source/Simulator.cpp:38-69).  This module
keeps many requests resident on one GPU through a scene batch (bnn_batch_*, FlipBatch):

* requests arrive with an arrival time and wait in a FIFO queue;
* before every batch step the queue's head is admitted while its byte estimate
  (bnn_scene_bytes_estimate) fits the HBM budget the batch was created with; a request
  that does not fit waits (and holds the queue, so admission stays in arrival order) until
  running requests finish and free their memory;
* every batch step advances each running scene by one sub-step (scenes admitted mid-run
  join at the next step, finished ones leave at once: the batch is re-formed every step);
* a request finishes after its number of sub-steps; its particles are read back and its
  scene is released.

Each scene computes exactly what a lone FlipSolver computes (the batch steps full solver
handles), so a request's result does not depend on what else is in the batch.

The batch object is anything with FlipBatch's methods (add_scene, step, scene_info,
get_scene, remove_scene); add_scene must raise an exception whose `code` is
STATUS_CODE["CAPACITY"] when the scene does not fit the budget.
"""
from __future__ import annotations

import time
from dataclasses import dataclass, field

import numpy as np

CAPACITY = 8  # BNN_ERR_CAPACITY


@dataclass
class Request:
    """One scene to run: parameters (bnn_params keys), particles, sub-steps to take, and
    its arrival time in seconds from the start of the run."""
    rid: int
    cfg: dict
    pos: np.ndarray
    vel: np.ndarray
    steps: int
    arrival: float = 0.0


@dataclass
class Result:
    rid: int
    pos: np.ndarray
    vel: np.ndarray
    arrival: float
    admitted: float
    finished: float
    steps: int
    particles: int

    @property
    def latency(self) -> float:
        """arrival to completion, seconds"""
        return self.finished - self.arrival

    @property
    def wait(self) -> float:
        """arrival to admission, seconds"""
        return self.admitted - self.arrival


@dataclass
class ServeStats:
    step_ms: list = field(default_factory=list)       # wall time of every batch step
    particle_steps: int = 0
    batch_steps: int = 0
    admitted: int = 0
    waits_for_memory: int = 0                          # admissions refused for the budget
    max_running: int = 0
    graph_instantiations: int = 0                      # staged-step segments built into new CUDA graphs
    graph_updates: int = 0                             # ... written into the existing graphs

    def summary(self, results: list, seconds: float) -> dict:
        lat = [r.latency for r in results]
        pct = lambda a, q: float(np.percentile(a, q)) if len(a) else None  # noqa: E731
        return {"particle_steps_per_s": self.particle_steps / seconds if seconds > 0 else 0.0,
                "batch_steps": self.batch_steps, "completed": len(results), "admitted": self.admitted,
                "waits_for_memory": self.waits_for_memory, "max_running": self.max_running,
                "graph_instantiations": self.graph_instantiations, "graph_updates": self.graph_updates,
                "step_latency_ms": {"p50": pct(self.step_ms, 50), "p99": pct(self.step_ms, 99)},
                "request_latency_s": {"p50": pct(lat, 50), "p99": pct(lat, 99)},
                "queue_wait_s": {"p50": pct([r.wait for r in results], 50),
                                 "p99": pct([r.wait for r in results], 99)}}


class SceneServer:
    """Continuous batching of scene requests over one scene batch."""

    def __init__(self, batch, clock=time.perf_counter):
        self.batch = batch
        self.clock = clock
        self.t0 = clock()
        self.queue: list[Request] = []       # arrived or future requests, arrival order
        self.running: dict[int, tuple[Request, float]] = {}  # scene id -> (request, admitted at)
        self.stats = ServeStats()

    def now(self) -> float:
        return self.clock() - self.t0

    def submit(self, req: Request) -> None:
        """Queue a request (kept in arrival order)."""
        k = len(self.queue)
        while k > 0 and self.queue[k - 1].arrival > req.arrival:
            k -= 1
        self.queue.insert(k, req)

    def _admit(self) -> None:
        now = self.now()
        while self.queue and self.queue[0].arrival <= now:
            q = self.queue[0]
            try:
                sid = self.batch.add_scene(q.cfg, q.pos, q.vel)
            except Exception as e:  # noqa: BLE001 -- only the budget refusal is expected here
                if getattr(e, "code", None) != CAPACITY:
                    raise
                if not self.running:
                    raise RuntimeError(f"request {q.rid} does not fit the HBM budget even alone") from e
                self.stats.waits_for_memory += 1
                return  # wait for running requests to free memory
            self.running[sid] = (q, now)
            self.queue.pop(0)
            self.stats.admitted += 1
        self.stats.max_running = max(self.stats.max_running, len(self.running))

    def step(self) -> list[Result]:
        """Admit what fits, advance every running scene by one sub-step, retire the
        finished ones.  Returns the requests that finished in this step."""
        self._admit()
        if not self.running:
            return []
        st = self.batch.step()
        self.stats.step_ms.append(float(st["wall_ms"]))
        self.stats.particle_steps += int(st["particle_steps"])
        self.stats.batch_steps += 1
        self.stats.graph_instantiations += int(st.get("graph_instantiations", 0))
        self.stats.graph_updates += int(st.get("graph_updates", 0))
        done = []
        for sid in list(self.running):
            q, admitted = self.running[sid]
            info = self.batch.scene_info(sid)
            if info["steps"] >= q.steps:
                pos, vel = self.batch.get_scene(sid)
                self.batch.remove_scene(sid)
                del self.running[sid]
                done.append(Result(q.rid, pos, vel, q.arrival, admitted, self.now(), int(info["steps"]),
                                   int(info["n"])))
        return done

    def idle_until_next_arrival(self, cap_s: float = 0.05) -> None:
        """Nothing running: sleep until the next request arrives (at most cap_s)."""
        if self.queue and not self.running:
            time.sleep(max(0.0, min(self.queue[0].arrival - self.now(), cap_s)))

    def run(self, requests, time_limit: float = float("inf")) -> list[Result]:
        """Serve a request stream until every request finished or time_limit seconds
        passed (what finished by then is returned)."""
        for q in requests:
            self.submit(q)
        self.t0 = self.clock()
        results = []
        while self.queue or self.running:
            if self.now() > time_limit:
                break
            if not self.running:
                self._admit()
                if not self.running:
                    self.idle_until_next_arrival()
                    continue
            results.extend(self.step())
        return results
