#!/usr/bin/env python
"""Benchmark: particle-steps/s of the 3D FLIP dam break at 256^3 (12,734,496 particles,
Jacobi PCG to 1e-6 max-norm relative residual), one sub-step per step.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

One process per GPU (torchrun for N > 1).  Every rank advances its own replica of the
scene (a single scene does not shard: its pressure solve needs a global reduction every
PCG iteration), so per-GPU work is fixed and `scaling` is "weak".  The timed region is
bracketed by a barrier and a device synchronize on both sides and timed with CUDA events
on the stream the solver launches on; the job time is the max over ranks.

Other workloads (`--workload`, one JSON line each, not the headline):
  batch   256 independent dam-break scenes (seed 11, 32..128 cells per axis), refined
          FP32 PCG, one sub-step of every scene per step; scenes are split over ranks
          (`scaling` strong).  Reports step-latency p50/p99.
  serve   Poisson request stream (20/s, seed 13, cubic 32..192 cells), 200 sub-steps per
          request, 150 GB admission budget; reports request- and step-latency p50/p99.
  nsearch 4M-point cell sort + neighbour lists (r = 0.01, seed 7).
  fp64err the 256^3 scene's first `--steps` sub-steps on the GPU (FP32 PCG and refined
          PCG) against the FP64 build of the oracle: max position error / dx, max face
          velocity and pressure errors relative to their max magnitude.
  pcg     standalone Jacobi PCG (bnn_pcg_solve_7pt) on the 102 x 153 x 102 box of fluid
          cells the 256^3 dam break starts with (1,591,812 rows), a fixed number of
          iterations (`--steps`); for profiling the solver alone.
  boundary the 256^3 dam break in a box container that turns about z before every
          sub-step (a dynamic boundary object: boundary SDF and face weights recomputed,
          weighted pressure system with per-face off-diagonals, grid velocity constraint).
  aniso   anisotropic kernels (AnisotropicKernelGenerator, the "AniKernel" frame output)
          of the 256^3 dam break after one sub-step: particles/s of the kernel pass, and
          end to end through bnn_flip_anisotropic_kernels into host arrays.

`--impl reference` times the reference's CPU algorithm (the oracle port of PIC_Solver /
FLIP_Solver / PCGSolver, reference arithmetic order, OpenMP over all host cores) on the
same workload; under torchrun only rank 0 runs it.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time
from pathlib import Path

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

import numpy as np  # noqa: E402

N_GRID = 256
METRIC = "particle-steps/s at 256^3 FLIP (1e-6 rel residual)"
UNIT = "particle-steps/s"
WORKLOAD = "flip_dam_break_256"
# DRAM bytes (read + write) per PCG iteration of k_pcg_persistent at 1.59M rows, from an ncu
# capture of the standalone solve at that row count (`--workload pcg`: 835.7 MB over 300
# iterations); a launch's traffic is this times its iterations
PCG_TRAFFIC_PER_ITER = 835.7e6 / 300


PCG_MODE = {"fp32": 0, "fp64": 1, "refined": 2}
# BNN_SOLVER_*: the headline is FLIP; the others run the same scene through the same step
SOLVERS = {"flip": 0, "apic": 1, "aflip": 2, "pic": 3}


def _pcg_flags(args) -> int:
    """BNN_PCG_SINGLE_REDUCTION when the single-reduction form is asked for; the default is
    PCGSolver's step order (two reductions per iteration)"""
    return 0x10 if getattr(args, "pcg_steps", "two") == "single" else 0


def _config(pcg_mode: str, cfg: dict | None = None, pcg_text: str | None = None):
    if pcg_text is not None:
        pcg = pcg_text
    elif pcg_mode == "refined":
        pcg = (f"Jacobi, FP32 inner to {cfg['refine_inner_tolerance'] if cfg else 1e-2:g} / FP64 outer refined to "
               f"{cfg['refine_tolerance'] if cfg else 1e-8:g} max-norm rel")
    else:
        pcg = f"Jacobi, {pcg_mode}, tol {cfg['cg_relative_tolerance'] if cfg else 1e-6:g} max-norm rel"
    return {"workload": WORKLOAD, "grid": f"{N_GRID}^3 (+2 padding cells per side = {N_GRID + 4}^3 stored)",
            "particles": None, "block": [0.4, 0.6, 0.4], "particles_per_cell": 8, "seed": 42,
            "solver": "FLIP", "pic_flip_ratio": 0.97, "cfl": 1.0, "pcg": pcg,
            "step": "one advanceFrame sub-step", "l2_policy": "inputs larger than L2 (particles 306 MB, faces 212 MB)",
            "parallelism": "replicas"}


class ClockSampler:
    """SM clocks and clock-event (throttle) reasons sampled during the timed region: NVML
    every 20 ms on the GPU this process computes on (matched by UUID), else nvidia-smi
    every 200 ms.  Read-only: nothing here changes a GPU setting."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
    # NVML clock-event reason bits (nvmlClocksEventReason*)
    REASON_BITS = {"sw_power_cap": 0x4, "hw_slowdown": 0x8, "sw_thermal_slowdown": 0x20,
                   "hw_thermal_slowdown": 0x40, "hw_power_brake_slowdown": 0x80}

    def __init__(self, gpu: int):
        self.gpu = gpu
        self.f = None
        self.p = None
        self.nvml = None
        self.samples = []
        self.stop_evt = None
        self.thread = None

    def _nvml_handle(self):
        import pynvml
        import torch
        pynvml.nvmlInit()
        try:
            uuid = str(torch.cuda.get_device_properties(self.gpu).uuid)
            return pynvml, pynvml.nvmlDeviceGetHandleByUUID(uuid if uuid.startswith("GPU-") else "GPU-" + uuid)
        except Exception:
            return pynvml, pynvml.nvmlDeviceGetHandleByIndex(self.gpu)

    def start(self):
        try:
            import threading
            nv, h = self._nvml_handle()
            reasons = getattr(nv, "nvmlDeviceGetCurrentClocksEventReasons", None) or \
                nv.nvmlDeviceGetCurrentClocksThrottleReasons
            mx = nv.nvmlDeviceGetMaxClockInfo(h, nv.NVML_CLOCK_SM)
            self.nvml = nv
            self.stop_evt = threading.Event()

            def run():
                while not self.stop_evt.is_set():
                    try:
                        self.samples.append((nv.nvmlDeviceGetClockInfo(h, nv.NVML_CLOCK_SM), mx, int(reasons(h))))
                    except Exception:
                        pass
                    self.stop_evt.wait(0.02)

            self.thread = threading.Thread(target=run, daemon=True)
            self.thread.start()
            return
        except Exception:
            self.nvml = None
        try:
            self.f = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
            self.p = subprocess.Popen(["nvidia-smi", "-i", str(self.gpu), f"--query-gpu={self.FIELDS}",
                                       "--format=csv,noheader,nounits", "-lms", "200"], stdout=self.f,
                                      stderr=subprocess.DEVNULL)
        except Exception:
            self.p = None

    def stop(self) -> dict:
        if self.nvml is not None:
            self.stop_evt.set()
            self.thread.join(timeout=5)
            sm = [float(c) for c, _, _ in self.samples]
            mx = [float(m) for _, m, _ in self.samples]
            reasons = {name for _, _, bits in self.samples for name, b in self.REASON_BITS.items() if bits & b}
            return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                    "reasons": sorted(reasons), "samples": len(sm), "source": "nvml, 20 ms"}
        if self.p is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.p.terminate()
        try:
            self.p.wait(timeout=5)
        except Exception:
            self.p.kill()
        self.f.flush()
        rows = [r.split(",") for r in Path(self.f.name).read_text().strip().splitlines() if r.strip()]
        sm, mx, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for r in rows:
            r = [x.strip() for x in r]
            try:
                sm.append(float(r[1]))
                mx.append(float(r[2]))
            except Exception:
                continue
            for k, name in enumerate(names):
                if len(r) > 5 + k and r[5 + k].lower().startswith("active"):
                    reasons.add(name)
        os.unlink(self.f.name)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": sorted(reasons), "samples": len(sm), "source": "nvidia-smi, 200 ms"}


def _peaks():
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        d = json.loads(p.read_text())
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def stage_bytes(npart: int, G: int, rows: float, iters: float) -> dict:
    """Algorithmic bytes of one sub-step's stages (each array touched once per stage, FP32):
    Np particles, C = G^3 cells, F = 3 (G+1) G^2 faces, A active rows, K PCG iterations.
    The G2P and the next move share one entry (the particle pass: grid-to-particle blend,
    RK2 advection, box projection), and so do P2G and the fluid SDF (one tiled pass over
    the particles); extrapolation counts 10 F per call (4 layers fused), the first call
    with the 4 F backup of the FLIP old velocities."""
    C = float(G) ** 3
    F = 3.0 * (G + 1) * float(G) ** 2
    Np, A = float(npart), float(rows)
    return {"sort": 72.0 * Np + 12.0 * C, "p2g+fluid_sdf": (24.0 * Np + 5.0 * F) + (12.0 * Np + 4.0 * C),
            "extrapolate": 10.0 * F + 4.0 * F, "system": 8.0 * C + 28.0 * A, "pcg": 52.0 * A * iters,
            "update": 9.0 * F + 4.0 * A + 10.0 * F, "move+g2p": 48.0 * Np + 8.0 * F}


def _stage_gbs(npart, G, stats, stage_tot):
    """Achieved GB/s of each stage: its algorithmic bytes (stage_bytes, with the measured
    rows and PCG iterations of every step) over its CUDA-event time."""
    tot = {}
    for s in stats:
        for k, b in stage_bytes(npart, G, s["n_active"], s["pcg_iterations"]).items():
            tot[k] = tot.get(k, 0.0) + b
    ms = dict(stage_tot)
    ms["move+g2p"] = stage_tot["move"] + stage_tot["g2p"]
    ms["p2g+fluid_sdf"] = stage_tot["p2g"] + stage_tot["fluid_sdf"]
    return {k: (tot[k] / (ms[k] * 1e-3) / 1e9 if ms.get(k, 0) > 0 else None) for k in tot}


def _dist():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return ws, rank, local


def cpu_port_steps(n_grid: int, steps: int, skip: int, threads: int):
    """Oracle port (reference order, OpenMP) on the same scene: time `steps` sub-steps after
    `skip` untimed ones.  Returns (particle-steps/s, particles, seconds)."""
    from banana_b200 import scenes
    from oracle import oracle as O
    O.set_threads(threads)
    pos, vel = scenes.dam_break(n_grid)
    cfg = scenes.dam_break_params(n_grid, reduce_mode=0, nthreads=threads, sort_each_step=0)
    o = O.Oracle(cfg)
    o.set_particles(pos, vel)
    for _ in range(skip):
        o.step()
    t0 = time.perf_counter()
    for _ in range(steps):
        o.step()
    dt = time.perf_counter() - t0
    o.close()
    return len(pos) * steps / dt, len(pos), dt


def run_reference(args, ws, rank):
    if rank != 0:
        return 0
    threads = os.cpu_count() or 1
    # full-size sub-steps of the same scene; when one step is slow the timed count shrinks
    # so the whole run stays within a few minutes (the line reports what was timed)
    from banana_b200 import scenes
    from oracle import oracle as O
    O.set_threads(threads)
    pos, vel = scenes.dam_break(N_GRID)
    precond = {"jacobi": 0, "ic0": 2}[args.ref_precond]
    cfg = scenes.dam_break_params(N_GRID, reduce_mode=0, nthreads=threads, sort_each_step=0, preconditioner=precond)
    o = O.Oracle(cfg)
    o.set_particles(pos, vel)
    t_w = time.perf_counter()
    w_done = 0
    for _ in range(args.warmup):
        o.step()
        w_done += 1
        if time.perf_counter() - t_w > 60:
            break
    per = (time.perf_counter() - t_w) / max(w_done, 1)
    steps = args.steps
    if per * steps > 150:
        steps = max(1, int(150 / max(per, 1e-9)))
    t0 = time.perf_counter()
    iters = []
    for _ in range(steps):
        st = o.step()
        iters.append(st["pcg_iterations"])
    dt = time.perf_counter() - t0
    o.close()
    value = len(pos) * steps / dt
    line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": ws, "steps": steps, "warmup": w_done,
            "ms_per_step": dt * 1e3 / steps, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f32", "data": "synthetic (seeded dam break, seed 42)", "impl": "reference",
            "config": dict(_config("fp32", cfg) if not precond else
                           _config("fp32", pcg_text="symmetric MIC(0) preconditioner (the reference default), "
                                                    f"fp32, tol {cfg['cg_relative_tolerance']:g} max-norm rel"),
                           particles=len(pos)),
            "arithmetic": "reference order: FP32 accumulators, serial left-to-right reductions per thread",
            "cpu_baseline": {"value": value, "unit": UNIT, "cores": threads, "kind": "port",
                             "sample": f"{steps} full sub-steps of the {N_GRID}^3 scene after {w_done} untimed "
                                       f"(oracle port of the reference CPU solver, OpenMP, {threads} threads)"},
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
            "pcg_iterations_mean": float(np.mean(iters))}
    print(json.dumps(line), flush=True)
    return 0


def run_ours(args, ws, rank, local):
    import torch
    import torch.distributed as dist

    from banana_b200 import FlipSolver, capi, scenes

    torch.cuda.set_device(local)
    if ws > 1:
        dist.init_process_group("nccl", device_id=torch.device("cuda", local),
                                timeout=__import__("datetime").timedelta(seconds=120))

    def barrier():
        if ws > 1:
            dist.barrier()

    pcg_mode = args.pcg_mode
    cfg = scenes.dam_break_params(N_GRID, pcg_mode={"fp32": 0, "fp64": 1, "refined": 2}[pcg_mode] | _pcg_flags(args))
    if args.inner_tol is not None:
        cfg["refine_inner_tolerance"] = args.inner_tol
    if args.tol is not None:
        cfg["cg_relative_tolerance"] = args.tol
    cfg["solver_kind"] = SOLVERS[args.solver]
    pos, vel = scenes.dam_break(N_GRID)
    npart = len(pos)
    if args.tile_shape is not None:
        capi.set_tile_shape(args.tile_shape)
    solver = FlipSolver(cfg)
    solver.set_particles(pos, vel)
    stream = torch.cuda.ExternalStream(solver.stream_ptr())
    for _ in range(args.warmup):
        solver.step()

    clocks = ClockSampler(local)
    clocks.start()
    barrier()
    torch.cuda.synchronize()
    launches0 = capi.launch_count()
    ev0 = torch.cuda.Event(enable_timing=True)
    ev1 = torch.cuda.Event(enable_timing=True)
    ev0.record(stream)
    stats = []
    for _ in range(args.steps):
        stats.append(solver.step())
    ev1.record(stream)
    torch.cuda.synchronize()
    barrier()
    clk = clocks.stop()
    launches = capi.launch_count() - launches0
    ms = ev0.elapsed_time(ev1)
    t_max = ms
    if ws > 1:
        t = torch.tensor([ms], device="cuda", dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        t_max = float(t.item())
    value = npart * ws * args.steps / (t_max * 1e-3)

    # stage breakdown and roofline of the PCG iteration (spmv + update kernels)
    stage_tot = {k: sum(s["stage_ms"][k] for s in stats) for k in capi.STAGES}
    iters = sum(s["pcg_iterations"] for s in stats)
    rows = [s["n_active"] for s in stats]
    pcg_bytes = sum(52.0 * s["n_active"] * s["pcg_iterations"] for s in stats)
    peak, peak_kind = _peaks()
    # the persistent launch alone (CUDA events around it on the solver's stream); the pcg
    # stage also holds the row packing and the host's read of the solve's outcome
    pcg_kernel_ms = sum(s["pcg_kernel_ms"] for s in stats)
    pcg_ms = pcg_kernel_ms if pcg_kernel_ms > 0 else stage_tot["pcg"]
    achieved = pcg_bytes / (pcg_ms * 1e-3) / 1e9 if pcg_ms > 0 else 0.0
    stage_gbs = _stage_gbs(npart, N_GRID + 4, stats, stage_tot)

    # end to end: host arrays in pinned memory, H2D + step + D2H per step
    e2e = None
    if not args.skip_e2e:
        hp = torch.empty((npart, 3), dtype=torch.float32, pin_memory=True)
        hv = torch.empty((npart, 3), dtype=torch.float32, pin_memory=True)
        p_np, v_np = solver.get_particles()
        hp.numpy()[:] = p_np
        hv.numpy()[:] = v_np
        barrier()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        for _ in range(args.steps):
            solver.step_host_ptr(hp.data_ptr(), hv.data_ptr())
        torch.cuda.synchronize()
        te = time.perf_counter() - t0
        if ws > 1:
            t = torch.tensor([te], device="cuda", dtype=torch.float64)
            dist.all_reduce(t, op=dist.ReduceOp.MAX)
            te = float(t.item())
        e2e = {"value": npart * ws * args.steps / te, "unit": UNIT, "h2d_bytes_per_step": 24 * npart,
               "d2h_bytes_per_step": 24 * npart,
               "api": "bnn_flip_step_host (pinned host AoS positions/velocities in and out every step), wall clock"}

    cpu = None
    if rank == 0 and ws == 1 and not args.no_cpu_baseline:
        threads = os.cpu_count() or 1
        v, n, sec = cpu_port_steps(N_GRID, steps=2, skip=1, threads=threads)
        cpu = {"value": v, "unit": UNIT, "cores": threads, "kind": "port",
               "sample": f"sub-steps 2-3 of the same {N_GRID}^3 scene ({n} particles), oracle port of the reference CPU "
                         f"solver in reference arithmetic order, OpenMP {threads} threads, {sec:.1f} s"}

    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": ws, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": t_max / args.steps, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f32", "data": "synthetic (seeded dam break, seed 42)",
            "config": dict(_config(pcg_mode, cfg), particles=npart, solver=args.solver.upper(),
                           workload=WORKLOAD if args.solver == "flip" else f"{args.solver}_dam_break_256"),
            "roofline": {"bound": "hbm", "kernel": "k_pcg_persistent (whole Jacobi PCG solve, one launch per step)",
                         "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak, "peak_kind": peak_kind,
                         "algorithmic_bytes": "52 B per active row per PCG iteration (x, r, z, s, q, 1/diag and "
                                              "the row's matrix data once each)",
                         "traffic": PCG_TRAFFIC_PER_ITER * iters / args.steps,
                         "traffic_note": "ncu DRAM bytes per iteration of the same kernel at the same row count "
                                         "(standalone capture) x iterations per launch; the solve is L2-resident"},
            "cpu_baseline": cpu, "e2e": e2e, "gpu_launches": int(launches),
            "clocks": clk,
            "detail": {"tile_tuning": capi.tile_tuning(),
                       "pcg_iterations_per_step": iters / args.steps, "active_rows_mean": float(np.mean(rows)),
                       "pcg_kernel_ms_per_step": pcg_kernel_ms / args.steps,
                       "stage_ms_per_step": {k: v / args.steps for k, v in stage_tot.items()},
                       "stage_gbs": stage_gbs},
        }
        if ws == 1 and N_GRID == 256 and not args.no_extras:
            solver.close()
            line["detail"]["more_workloads"] = _more_workloads()
        if args.per_step:
            # every timed sub-step (numbered from 1 over the whole run, warm-up included)
            line["detail"]["per_step"] = [
                {"step": args.warmup + i + 1, "dt": s["dt"], "pcg_iterations": s["pcg_iterations"],
                 "n_active": s["n_active"], "stage_ms": {k: round(v, 4) for k, v in s["stage_ms"].items()}}
                for i, s in enumerate(stats)]
        print(json.dumps(line), flush=True)
    solver.close()
    if ws > 1:
        dist.destroy_process_group()
    return 0


def _torch_dist(ws, local):
    import torch
    import torch.distributed as dist
    torch.cuda.set_device(local)
    if ws > 1:
        dist.init_process_group("nccl", device_id=torch.device("cuda", local),
                                timeout=__import__("datetime").timedelta(seconds=300))
    return torch, dist


def run_batch(args, ws, rank, local):
    """256 independent scenes on the GPU(s), one sub-step of each per step."""
    torch, dist = _torch_dist(ws, local)
    from banana_b200 import FlipBatch, capi, dist as bdist, scenes

    if args.tile_shape is not None:
        capi.set_tile_shape(args.tile_shape)
    specs = scenes.batch_scene_specs()
    costs = []
    for s in specs:
        cells = [int(np.floor(f * r + 1e-9)) for f, r in zip(s["block_frac"], s["res"])]
        costs.append(bdist.scene_bytes_per_step(s["res"], 8 * cells[0] * cells[1] * cells[2]))
    mine = bdist.shard_scenes(costs, ws)[rank]
    mode = capi.BATCH_PER_SCENE if args.batch_mode == "per_scene" else capi.BATCH_STAGED
    b = FlipBatch(worker_threads=args.workers, step_mode=mode)
    over = {} if args.inner_tol is None else {"refine_inner_tolerance": args.inner_tol}
    built = [scenes.batch_scene(specs[i], **over) for i in mine]
    npart = sum(len(p) for _, p, _ in built)
    t_up = time.perf_counter()
    ids, add_ms = [], []
    for cfg, pos, vel in built:
        ta = time.perf_counter()
        ids.append(b.add_scene(cfg, pos, vel))
        add_ms.append((time.perf_counter() - ta) * 1e3)
    t_up = time.perf_counter() - t_up
    for _ in range(args.warmup):
        b.step()
    clocks = ClockSampler(local)
    clocks.start()
    if ws > 1:
        dist.barrier()
    torch.cuda.synchronize()
    launches0 = capi.launch_count()
    lat, ps, iters, staged = [], 0, 0, 0
    stage_ms = {k: 0.0 for k in capi.STAGES}
    t0 = time.perf_counter()
    for _ in range(args.steps):
        st = b.step()
        lat.append(st["wall_ms"])
        ps += st["particle_steps"]
        iters += st["pcg_iterations"]
        staged = max(staged, st["staged_scenes"])
        for k, v in b.scene_info(ids[0])["stage_ms"].items():
            stage_ms[k] += v
    torch.cuda.synchronize()
    te = time.perf_counter() - t0
    t_dl = time.perf_counter()
    for sid in ids:
        b.get_scene(sid)
    t_dl = time.perf_counter() - t_dl
    clk = clocks.stop()
    launches = capi.launch_count() - launches0
    b.close()
    # the same scenes one at a time (one worker thread, no staged step: each scene's
    # sub-step runs alone on the GPU before the next one starts), and each on its own
    # stream from the worker pool, for the batching's gain
    def other_mode(workers, step_mode, n_steps=2):
        bo = FlipBatch(worker_threads=workers, step_mode=step_mode)
        for cfg, pos, vel in built:
            bo.add_scene(cfg, pos, vel)
        bo.step()
        torch.cuda.synchronize()
        t = time.perf_counter()
        pso = 0
        for _ in range(n_steps):
            pso += bo.step()["particle_steps"]
        torch.cuda.synchronize()
        t = time.perf_counter() - t
        bo.close()
        return pso / t, t * 1e3 / n_steps
    if args.no_compare:
        seq_value = seq_ms = pool_value = pool_ms = None
    else:
        seq_value, seq_ms = other_mode(1, capi.BATCH_PER_SCENE)
        pool_value, pool_ms = (other_mode(args.workers, capi.BATCH_PER_SCENE) if mode == capi.BATCH_STAGED
                               else (ps / te, te * 1e3 / args.steps))
    tot_ps = ps
    t_max = te
    e2e_t = te + t_up + t_dl
    if ws > 1:
        v = torch.tensor([ps], dtype=torch.float64, device="cuda")
        dist.all_reduce(v)
        tot_ps = float(v.item())
        t = torch.tensor([te, e2e_t], dtype=torch.float64, device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        t_max, e2e_t = (float(x) for x in t.tolist())
    if rank == 0:
        line = {"metric": "particle-steps/s, 256 batched dam-break scenes", "value": tot_ps / t_max,
                "unit": UNIT, "n_gpus": ws, "steps": args.steps, "warmup": args.warmup,
                "ms_per_step": t_max * 1e3 / args.steps, "higher_is_better": True, "scaling": "strong",
                "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded scenes, seed 11)",
                "config": {"workload": "batch_256_scenes", "scenes": len(specs), "scenes_rank0": len(mine),
                           "particles_rank0": npart, "res_choices": [32, 48, 64, 96, 128], "cell_size": "1/64",
                           "pcg": "Jacobi, refined FP32 inner / FP64 outer to 1e-6, inner "
                                  f"{args.inner_tol if args.inner_tol is not None else 1e-3:g}",
                           "batch_mode": args.batch_mode, "staged_scenes_rank0": staged,
                           "worker_threads": args.workers or "min(16, cores)", "parallelism": f"scenes/{ws} ranks"},
                "latency_ms": {"p50": float(np.percentile(lat, 50)), "p99": float(np.percentile(lat, 99))},
                "e2e": {"value": tot_ps / e2e_t, "unit": UNIT, "h2d_bytes_per_step": 24 * npart / args.steps,
                        "d2h_bytes_per_step": 24 * npart / args.steps,
                        "api": "bnn_batch_add_scene (upload) + steps + bnn_batch_get_scene (download), wall clock",
                        "upload_s": t_up, "download_s": t_dl,
                        "add_scene_ms": {"p50": float(np.median(add_ms)), "max": float(np.max(add_ms)),
                                         "first": add_ms[0]}},
                "gpu_launches": int(launches), "clocks": clk,
                "detail": {"tile_tuning": capi.tile_tuning(),
                           "pcg_iterations_per_step": iters / args.steps, "timing": "host wall clock per batch step",
                           "stage_ms_per_step": {k: round(v / args.steps, 3) for k, v in stage_ms.items()},
                           "stage_ms_note": "device time per stage of the staged step (scene 0's record; all "
                                            "staged scenes share it), or scene 0's own stream in per_scene mode",
                           "one_scene_at_a_time": {"value": seq_value, "ms_per_step": seq_ms,
                                                   "note": "rank 0's scenes, one worker thread, same accuracy"},
                           "per_scene_streams": {"value": pool_value, "ms_per_step": pool_ms,
                                                 "note": "rank 0's scenes, each on its own stream from the worker pool"},
                           "batched_over_one_at_a_time": (ps / te) / seq_value if seq_value else None}}
        print(json.dumps(line), flush=True)
    if ws > 1:
        dist.destroy_process_group()
    return 0


def run_serve(args, ws, rank, local):
    """Poisson request stream: each request is a scene that runs 200 sub-steps, served by
    banana_b200.serving.SceneServer (admission against the HBM budget, continuous
    batching)."""
    torch, dist = _torch_dist(ws, local)
    from banana_b200 import FlipBatch, capi, scenes
    from banana_b200.serving import Request, SceneServer
    if args.tile_shape is not None:
        capi.set_tile_shape(args.tile_shape)

    reqs = scenes.serve_requests(args.requests)
    mine = [(k, q) for k, q in enumerate(reqs) if k % ws == rank]
    budget = int(150e9)
    b = FlipBatch(hbm_budget_bytes=budget, worker_threads=args.workers)
    server = SceneServer(b)
    stream = []
    for k, q in mine:
        cfg, pos, vel = scenes.batch_scene(q)
        stream.append(Request(k, cfg, pos, vel, args.req_steps, q["t"]))
    launches0 = capi.launch_count()
    clocks = ClockSampler(local)
    clocks.start()
    t0 = time.perf_counter()
    results = server.run(stream, time_limit=args.time_limit)
    te = time.perf_counter() - t0
    clk = clocks.stop()
    launches = capi.launch_count() - launches0
    summ = server.stats.summary(results, te)
    tot = server.stats.particle_steps
    if ws > 1:
        v = torch.tensor([tot], dtype=torch.float64, device="cuda")
        dist.all_reduce(v)
        tot = float(v.item())
        t = torch.tensor([te], dtype=torch.float64, device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        te = float(t.item())
    if rank == 0:
        line = {"metric": "served particle-steps/s, Poisson dam-break requests", "value": tot / te, "unit": UNIT,
                "n_gpus": ws, "steps": summ["batch_steps"], "warmup": 0,
                "ms_per_step": float(np.mean(server.stats.step_ms)) if server.stats.step_ms else None,
                "higher_is_better": True, "scaling": "strong", "vs_baseline": None, "dtype": "f32",
                "data": "synthetic (seeded request stream, seed 13)",
                "config": {"workload": "serve_poisson", "requests": len(reqs), "rate_per_s": 20,
                           "res": "cubic, log-uniform 32..192", "steps_per_request": args.req_steps,
                           "hbm_budget_gb": 150, "pcg": "refined FP32 (inner 1e-3) to 1e-6", "parallelism": f"requests/{ws} ranks",
                           "time_limit_s": args.time_limit},
                "completed_requests": summ["completed"], "admitted_requests": summ["admitted"],
                "waits_for_memory": summ["waits_for_memory"], "max_running": summ["max_running"],
                "graphs": {"instantiated": summ["graph_instantiations"], "updated": summ["graph_updates"]},
                "tile_shapes_tuned": len(capi.tile_tuning()),
                "request_latency_s": summ["request_latency_s"], "queue_wait_s": summ["queue_wait_s"],
                "step_latency_ms": summ["step_latency_ms"], "seconds": te,
                "gpu_launches": int(launches), "clocks": clk}
        print(json.dumps(line), flush=True)
    b.close()
    if ws > 1:
        dist.destroy_process_group()
    return 0


def run_nsearch(args, ws, rank, local):
    """4M points: cell sort (bit-exact ids + sorted index) and CSR neighbour lists."""
    import ctypes as C

    torch, dist = _torch_dist(ws, local)
    from banana_b200 import capi, scenes

    L = capi.load()
    pts = scenes.point_cloud(4_000_000, seed=7)
    n = len(pts)
    r = np.float32(0.01)
    dev = torch.from_numpy(pts).cuda()
    cid = torch.empty(n, dtype=torch.int32, device="cuda")
    srt = torch.empty(n, dtype=torch.int32, device="cuda")
    nc = (C.c_int32 * 3)(100, 100, 100)
    bmin = (C.c_float * 3)(0.0, 0.0, 0.0)
    oor = C.c_uint32()
    off = torch.empty(n + 1, dtype=torch.int64, device="cuda")
    total = C.c_uint64()
    cap = 1_200_000_000
    idx = torch.empty(cap, dtype=torch.int32, device="cuda")
    s = torch.cuda.current_stream()
    sp = C.c_void_p(s.cuda_stream)

    def once():
        capi.check(L.bnn_cell_sort(C.c_void_p(dev.data_ptr()), n, bmin, C.c_float(0.01), nc, C.c_void_p(cid.data_ptr()),
                                   C.c_void_p(srt.data_ptr()), None, C.byref(oor), sp), "bnn_cell_sort")
        capi.check(L.bnn_neighbors(C.c_void_p(dev.data_ptr()), n, C.c_float(r), C.c_void_p(off.data_ptr()),
                                   C.c_void_p(idx.data_ptr()), cap, C.byref(total), sp), "bnn_neighbors")

    for _ in range(args.warmup):
        once()
    torch.cuda.synchronize()
    launches0 = capi.launch_count()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(s)
    for _ in range(args.steps):
        once()
    e1.record(s)
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1) / args.steps
    launches = capi.launch_count() - launches0
    if rank == 0:
        line = {"metric": "points/s, 4M-point cell sort + neighbour lists (r = 0.01)", "value": n / (ms * 1e-3),
                "unit": "points/s", "n_gpus": 1, "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms,
                "higher_is_better": True, "scaling": "replicas", "vs_baseline": None, "dtype": "f32",
                "data": "synthetic (2M uniform + 2M in 16 Gaussians, sigma 0.03, seed 7)",
                "config": {"workload": "nsearch_4m", "points": n, "radius": 0.01, "grid": "100^3"},
                "neighbour_entries": int(total.value),
                "entries_per_s": int(total.value) / (ms * 1e-3), "gpu_launches": int(launches)}
        print(json.dumps(line), flush=True)
    if ws > 1:
        dist.destroy_process_group()
    return 0


def run_aniso(args, ws, rank, local):
    """Anisotropic kernels of the dam break's particles (reference defaults: kernel radius
    8 particle radii = 4 cells, threshold 25 neighbours)."""
    torch, dist = _torch_dist(ws, local)
    from banana_b200 import capi, scenes

    cfg = scenes.dam_break_params(N_GRID)
    pos, vel = scenes.dam_break(N_GRID)
    g = capi.FlipSolver(cfg)
    g.set_particles(pos, vel)
    g.step()
    n = len(pos)
    for _ in range(args.warmup):
        g.anisotropic_kernels()
    launches0 = capi.launch_count()
    kernel_ms, wall = [], []
    st = None
    for _ in range(args.steps):
        t0 = time.perf_counter()
        _, _, st = g.anisotropic_kernels()
        wall.append((time.perf_counter() - t0) * 1e3)
        kernel_ms.append(st["ms"])
    launches = capi.launch_count() - launches0
    cpu = None
    if rank == 0 and not args.no_cpu_baseline:
        from oracle import oracle as O
        threads = os.cpu_count() or 1
        O.set_threads(threads)
        small = 64
        sp, _ = scenes.dam_break(small)
        sc = scenes.dam_break_params(small)
        o = capi.FlipSolver(sc)
        o.set_particles(sp, np.zeros_like(sp))
        _, _, sst = o.anisotropic_kernels()
        o.close()
        t0 = time.perf_counter()
        O.aniso_kernels(sp, sst["grid_bmin"], np.float32(sst["grid_cell_size"]), sst["grid_dims"],
                        np.float32(sc["cell_size"] / 2.0))
        dt = time.perf_counter() - t0
        cpu = {"value": len(sp) / dt, "unit": "particles/s", "cores": threads, "kind": "port",
               "sample": f"the oracle over all {len(sp)} particles of the {small}^3 dam break"}
    ms = statistics.median(kernel_ms)
    if rank == 0:
        line = {"metric": f"particles/s, anisotropic kernels of the {N_GRID}^3 dam break", "value": n / (ms * 1e-3),
                "unit": "particles/s", "n_gpus": 1, "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms,
                "higher_is_better": True, "scaling": "replicas", "vs_baseline": None, "dtype": "f32",
                "data": "synthetic (seeded dam break after one sub-step)",
                "config": {"workload": f"aniso_dam_break_{N_GRID}", "particles": n, "kernel_ratio": 8,
                           "particle_radius": "cell / 2", "neighbor_threshold": 25},
                "sprays": st["sprays"],
                "e2e": {"value": n / (statistics.median(wall) * 1e-3), "unit": "particles/s",
                        "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 48 * n,
                        "note": "bnn_flip_anisotropic_kernels: re-sort, kernel pass, centres and matrices to host"},
                "cpu_baseline": cpu, "gpu_launches": int(launches)}
        print(json.dumps(line), flush=True)
    g.close()
    if ws > 1:
        dist.destroy_process_group()
    return 0


def run_boundary(args, ws, rank, local):
    """Dam break with a dynamic boundary object: a box container of half-size 0.55 about the
    domain's centre turns about z by 0.2 degrees before every sub-step (update_grid each
    time, in the timed region, as the reference recomputes the boundary SDF whenever a
    dynamic object moved).  It cuts the domain's vertical edges, so the boundary SDF, the
    face weights below 1 and the solid part of the fluid SDF all take part; the fluid starts
    inside it."""
    torch, dist = _torch_dist(ws, local)
    from banana_b200 import capi, scenes

    cfg = scenes.dam_break_params(N_GRID)
    pos, vel = scenes.dam_break(N_GRID)
    n = len(pos)
    g = capi.FlipSolver(cfg)
    g.set_particles(pos, vel)
    stream = torch.cuda.ExternalStream(g.stream_ptr())

    def box(k):
        return capi.boundary_object("box", (-0.55, -0.55, -0.55), (0.55, 0.55, 0.55), translation=(0.5, 0.5, 0.5),
                                    axis_angle=(0.0, 0.0, 1.0, np.radians(0.2 * k)), dynamic=True)

    k = 0
    for _ in range(args.warmup):
        g.set_boundaries([box(k)])
        g.step()
        k += 1
    torch.cuda.synchronize()
    launches0 = capi.launch_count()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    stats = []
    for _ in range(args.steps):
        g.set_boundaries([box(k)])
        stats.append(g.step())
        k += 1
    e1.record(stream)
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1) / args.steps
    launches = capi.launch_count() - launches0
    if rank == 0:
        pk = sum(s["pcg_kernel_ms"] for s in stats) / args.steps
        it = sum(s["pcg_iterations"] for s in stats) / args.steps
        rows = float(np.mean([s["n_active"] for s in stats]))
        line = {"metric": f"particle-steps/s at {N_GRID}^3 FLIP with a turning box container", "value": n / (ms * 1e-3),
                "unit": "particle-steps/s", "n_gpus": 1, "steps": args.steps, "warmup": args.warmup,
                "ms_per_step": ms, "higher_is_better": True, "scaling": "replicas", "vs_baseline": None,
                "dtype": "f32", "data": "synthetic (seeded dam break, seed 42)",
                "config": {"workload": f"boundary_dam_break_{N_GRID}", "particles": n,
                           "boundary": "box container of half-size 0.55 about (0.5, 0.5, 0.5) turning 0.2 deg "
                                       "about z per sub-step"},
                "detail": {"pcg_iterations_per_step": it, "active_rows_mean": rows, "pcg_kernel_ms_per_step": pk,
                           "pcg_us_per_iteration": 1e3 * pk / it if it else None,
                           "stage_ms_per_step": {key: sum(s["stage_ms"][key] for s in stats) / args.steps
                                                 for key in capi.STAGES}},
                "gpu_launches": int(launches)}
        print(json.dumps(line), flush=True)
    g.close()
    if ws > 1:
        dist.destroy_process_group()
    return 0


def _box_system(nx, ny, nz, seed=1):
    """7-point system on a full box of cells in cell order (the layout of a grid)."""
    n = nx * ny * nz
    dt = np.float32(1.0 / 30)
    i = np.arange(n)
    x, y, z = i % nx, (i // nx) % ny, i // (nx * ny)
    nbr = -np.ones((n, 6), np.int32)
    nbr[:, 0] = np.where(z > 0, i - nx * ny, -1)
    nbr[:, 1] = np.where(y > 0, i - nx, -1)
    nbr[:, 2] = np.where(x > 0, i - 1, -1)
    nbr[:, 3] = np.where(x < nx - 1, i + 1, -1)
    nbr[:, 4] = np.where(y < ny - 1, i + nx, -1)
    nbr[:, 5] = np.where(z < nz - 1, i + nx * ny, -1)
    cnt = (nbr >= 0).sum(1)
    diag = (cnt * dt + (6 - cnt) * dt / np.float32(0.5)).astype(np.float32)
    rhs = (np.random.default_rng(seed).standard_normal(n) * 1e-3).astype(np.float32)
    return diag, nbr, -dt, rhs


def _more_workloads() -> dict:
    """The other configurations' headline numbers, measured in the same run (each workload in
    its own process, after the headline solver has released its memory): the 256-scene
    batch (config 4), the served Poisson stream (config 5), and the 256^3 step with FP64 PCG
    and with refined FP32 PCG, both to 1e-8 (config 2's two precision runs)."""
    import subprocess
    runs = {
        "batch_256_scenes": ["--workload", "batch", "--steps", "10", "--warmup", "3"],
        "serve_poisson": ["--workload", "serve", "--workers", "8"],
        "fp64_pcg_to_1e-8": ["--pcg-mode", "fp64", "--tol", "1e-8", "--steps", "10", "--warmup", "5",
                             "--no-cpu-baseline", "--skip-e2e", "--no-extras"],
        "refined_pcg_to_1e-8": ["--pcg-mode", "refined", "--steps", "10", "--warmup", "5", "--no-cpu-baseline",
                                "--skip-e2e", "--no-extras"],
    }
    keep = ("metric", "value", "unit", "ms_per_step", "steps", "warmup", "latency_ms", "step_latency_ms",
            "request_latency_s", "queue_wait_s", "completed_requests", "gpu_launches", "clocks", "seconds")
    out = {"note": "each measured by this bench.py run in a child process (same box, after the headline)"}
    for name, extra in runs.items():
        try:
            r = subprocess.run([sys.executable, os.path.abspath(__file__), *extra], capture_output=True, text=True,
                               timeout=600, env=dict(os.environ))
            lines = [json.loads(l) for l in r.stdout.splitlines() if l.startswith("{")]
            if r.returncode != 0 or not lines:
                out[name] = {"error": f"exit {r.returncode}: {r.stderr.strip()[-300:]}"}
                continue
            d = lines[-1]
            rec = {k: d[k] for k in keep if k in d}
            rec["config"] = {k: v for k, v in d.get("config", {}).items() if k in ("workload", "pcg", "scenes", "requests",
                                                                                  "particles_rank0", "particles")}
            if d.get("e2e"):
                rec["e2e"] = {k: d["e2e"].get(k) for k in ("value", "api", "upload_s", "download_s", "add_scene_ms")
                              if k in d["e2e"]}
            det = d.get("detail", {})
            for k in ("per_scene_streams", "one_scene_at_a_time", "pcg_iterations_per_step", "stage_ms_per_step"):
                if k in det:
                    rec[k] = det[k]
            out[name] = rec
        except Exception as e:  # noqa: BLE001 -- a failing extra must not take the headline line with it
            out[name] = {"error": repr(e)[:300]}
    return out


def run_pcg(args, ws, rank, local):
    torch, dist = _torch_dist(ws, local)
    from banana_b200 import capi, pcg_solve_7pt

    diag, nbr, off, rhs = _box_system(102, 153, 102)
    n = len(rhs)
    for _ in range(args.warmup):
        pcg_solve_7pt(diag, nbr, off, rhs, 1e-30, args.steps, mode=PCG_MODE[args.pcg_mode] | _pcg_flags(args))
    launches0 = capi.launch_count()
    _, st = pcg_solve_7pt(diag, nbr, off, rhs, 1e-30, args.steps, mode=PCG_MODE[args.pcg_mode] | _pcg_flags(args))
    launches = capi.launch_count() - launches0
    it = max(st["iterations"], 1)
    us = 1e3 * st["ms"] / it
    peak, peak_kind = _peaks()
    achieved = 52.0 * n / (us * 1e-6) / 1e9
    if rank == 0:
        line = {"metric": "us per PCG iteration, 1,591,812-row 7-point system", "value": us, "unit": "us/iteration",
                "n_gpus": 1, "steps": it, "warmup": args.warmup, "ms_per_step": st["ms"], "higher_is_better": False,
                "scaling": "replicas", "vs_baseline": None, "dtype": args.pcg_mode,
                "data": "synthetic (box of fluid cells, random rhs, seed 1)",
                "config": {"workload": "pcg_box_102x153x102", "rows": n,
                           "pcg": f"Jacobi, {args.pcg_mode}, {args.pcg_steps} reduction step order",
                           "layout": "grid rows (packed 16-byte records)"},
                "roofline": {"bound": "hbm", "kernel": "k_pcg_persistent", "achieved": achieved, "peak": peak,
                             "unit": "GB/s", "frac": achieved / peak, "peak_kind": peak_kind,
                             "algorithmic_bytes": "52 B per row per iteration", "traffic": None},
                "gpu_launches": int(launches)}
        print(json.dumps(line), flush=True)
    if ws > 1:
        dist.destroy_process_group()
    return 0


def run_fp64err(args, ws, rank, local):
    torch, dist = _torch_dist(ws, local)
    from banana_b200 import FlipSolver, scenes
    from oracle import oracle as O

    if rank != 0:
        return 0
    threads = os.cpu_count() or 1
    O.set_threads(threads)
    pos, vel = scenes.dam_break(N_GRID)
    dx = 1.0 / N_GRID
    ref = O.Oracle(scenes.dam_break_params(N_GRID, reduce_mode=0, nthreads=threads, sort_each_step=0, pcg_mode=1),
                   use_double=True)
    ref.set_particles(pos, vel)
    gpus = {}
    for name, mode in (("fp32", 0), ("refined", 2)):
        s = FlipSolver(scenes.dam_break_params(N_GRID, pcg_mode=mode))
        s.set_particles(pos, vel)
        gpus[name] = s
    per_step = []
    t0 = time.perf_counter()
    for k in range(args.steps):
        so = ref.step()
        row = {"step": k + 1, "dt_fp64": so["dt"]}
        po, _ = ref.get_particles(f64=True)
        for name, s in gpus.items():
            sg = s.step()
            pg, _ = s.get_particles()
            row[name] = {"dt": sg["dt"], "pos_err_dx": float(np.abs(pg.astype(np.float64) - po).max() / dx)}
        per_step.append(row)
    # velocity errors relative to the flow's top speed (a component that is nearly 0, like
    # the horizontal ones while the block falls, would make a per-component relative
    # error meaningless); the pressure error absolute, beside the FP64 pressure's range
    vref = {w: ref.grid(w, f64=True) for w in (0, 1, 2)}
    speed = max(float(np.abs(vref[w]).max()) for w in (0, 1, 2))
    pref = ref.grid(4, f64=True)
    fields = {"top_speed_fp64": speed, "pressure_abs_max_fp64": float(np.abs(pref).max())}
    for name, s in gpus.items():
        e = {}
        for f_, w in (("u", 0), ("v", 1), ("w", 2)):
            e[f_ + "_err_over_top_speed"] = float(np.abs(s.grid(w).astype(np.float64) - vref[w]).max() / speed)
        e["pressure_abs_err"] = float(np.abs(s.grid(4).astype(np.float64) - pref).max())
        fields[name] = e
    sec = time.perf_counter() - t0
    ref.close()
    line = {"metric": f"FP64-referenced error after the first sub-steps of the {N_GRID}^3 FLIP scene",
            "value": per_step[-1]["fp32"]["pos_err_dx"], "unit": "max |x - x_fp64| / dx", "n_gpus": 1,
            "steps": args.steps, "warmup": 0, "higher_is_better": False, "dtype": "f32 vs f64",
            "data": "synthetic (seeded dam break, seed 42)",
            "config": {"workload": "fp64_error_256", "reference": "oracle FP64 build (reference order, OpenMP)"},
            "per_step": per_step, "fields_last_step": fields, "seconds": sec}
    print(json.dumps(line), flush=True)
    return 0


def _spawn_ranks(n: int) -> int:
    """`--gpus N` (N > 1) run without a launcher: start N ranks of this same command on this
    node with torch.distributed.run (rendezvous on 127.0.0.1, a free port) and return the
    launcher's exit status."""
    import socket
    with socket.socket() as so:
        so.bind(("127.0.0.1", 0))
        port = so.getsockname()[1]
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", f"--nproc-per-node={n}",
           "--master-addr", "127.0.0.1", "--master-port", str(port), str(Path(__file__).resolve())] + sys.argv[1:]
    p = subprocess.Popen(cmd, start_new_session=True)
    try:
        return p.wait(timeout=3600)
    except subprocess.TimeoutExpired:
        os.killpg(p.pid, 9)
        p.wait()
        return 124


def main():
    global N_GRID, METRIC, WORKLOAD
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--pcg-mode", choices=["fp32", "fp64", "refined"], default="fp32")
    ap.add_argument("--solver", choices=list(SOLVERS), default="flip",
                    help="flip workload: the particle solver (FLIP is the headline; APIC / AFLIP / PIC the "
                         "reference's other PIC-family solvers on the same scene)")
    ap.add_argument("--pcg-steps", choices=["single", "two"], default="two",
                    help="PCG iteration form: PCGSolver's two-reduction order (default) or single reduction")
    ap.add_argument("--inner-tol", type=float, default=None, help="refined PCG: inner (FP32) relative tolerance")
    ap.add_argument("--tol", type=float, default=None,
                    help="fp32 / fp64 PCG: relative tolerance (the refined mode's outer tolerance is 1e-8)")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--tile-shape", type=int, default=None,
                    help="flip / batch / serve: use this P2G tile shape (bnn_set_tile_shape) instead of the "
                         "tuner's choice")
    ap.add_argument("--no-extras", action="store_true",
                    help="flip at 256^3 on one GPU: skip the other configurations' runs in detail.more_workloads")
    ap.add_argument("--per-step", action="store_true",
                    help="flip: add every timed sub-step's stage times to the line (detail.per_step)")
    ap.add_argument("--no-compare", action="store_true",
                    help="batch: skip the one-at-a-time and per-scene-stream comparison runs")
    ap.add_argument("--skip-e2e", action="store_true")
    ap.add_argument("--grid", type=int, default=N_GRID, help="fluid-domain resolution (profiling of smaller cases)")
    ap.add_argument("--ref-precond", choices=["jacobi", "ic0"], default="jacobi",
                    help="reference arm: Jacobi (the configs) or the reference's default symmetric MIC(0)")
    ap.add_argument("--workload", choices=["flip", "batch", "serve", "nsearch", "pcg", "fp64err", "aniso", "boundary"], default="flip")
    ap.add_argument("--workers", type=int, default=0, help="batch/serve: host threads stepping scenes (0 = auto)")
    ap.add_argument("--batch-mode", choices=["staged", "per_scene"], default="staged",
                    help="batch/serve: one launch per stage over the scenes (staged) or each scene on its own stream")
    ap.add_argument("--requests", type=int, default=100, help="serve: number of requests")
    ap.add_argument("--req-steps", type=int, default=200, help="serve: sub-steps per request")
    ap.add_argument("--time-limit", type=float, default=240.0, help="serve: stop after this many seconds")
    args = ap.parse_args()
    if "WORLD_SIZE" not in os.environ and args.gpus > 1:
        return _spawn_ranks(args.gpus)
    ws, rank, local = _dist()
    if ws != args.gpus:
        print(f"bench.py: --gpus {args.gpus} but the launcher started {ws} ranks", file=sys.stderr)
        return 2
    N_GRID = args.grid
    if N_GRID != 256:
        # a smaller (profiling) case names its own size
        METRIC = f"particle-steps/s at {N_GRID}^3 FLIP (1e-6 rel residual)"
        WORKLOAD = f"flip_dam_break_{N_GRID}"
    if args.impl == "reference":
        return run_reference(args, ws, rank)
    if args.workload == "batch":
        return run_batch(args, ws, rank, local)
    if args.workload == "serve":
        return run_serve(args, ws, rank, local)
    if args.workload == "nsearch":
        return run_nsearch(args, ws, rank, local)
    if args.workload == "pcg":
        return run_pcg(args, ws, rank, local)
    if args.workload == "fp64err":
        return run_fp64err(args, ws, rank, local)
    if args.workload == "aniso":
        return run_aniso(args, ws, rank, local)
    if args.workload == "boundary":
        return run_boundary(args, ws, rank, local)
    return run_ours(args, ws, rank, local)


if __name__ == "__main__":
    sys.exit(main())
