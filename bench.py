"""Throughput of the batched arena tick on B200 (arena-ticks/s), one JSON line on rank 0.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Workload: 16,384 ball-only arenas in the procedural ~11k-triangle arena, each ball started from a seeded position
with a seeded velocity (uniform direction, speed up to 6000 uu/s); a step is one BatchSim step of 8 ticks (one
kernel launch), as the reference's bench steps 8 ticks per call. Arenas are independent, so N GPUs run N shards of
16,384 arenas each ("scaling": "weak") with no data-path collective; the only cross-rank traffic is the timing
max-reduction.

Timing: W untimed warm-up steps; then K steps, each timed with CUDA events on the launching stream after a 256 MiB L2
flush (outside the events), barrier + synchronize around the timed region, max over ranks. `e2e` times the same steps
through the C ABI from host code, including each step's device-to-host copy of every ball state (the observation) into
pinned memory; BatchSim::step takes no per-step input, so h2d_bytes_per_step is 0.

`--impl reference` times the reference's own CPU implementation (oracle/_ref, built from the reference's sources) on
the same workload with all host threads, on a bounded sample of steps.
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

ENVS = 16384
TICKS_PER_STEP = 8
METRIC = "arena-ticks/s"
WORKLOAD = "ball-only arenas, 16384 arenas/GPU, procedural 11k-tri arena, 8 ticks per step"
# dram__bytes_read.sum + dram__bytes_write.sum of one tick_kernel launch at this workload, from the ncu capture
# summarised in profiles/tick_kernel_ball_arenas_16k.md
TRAFFIC_PER_LAUNCH = 16.01e6
STATE_BYTES_PER_ARENA = 288 + 288 + 44  # ball struct + ball contact state + env struct, read and written per launch


def peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            d = json.load(f)
        return float(d.get("hbm_gbs", 6650.0)), "measured"
    return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi clocks / throttle reasons sampled every 200 ms during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu: int):
        self.gpu = gpu
        self.rows = []
        self.proc = None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.gpu), f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "200"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except (OSError, FileNotFoundError):
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.rows.append([x.strip() for x in line.split(",")])

    def __exit__(self, *exc):
        if self.proc:
            time.sleep(0.25)
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        if not self.rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = [float(r[1]) for r in self.rows if r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in self.rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[k] for r in self.rows for k in range(4) if len(r) > 5 + k and r[5 + k] == "Active"})
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(self.rows)}


def dist_setup(n_gpus):
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import datetime

        import torch
        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    return world, rank, local


def max_over_ranks(x: float, world: int) -> float:
    if world == 1:
        return x
    import torch
    import torch.distributed as dist
    t = torch.tensor([x], dtype=torch.float64, device="cuda")
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def barrier(world):
    if world > 1:
        import torch.distributed as dist
        dist.barrier()


def run_ours(args, world, rank, local):
    import ctypes

    import torch

    from rocketgpu_b200 import abi, arena
    from rocketgpu_b200.batch_sim import BatchSim, SimConfig
    from tests import scenarios

    torch.cuda.set_device(local)
    v, i = arena.generate()
    sim = BatchSim(SimConfig(env_count=ENVS, max_cars_per_env=2), v, i, device=local)
    sim.set_env_car_count(np.zeros(ENVS, np.int32))
    default_ball = np.zeros(288, np.uint8)
    abi.lib().rg_default_ball_state(default_ball.ctypes.data)
    init = scenarios.ball_states(default_ball, ENVS, seed=1000 + rank)
    sim.upload_ball_states(init)
    stream = torch.cuda.current_stream()
    s_handle = ctypes.c_void_p(stream.cuda_stream)
    flush = torch.empty(256 * 1024 * 1024, dtype=torch.uint8, device="cuda")
    lib = abi.lib()

    def step():
        rc = lib.rg_batch_step(sim._h, TICKS_PER_STEP, s_handle)
        if rc != 0:
            raise RuntimeError(lib.rg_last_error().decode())

    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()
    # device-timed region
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
    barrier(world)
    torch.cuda.synchronize()
    with ClockSampler(local) as clocks:
        for k in range(args.steps):
            flush.zero_()
            ev[k][0].record(stream)
            step()
            ev[k][1].record(stream)
        torch.cuda.synchronize()
    barrier(world)
    launch_ms = [a.elapsed_time(b) for a, b in ev]
    dev_s = max_over_ranks(sum(launch_ms) / 1e3, world)
    arena_ticks = ENVS * TICKS_PER_STEP * args.steps * world
    value = arena_ticks / dev_s

    # end to end through the C ABI: step + D2H of all ball states into pinned memory, host wall time per step
    pinned = torch.empty((ENVS, 288), dtype=torch.uint8, pin_memory=True)
    barrier(world)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for _ in range(args.steps):
        step()
        rc = lib.rg_batch_download_ball_states(sim._h, ctypes.c_void_p(pinned.data_ptr()), ENVS, s_handle)
        if rc != 0:
            raise RuntimeError(lib.rg_last_error().decode())
    torch.cuda.synchronize()
    e2e_s = max_over_ranks(time.perf_counter() - t0, world)
    e2e = arena_ticks / e2e_s

    hbm, peak_kind = peaks()
    per_launch_ms = float(np.mean(launch_ms))
    bytes_per_launch = 2 * STATE_BYTES_PER_ARENA * ENVS
    achieved = bytes_per_launch / (per_launch_ms / 1e3) / 1e9
    line = {
        "metric": METRIC, "value": value, "unit": "arena-ticks/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": dev_s * 1e3 / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded ball states)",
        "config": {"workload": WORKLOAD, "arenas_per_gpu": ENVS, "ticks_per_step": TICKS_PER_STEP,
                   "l2": "256 MiB flush before every timed step", "parallelism": f"arena shards x{world}"},
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": hbm, "unit": "GB/s", "frac": achieved / hbm,
                     "peak_source": peak_kind, "traffic": TRAFFIC_PER_LAUNCH,
                     "note": "state traffic only; the tick is FP32-issue/latency bound, not HBM bound"},
        "e2e": {"value": e2e, "unit": "arena-ticks/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": ENVS * 288},
        "gpu_launches": args.steps,
        "clocks": clocks.summary(),
    }
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        line["cpu_baseline"] = cpu_baseline(sample_steps=args.cpu_steps)
    return line


def cpu_baseline(sample_steps: int = 4):
    """The reference's own CPU BatchSim (oracle/_ref) on the same workload, all host threads, a bounded sample."""
    from rocketgpu_b200 import arena
    from tests import oracle_ref, scenarios
    if not oracle_ref.available():
        return {"value": None, "unit": "arena-ticks/s", "cores": 0, "kind": "reference",
                "sample": "oracle/_ref not built"}
    cores = os.cpu_count() or 1
    os.environ["ROCKETGPU_CPU_THREADS"] = str(cores)
    v, i = arena.generate()
    sim = oracle_ref.OracleSim(ENVS, 2, v, i, kickoff_settled=False)
    sim.set_env_car_count([0] * ENVS)
    _, default_ball, _, _, _ = oracle_ref.default_states()
    sim.upload_balls(scenarios.ball_states(default_ball, ENVS, seed=1000))
    sim.step(TICKS_PER_STEP)
    t0 = time.perf_counter()
    for _ in range(sample_steps):
        sim.step(TICKS_PER_STEP)
    dt = time.perf_counter() - t0
    return {"value": ENVS * TICKS_PER_STEP * sample_steps / dt, "unit": "arena-ticks/s", "cores": cores,
            "kind": "reference",
            "sample": f"{sample_steps} steps x {TICKS_PER_STEP} ticks x {ENVS} arenas, ROCKETGPU_CPU_THREADS={cores}"}


def run_reference(args, world, rank):
    if rank != 0:
        return None
    cb = cpu_baseline(sample_steps=max(1, args.steps))
    line = {
        "impl": "reference", "metric": METRIC, "value": cb["value"], "unit": "arena-ticks/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded ball states)",
        "config": {"workload": WORKLOAD, "arenas_per_gpu": ENVS, "ticks_per_step": TICKS_PER_STEP},
        "cpu_baseline": cb,
        "e2e": {"value": cb["value"], "unit": "arena-ticks/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    return line


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=50)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--cpu-steps", type=int, default=4)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3
    if args.impl == "reference":
        world = int(os.environ.get("WORLD_SIZE", "1"))
        rank = int(os.environ.get("RANK", "0"))
        line = run_reference(args, world, rank)
    else:
        world, rank, local = dist_setup(args.gpus)
        line = run_ours(args, world, rank, local)
        if world > 1:
            import torch.distributed as dist
            dist.destroy_process_group()
    if line is not None and int(os.environ.get("RANK", "0")) == 0:
        print(json.dumps(line), flush=True)


if __name__ == "__main__":
    main()
