"""Throughput of the batched arena tick on B200 (arena-ticks/s), one JSON line on rank 0.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference] [--workload mixed|balls]

Workload `mixed` (default): 16,384 arenas per GPU mixed 55% 1v1 / 27% 2v2 / 18% 3v3 (seeded), default car body, in
the procedural ~11k-triangle arena, started with reset_to_kickoff. Controls come from the seeded generator (throttle,
steer, pitch, yaw, roll U[-1, 1]; jump / boost / handbrake Bernoulli 0.1 / 0.3 / 0.1; each sample held for U{1..30}
ticks). A step is one BatchSim::step_with_device_controls of 8 ticks (one kernel launch) over a [8, car_capacity]
control block resident in HBM. Workload `balls`: 16,384 ball-only arenas, balls at seeded positions with seeded
velocities up to 6000 uu/s, 8 ticks per step.

Arenas are independent, so N GPUs run N shards of 16,384 arenas each ("scaling": "weak") with no data-path collective;
the only cross-rank traffic is the timing max-reduction.

Timing: W untimed warm-up steps; then K steps, each timed with CUDA events on the launching stream after a 256 MiB L2
flush (outside the events), barrier + synchronize around the timed region, max over ranks. `e2e` times the same steps
through the public API from host code: each step copies its control block from pinned host memory to the device and
reads every car and ball state back into pinned memory (the observation), both inside the timed region.

`--impl reference` times the reference's own CPU implementation (oracle/_ref, built from the reference's sources) on
the same workload with all host threads, on a bounded sample of steps.
"""
from __future__ import annotations

import argparse
import ctypes
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
MAX_CARS = 6
METRIC = "arena-ticks/s"
CAR_BYTES, BALL_BYTES, ENV_BYTES, WHEEL_BYTES, CAR_MANIFOLD_BYTES, CTRL_BYTES, PAD_BYTES = 880, 288, 44, 292, 208, 24, 16
WORKLOADS = {
    "mixed": "16384 arenas/GPU mixed 55% 1v1 / 27% 2v2 / 18% 3v3 from kickoff, seeded held controls, procedural "
             "11k-tri arena, 8 ticks per launch",
    "balls": "ball-only arenas, 16384 arenas/GPU, procedural 11k-tri arena, 8 ticks per step",
}
# DRAM bytes (dram__bytes_read.sum + dram__bytes_write.sum) per step, from the ncu captures summarised under profiles/:
# balls, one tick_kernel launch of 8 ticks at 16,384 arenas; mixed, arena_finish + car_vehicle per tick at 4,096
# arenas times 8 ticks, scaled by 4 to 16,384 arenas (profiles/tick_kernels_mixed_car_arenas.md)
TRAFFIC_PER_LAUNCH = {"balls": 16.01e6, "mixed": 1.72e9}


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


# ---- the mixed workload's inputs (shared by both arms) -----------------------------------------------------------
def mixed_layout(seed: int):
    """Cars per arena (2/4/6 with p = .55/.27/.18) and teams (the first half of an arena's cars blue, the rest
    orange)."""
    rng = np.random.default_rng(seed)
    counts = rng.choice(np.array([2, 4, 6], np.int32), size=ENVS, p=[0.55, 0.27, 0.18]).astype(np.int32)
    teams = np.zeros(ENVS * MAX_CARS, np.uint8)
    for n in (2, 4, 6):
        idx = np.nonzero(counts == n)[0]
        for s in range(n // 2, n):
            teams[idx * MAX_CARS + s] = 1
    return counts, teams


def control_blocks(n_steps: int, seed: int) -> np.ndarray:
    """[n_steps, TICKS_PER_STEP, capacity, 24] control rows from the seeded generator (held U{1..30} ticks)."""
    from tests import scenarios
    cap = ENVS * MAX_CARS
    stream = scenarios.ControlStream(cap, seed=seed, p_jump=0.1, hold_max=30)
    out = np.empty((n_steps, TICKS_PER_STEP, cap, CTRL_BYTES), np.uint8)
    for s in range(n_steps):
        for t in range(TICKS_PER_STEP):
            out[s, t] = stream.next()
    return out


def run_ours(args, world, rank, local):
    import torch

    from rocketgpu_b200 import abi, arena
    from rocketgpu_b200.batch_sim import BatchSim, SimConfig

    torch.cuda.set_device(local)
    v, i = arena.generate()
    lib = abi.lib()
    stream = torch.cuda.current_stream()
    s_handle = ctypes.c_void_p(stream.cuda_stream)
    flush = torch.empty(256 * 1024 * 1024, dtype=torch.uint8, device="cuda")
    mixed = args.workload == "mixed"
    n_steps = args.warmup + args.steps
    if mixed:
        sim = BatchSim(SimConfig(env_count=ENVS, max_cars_per_env=MAX_CARS, kickoff_settled=0), v, i, device=local)
        counts, teams = mixed_layout(seed=7 + rank)
        sim.set_env_car_count(counts)
        sim.set_teams(teams)
        sim.reset_to_kickoff(1000 + rank)
        cap = sim.car_capacity()
        blocks_host = control_blocks(n_steps, seed=2000 + rank)
        blocks_dev = torch.from_numpy(blocks_host.reshape(n_steps, -1)).to("cuda")
        cars_total = int(counts.sum())
    else:
        from tests import scenarios
        sim = BatchSim(SimConfig(env_count=ENVS, max_cars_per_env=2), v, i, device=local)
        sim.set_env_car_count(np.zeros(ENVS, np.int32))
        default_ball = np.zeros(BALL_BYTES, np.uint8)
        lib.rg_default_ball_state(default_ball.ctypes.data)
        sim.upload_ball_states(scenarios.ball_states(default_ball, ENVS, seed=1000 + rank))
        cap, cars_total = 0, 0

    def step(k, ctrl_ptr=None):
        if mixed:
            ptr = ctrl_ptr if ctrl_ptr is not None else blocks_dev[k].data_ptr()
            rc = lib.rg_batch_step_with_device_controls(sim._h, ctypes.c_void_p(ptr), TICKS_PER_STEP, cap, s_handle)
        else:
            rc = lib.rg_batch_step(sim._h, TICKS_PER_STEP, s_handle)
        if rc != 0:
            raise RuntimeError(lib.rg_last_error().decode())

    for k in range(args.warmup):
        step(k)
    torch.cuda.synchronize()
    # device-timed region
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
    barrier(world)
    torch.cuda.synchronize()
    with ClockSampler(local) as clocks:
        for k in range(args.steps):
            flush.zero_()
            ev[k][0].record(stream)
            step(args.warmup + k)
            ev[k][1].record(stream)
        torch.cuda.synchronize()
    barrier(world)
    launch_ms = [a.elapsed_time(b) for a, b in ev]
    dev_s = max_over_ranks(sum(launch_ms) / 1e3, world)
    arena_ticks = ENVS * TICKS_PER_STEP * args.steps * world
    value = arena_ticks / dev_s

    # end to end through the public API: per step, the H2D copy of the step's control block from pinned memory, the
    # step, and the D2H read of every car and ball state into pinned memory; host wall time
    ball_pin = torch.empty((ENVS, BALL_BYTES), dtype=torch.uint8, pin_memory=True)
    h2d = 0
    if mixed:
        car_pin = torch.empty((cap, CAR_BYTES), dtype=torch.uint8, pin_memory=True)
        ctrl_pin = torch.from_numpy(blocks_host[args.warmup:].reshape(args.steps, -1)).pin_memory()
        ctrl_dev = torch.empty(ctrl_pin.shape[1], dtype=torch.uint8, device="cuda")
        h2d = ctrl_pin.shape[1]
        # the e2e pass replays the same control blocks from the state the timed pass left: same work per step
    barrier(world)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for k in range(args.steps):
        if mixed:
            ctrl_dev.copy_(ctrl_pin[k], non_blocking=True)
            step(None, ctrl_dev.data_ptr())
            rc = lib.rg_batch_download_car_states(sim._h, ctypes.c_void_p(car_pin.data_ptr()), cap, s_handle)
            if rc != 0:
                raise RuntimeError(lib.rg_last_error().decode())
        else:
            step(k)
        rc = lib.rg_batch_download_ball_states(sim._h, ctypes.c_void_p(ball_pin.data_ptr()), ENVS, s_handle)
        if rc != 0:
            raise RuntimeError(lib.rg_last_error().decode())
    torch.cuda.synchronize()
    e2e_s = max_over_ranks(time.perf_counter() - t0, world)
    e2e = arena_ticks / e2e_s
    d2h = ENVS * BALL_BYTES + cap * CAR_BYTES

    hbm, peak_kind = peaks()
    per_launch_ms = float(np.mean(launch_ms))
    if mixed:
        # algorithmic state bytes of one launch: each arena's ball, ball contact state, env, broadphase history and
        # pads read and written once; each active car's state, wheel record and car-mesh manifold read and written
        # once per tick, its controls read once per tick
        per_arena = 2 * (BALL_BYTES + 288 + ENV_BYTES + 1104 + 34 * PAD_BYTES)
        per_car_tick = 2 * (CAR_BYTES + WHEEL_BYTES + CAR_MANIFOLD_BYTES) + CTRL_BYTES
        bytes_per_launch = ENVS * per_arena + cars_total * per_car_tick * TICKS_PER_STEP
    else:
        bytes_per_launch = 2 * (BALL_BYTES + 288 + ENV_BYTES) * ENVS
    achieved = bytes_per_launch / (per_launch_ms / 1e3) / 1e9
    line = {
        "metric": METRIC, "value": value, "unit": "arena-ticks/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": dev_s * 1e3 / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic (seeded kickoff arenas and controls)" if mixed else "synthetic (seeded ball states)",
        "config": {"workload": WORKLOADS[args.workload], "arenas_per_gpu": ENVS, "ticks_per_step": TICKS_PER_STEP,
                   "cars_per_gpu": cars_total, "l2": "256 MiB flush before every timed step",
                   "parallelism": f"arena shards x{world}"},
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": hbm, "unit": "GB/s", "frac": achieved / hbm,
                     "peak_source": peak_kind, "traffic": TRAFFIC_PER_LAUNCH[args.workload],
                     "note": "per step (mixed: 8 ticks x 4 launches): algorithmic state bytes / step time; the tick is "
                             "latency bound (one thread per arena, data-dependent branches, dependent loads), not HBM "
                             "bound"},
        "e2e": {"value": e2e, "unit": "arena-ticks/s", "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h},
        # mixed: four kernels per tick (arena begin, per-car tick start, per-car vehicle update, arena finish);
        # balls: one per step
        "gpu_launches": args.steps * TICKS_PER_STEP * 4 if mixed else args.steps,
        "clocks": clocks.summary(),
    }
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        line["cpu_baseline"] = cpu_baseline(args.workload, sample_steps=args.cpu_steps)
    return line


def cpu_baseline(workload: str, sample_steps: int = 60):
    """The reference's own CPU BatchSim (oracle/_ref) on the same workload, all host threads, a bounded sample."""
    from rocketgpu_b200 import arena
    from tests import oracle_ref, scenarios
    if not oracle_ref.available():
        return {"value": None, "unit": "arena-ticks/s", "cores": 0, "kind": "reference",
                "sample": "oracle/_ref not built"}
    cores = os.cpu_count() or 1
    os.environ["ROCKETGPU_CPU_THREADS"] = str(cores)
    v, i = arena.generate()
    if workload == "mixed":
        sim = oracle_ref.OracleSim(ENVS, MAX_CARS, v, i, kickoff_settled=False)
        counts, teams = mixed_layout(seed=7)
        sim.set_env_car_count(counts)
        sim.set_teams(teams)
        sim.reset_to_kickoff(1000)
        cap = ENVS * MAX_CARS
        stream = scenarios.ControlStream(cap, seed=2000, p_jump=0.1, hold_max=30)

        def one(k):
            block = np.stack([stream.next() for _ in range(TICKS_PER_STEP)])
            sim.step_with_controls(block.reshape(-1, CTRL_BYTES), TICKS_PER_STEP, cap)
    else:
        sim = oracle_ref.OracleSim(ENVS, 2, v, i, kickoff_settled=False)
        sim.set_env_car_count([0] * ENVS)
        _, default_ball, _, _, _ = oracle_ref.default_states()
        sim.upload_balls(scenarios.ball_states(default_ball, ENVS, seed=1000))

        def one(k):
            sim.step(TICKS_PER_STEP)
    one(0)
    t0 = time.perf_counter()
    for k in range(sample_steps):
        one(k + 1)
    dt = time.perf_counter() - t0
    return {"value": ENVS * TICKS_PER_STEP * sample_steps / dt, "unit": "arena-ticks/s", "cores": cores,
            "kind": "reference",
            "sample": f"{sample_steps} steps x {TICKS_PER_STEP} ticks x {ENVS} arenas ({workload}), "
                      f"ROCKETGPU_CPU_THREADS={cores}"}


def run_reference(args, world, rank):
    if rank != 0:
        return None
    cb = cpu_baseline(args.workload, sample_steps=max(1, min(args.steps, args.cpu_steps)))
    line = {
        "impl": "reference", "metric": METRIC, "value": cb["value"], "unit": "arena-ticks/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded kickoff arenas and controls)",
        "config": {"workload": WORKLOADS[args.workload], "arenas_per_gpu": ENVS, "ticks_per_step": TICKS_PER_STEP},
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
    ap.add_argument("--workload", default="mixed", choices=sorted(WORKLOADS))
    ap.add_argument("--cpu-steps", type=int, default=60)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--arenas", type=int, default=ENVS, help="arenas per GPU (smaller cases for profiling)")
    args = ap.parse_args()
    if args.arenas != ENVS:
        globals()["ENVS"] = args.arenas
        for k in WORKLOADS:
            WORKLOADS[k] = WORKLOADS[k].replace("16384 arenas", f"{args.arenas} arenas")
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
