"""Throughput of the batched arena tick on B200 (arena-ticks/s), one JSON line on rank 0.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference] [--workload mixed|balls]

Workload `mixed` (default): 16,384 arenas per GPU mixed 55% 1v1 / 27% 2v2 / 18% 3v3 (seeded), car bodies drawn
uniformly from the six hitbox presets (Octane, Dominus, Plank, Breakout, Hybrid, Merc), in the procedural ~11k-triangle
arena. Controls come from the seeded generator (throttle, steer, pitch, yaw, roll U[-1, 1]; jump / boost / handbrake
Bernoulli 0.1 / 0.3 / 0.1; each sample held for U{1..30} ticks). An arena resets to kickoff when its ball is scored or
when no car has touched the ball for 300 ticks; the no-touch clocks start at seeded ages, so resets are spread over the
ticks. A step is 8 ticks: one BatchSim::step_with_device_commands over a [8, car_capacity] control block resident in
HBM, whose first tick applies the resets rg_batch_episode_commands chose after the previous step (6 kernels per tick
plus the episode kernel, 49 launches per step).

Steady state: every arena starts from kickoff, so SETTLE_STEPS untimed steps (320 ticks) run first, then W warm-up
steps; the K timed steps follow. Every pass (the device-timed pass, the end-to-end pass and the CPU baseline / the
reference arm) runs the same settle and warm-up and then times the same K steps, so all numbers cover the same ticks.

Workload `balls`: 16,384 ball-only arenas, balls at seeded positions with seeded velocities up to 6000 uu/s, 8 ticks
per step (one launch).

Arenas are independent, so N GPUs run N shards of 16,384 arenas each ("scaling": "weak") with no data-path collective;
the only cross-rank traffic is the timing max-reduction.

Timing: K steps, each timed with CUDA events on the launching stream after a 256 MiB L2 flush (outside the events),
barrier + synchronize around the timed region, max over ranks; p50 / p99 of the per-step times. `e2e` times the same
K steps through the public API on a second batch brought to the same state: each step copies its control block from
pinned host memory to the device, steps, and reads every car and ball state back into pinned memory, all inside the
timed region (host wall clock).

Parity: rank 0 at N=1 steps the oracle (the reference's own CPU BatchSim, oracle/_ref) through the same settle,
warm-up and K steps with the same controls and the same reset decisions (made on the host from the oracle's state),
and compares every arena's cars and ball after each of the K steps of the end-to-end pass, and every arena's cars,
ball, env and pads at the end of the device-timed pass, bitwise (NaN payloads aside). The oracle's K step calls,
timed, are the CPU baseline.

`--impl reference` runs that CPU leg alone and reports it (the reference's own CPU implementation with all host
threads, on the same workload, settle, warm-up and timed steps).
"""
from __future__ import annotations

import argparse
import hashlib
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
EVENTS = 0  # --events: physics event records per arena (0: the stream is off)
TICKS_PER_STEP = 8
KERNELS_PER_TICK = 7  # arena begin, car tick start, wheel rays, vehicle updates, arena finish, car post-tick, arena tail
SETTLE_STEPS = 40
NO_TOUCH_TICKS = 300
MAX_CARS = 6
METRIC = "arena-ticks/s"
CAR_BYTES, BALL_BYTES, ENV_BYTES, PAD_BYTES, CTRL_BYTES, CMD_BYTES = 880, 288, 44, 16, 24, 16
WORKLOADS = {
    "mixed": "16384 arenas/GPU mixed 55% 1v1 / 27% 2v2 / 18% 3v3, six hitbox presets, goal or 300-tick no-touch "
             "resets (staggered clocks), seeded held controls, procedural 11k-tri arena, 8 ticks per step, "
             "320-tick settle before warm-up",
    "balls": "ball-only arenas, 16384 arenas/GPU, procedural 11k-tri arena, 8 ticks per step",
    "serve": "serving loop (see config.workload)",
}
# Algorithmic bytes of one launch (one tick) of each kernel of the car path: read + write of the state it owns, as
# (bytes per arena, per active car, per car pair). Struct sizes: car 880, wheel record 292, car config 120, controls
# 24, tick record 136, car stage 1,176 (prestep 56, predictive contact 20, proxy 148, car/mesh manifold 176, query
# rows and result 776), car/mesh manifold 176, car/ball manifold 272, car-pair manifold 260, ball 288, ball contact
# state 288, env 44, broadphase history 1,376, 34 pads x 16, tick snapshot 24.
KERNEL_BYTES = {
    "arena_begin": (2 * (288 + 44 + 34 * 16) + 24 + 16, 0, 0),
    "car_pre": (0, 2 * (880 + 292) + 120 + 24 + 136, 0),
    "car_vehicle": (0, 2 * (880 + 292) + 120 + 24 + 288 + 136 + 176 + 1176, 0),
    "arena_finish": (2 * (288 + 288 + 1344) + 44 + 24, 2 * (880 + 176 + 272) + 120 + 136 + 1176, 2 * 260),
    "car_post": (0, 2 * 880 + 292 + 56 + 24, 0),
    "arena_tail": (2 * (288 + 44 + 34 * 16), 2 * 880 + 120, 0),
}
KERNEL_NAMES = ("arena_begin", "car_pre", "car_vehicle", "arena_finish", "car_post", "arena_tail")
# DRAM bytes (dram__bytes_read.sum + dram__bytes_write.sum) per car of one car_vehicle_kernel launch, from an ncu
# --set full capture of the mixed workload at 4,096 arenas (13,350 cars: 31.01 MB read + 13.92 MB written); a launch
# at the bench's size is scaled by its cars (the kernel's traffic is per car: its state, stage and mesh reads).
KERNEL_TRAFFIC_PER_CAR = {"car_vehicle": (31.014656e6 + 13.916416e6) / 13350}


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
            time.sleep(0.3)
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
    device = "cuda" if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor([x], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def barrier(world):
    if world > 1:
        import torch.distributed as dist
        dist.barrier()


# ---- the mixed workload's inputs (shared by every pass) ----------------------------------------------------------
class MixedWorkload:
    """Cars per arena (2/4/6 with p = .55/.27/.18), teams (the first half of an arena's cars blue), car bodies (uniform
    over the six presets), and the seeded control stream, for shard `rank`."""

    def __init__(self, rank: int):
        rng = np.random.default_rng(7 + rank)
        self.counts = rng.choice(np.array([2, 4, 6], np.int32), size=ENVS, p=[0.55, 0.27, 0.18]).astype(np.int32)
        self.teams = np.zeros(ENVS * MAX_CARS, np.uint8)
        for n in (2, 4, 6):
            idx = np.nonzero(self.counts == n)[0]
            for s in range(n // 2, n):
                self.teams[idx * MAX_CARS + s] = 1
        self.bodies = rng.integers(0, 6, ENVS * MAX_CARS)
        self.reset_seed = 1000 + rank
        self.control_seed = 2000 + rank
        self.stagger_seed = 3000 + rank

    def car_configs(self, presets: list[np.ndarray]) -> np.ndarray:
        return np.stack(presets)[self.bodies]

    def controls(self):
        """Generator of [TICKS_PER_STEP * capacity, 24] control blocks, one per step from the first settle step."""
        from tests import scenarios
        stream = scenarios.ControlStream(ENVS * MAX_CARS, seed=self.control_seed, p_jump=0.1, hold_max=30)
        while True:
            yield np.stack([stream.next() for _ in range(TICKS_PER_STEP)]).reshape(-1, CTRL_BYTES)


def _presets():
    """The six hitbox presets (CarConfig rows) from the library."""
    from rocketgpu_b200.batch_sim import car_preset
    return [car_preset(k) for k in range(6)]


def arena_hashes(rows: np.ndarray, per_arena: int) -> np.ndarray:
    """One 64-bit polynomial hash per arena of its rows (NaN words canonicalised), for per-step parity checks."""
    flat = np.ascontiguousarray(rows).reshape(ENVS, -1)
    pad = (-flat.shape[1]) % 8
    if pad:
        flat = np.concatenate([flat, np.zeros((ENVS, pad), np.uint8)], axis=1)
    w32 = flat.view(np.uint32).copy()
    w32[np.isnan(w32.view(np.float32))] = 0x7FC00000
    w = w32.view(np.uint64)
    k = (np.arange(w.shape[1], dtype=np.uint64) * np.uint64(0x9E3779B97F4A7C15)) | np.uint64(1)
    with np.errstate(over="ignore"):
        return (w * k).sum(axis=1, dtype=np.uint64) ^ (w ^ k).sum(axis=1, dtype=np.uint64)


def _active_car_rows(cars: np.ndarray, counts: np.ndarray) -> np.ndarray:
    """Car rows with the inactive slots zeroed (they are not part of the comparison)."""
    c = cars.reshape(ENVS, MAX_CARS, CAR_BYTES).copy()
    c[np.arange(MAX_CARS)[None, :] >= counts[:, None]] = 0
    return c


# ---- the CPU leg: the reference's own CPU BatchSim --------------------------------------------------------------
def oracle_lib_path():
    """The timed CPU build (-march=x86-64-v3) when it loads on this host, else the portable one."""
    from tests import oracle_ref
    native = os.path.join(ROOT, "oracle", "_ref", "librg_oracle_native.so")
    if os.path.exists(native):
        try:
            ctypes.CDLL(native)
            return native, "x86-64-v3"
        except OSError:
            pass
    return oracle_ref.LIB_PATH, "x86-64"


def cpu_leg(workload: str, warmup: int, steps: int, parity: bool):
    """Runs the reference's CPU BatchSim through the settle, warm-up and `steps` timed steps of the workload with all
    host threads. Returns the timing record and, with `parity`, the per-step arena hashes and the final state."""
    from rocketgpu_b200 import arena
    from tests import oracle_ref, scenarios
    if not oracle_ref.available():
        return {"value": None, "unit": "arena-ticks/s", "cores": 0, "kind": "reference",
                "sample": "oracle/_ref not built"}, None
    cores = os.cpu_count() or 1
    os.environ["ROCKETGPU_CPU_THREADS"] = str(cores)
    path, arch = oracle_lib_path()
    if oracle_ref.LIB_PATH != path:
        oracle_ref.LIB_PATH = path
        oracle_ref._lib = None
    v, i = arena.generate()
    record = {"hashes": [], "final": None}
    step_s = []
    if workload == "mixed":
        w = MixedWorkload(0)
        sim = oracle_ref.OracleSim(ENVS, MAX_CARS, v, i, kickoff_settled=False)
        sim.set_env_car_count(w.counts)
        sim.set_teams(w.teams)
        sim.set_car_configs(w.car_configs(_presets()))
        sim.reset_to_kickoff(w.reset_seed)
        events = sim.set_physics_event_stream(EVENTS) if EVENTS else None
        clock = scenarios.EpisodeClock(sim.envs(), sim.cars(), MAX_CARS, NO_TOUCH_TICKS, w.stagger_seed)
        cmds = np.zeros((TICKS_PER_STEP * ENVS, CMD_BYTES), np.uint8)
        gen = w.controls()
        total = SETTLE_STEPS + warmup + steps
        for k in range(total):
            block = next(gen)
            t0 = time.perf_counter()
            if events is not None:
                events[1].view(np.uint32).reshape(-1, 4)[:, 2:] = 0  # each window's count and overflow
            sim.step_with_commands(block, ENVS * MAX_CARS, cmds, ENVS, TICKS_PER_STEP)
            dt = time.perf_counter() - t0
            cars, envs = sim.cars(), sim.envs()
            timed = k >= SETTLE_STEPS + warmup
            if timed:
                step_s.append(dt)
                if parity:
                    record["hashes"].append((arena_hashes(_active_car_rows(cars, w.counts), MAX_CARS * CAR_BYTES),
                                             arena_hashes(sim.balls(), BALL_BYTES)))
            cmds[:ENVS] = clock.commands(envs, cars, w.counts)
        if parity:
            record["final"] = (_active_car_rows(sim.cars(), w.counts), sim.balls(), sim.envs(), sim.pads())
    else:
        sim = oracle_ref.OracleSim(ENVS, 2, v, i, kickoff_settled=False)
        sim.set_env_car_count([0] * ENVS)
        _, default_ball, _, _, _ = oracle_ref.default_states()
        sim.upload_balls(scenarios.ball_states(default_ball, ENVS, seed=1000))
        for k in range(warmup + steps):
            t0 = time.perf_counter()
            sim.step(TICKS_PER_STEP)
            if k >= warmup:
                step_s.append(time.perf_counter() - t0)
        if parity:
            record["final"] = (None, sim.balls(), sim.envs(), None)
    sim.close()
    value = ENVS * TICKS_PER_STEP * len(step_s) / sum(step_s)
    timing = {"value": value, "unit": "arena-ticks/s", "cores": cores, "kind": "reference",
              "sample": f"the timed {len(step_s)} steps x {TICKS_PER_STEP} ticks x {ENVS} arenas ({workload}) after "
                        f"the same settle and warm-up, step calls only, ROCKETGPU_CPU_THREADS={cores}, oracle built "
                        f"for {arch}"}
    return timing, record


# ---- our arm ------------------------------------------------------------------------------------------------------
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

    def check(rc):
        if rc != 0:
            raise RuntimeError(lib.rg_last_error().decode())

    w = MixedWorkload(rank) if mixed else None
    presets = _presets() if mixed else None

    def make_sim():
        if mixed:
            sim = BatchSim(SimConfig(kickoff_settled=0, env_count=ENVS, max_cars_per_env=MAX_CARS), v, i, device=local)
            sim.set_env_car_count(w.counts)
            sim.set_teams(w.teams)
            sim.set_car_configs(w.car_configs(presets))
            sim.reset_to_kickoff(w.reset_seed)
            if EVENTS:
                sim.events = (torch.zeros(ENVS * EVENTS * 104, dtype=torch.uint8, device="cuda"),
                              torch.zeros(ENVS * 16, dtype=torch.uint8, device="cuda"))
                sim.set_physics_event_stream(sim.events[0].data_ptr(), sim.events[1].data_ptr(), EVENTS)
            cmds = torch.zeros((TICKS_PER_STEP, ENVS, CMD_BYTES), dtype=torch.uint8, device="cuda")
            check(lib.rg_batch_episode_commands(sim._h, NO_TOUCH_TICKS, w.stagger_seed, 1,
                                                ctypes.c_void_p(cmds.data_ptr()), s_handle))
            return sim, cmds
        from tests import scenarios
        sim = BatchSim(SimConfig(kickoff_settled=0, env_count=ENVS, max_cars_per_env=2), v, i, device=local)
        sim.set_env_car_count(np.zeros(ENVS, np.int32))
        default_ball = np.zeros(BALL_BYTES, np.uint8)
        lib.rg_default_ball_state(default_ball.ctypes.data)
        sim.upload_ball_states(scenarios.ball_states(default_ball, ENVS, seed=1000 + rank))
        return sim, None

    cap = ENVS * MAX_CARS

    def step(sim, cmds, ctrl_ptr):
        if mixed:
            if EVENTS:
                sim.events[1].zero_()  # the windows, on the step's stream
            check(lib.rg_batch_step_with_device_commands(sim._h, ctypes.c_void_p(ctrl_ptr), cap,
                                                         ctypes.c_void_p(cmds.data_ptr()), ENVS, TICKS_PER_STEP,
                                                         s_handle))
            check(lib.rg_batch_episode_commands(sim._h, NO_TOUCH_TICKS, 0, 0, ctypes.c_void_p(cmds.data_ptr()),
                                                s_handle))
        else:
            check(lib.rg_batch_step(sim._h, TICKS_PER_STEP, s_handle))

    # the timed steps' control blocks, resident in HBM (device pass) and in pinned host memory (end-to-end pass)
    settle = SETTLE_STEPS if mixed else 0
    pre_steps = settle + args.warmup
    gen = w.controls() if mixed else None
    ctrl_dev = torch.empty(cap * TICKS_PER_STEP * CTRL_BYTES, dtype=torch.uint8, device="cuda") if mixed else None
    pre_blocks = []
    timed_pin = None
    if mixed:
        for k in range(pre_steps):
            pre_blocks.append(next(gen))
        timed_pin = torch.empty((args.steps, cap * TICKS_PER_STEP * CTRL_BYTES), dtype=torch.uint8, pin_memory=True)
        for k in range(args.steps):
            timed_pin[k].copy_(torch.from_numpy(next(gen).reshape(-1)))
        timed_dev = timed_pin.to("cuda")

    def bring_up():
        sim, cmds = make_sim()
        for k in range(pre_steps):
            if mixed:
                ctrl_dev.copy_(torch.from_numpy(pre_blocks[k].reshape(-1)))
                step(sim, cmds, ctrl_dev.data_ptr())
            else:
                step(sim, None, None)
        torch.cuda.synchronize()
        return sim, cmds

    # device-timed pass
    sim_a, cmds_a = bring_up()
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
    if mixed:
        check(lib.rg_batch_phase_timing(sim_a._h, 1))
    barrier(world)
    torch.cuda.synchronize()
    with ClockSampler(local) as clocks:
        torch.cuda.nvtx.range_push("timed")  # profilers select the timed steps' launches by this range
        for k in range(args.steps):
            flush.zero_()
            ev[k][0].record(stream)
            step(sim_a, cmds_a, timed_dev[k].data_ptr() if mixed else None)
            ev[k][1].record(stream)
        torch.cuda.synchronize()
        torch.cuda.nvtx.range_pop()
    barrier(world)
    step_ms = [a.elapsed_time(b) for a, b in ev]
    phase_ms = (ctypes.c_float * 6)()
    phase_ticks = ctypes.c_int64(0)
    if mixed:
        check(lib.rg_batch_phase_times(sim_a._h, phase_ms, ctypes.byref(phase_ticks)))
        check(lib.rg_batch_phase_timing(sim_a._h, 0))
    dev_s = max_over_ranks(sum(step_ms) / 1e3, world)
    arena_ticks = ENVS * TICKS_PER_STEP * args.steps * world
    value = arena_ticks / dev_s
    final_a = None
    if mixed:
        final_a = (_active_car_rows(sim_a.download_car_states(), w.counts), sim_a.download_ball_states(),
                   sim_a.download_env_states(), sim_a.download_boost_pad_states())
    else:
        final_a = (None, sim_a.download_ball_states(), sim_a.download_env_states(), None)
    sim_a.close()

    # end-to-end pass through the public API, on a second batch brought to the same state
    sim_b, cmds_b = bring_up()
    ball_pin = torch.empty((ENVS, BALL_BYTES), dtype=torch.uint8, pin_memory=True)
    car_pin = torch.empty((max(cap, 1), CAR_BYTES), dtype=torch.uint8, pin_memory=True)
    e2e_hashes = []
    e2e_ms = []
    barrier(world)
    torch.cuda.synchronize()
    for k in range(args.steps):
        t0 = time.perf_counter()
        if mixed:
            ctrl_dev.copy_(timed_pin[k], non_blocking=True)
            step(sim_b, cmds_b, ctrl_dev.data_ptr())
            check(lib.rg_batch_download_car_states(sim_b._h, ctypes.c_void_p(car_pin.data_ptr()), cap, s_handle))
        else:
            step(sim_b, None, None)
        check(lib.rg_batch_download_ball_states(sim_b._h, ctypes.c_void_p(ball_pin.data_ptr()), ENVS, s_handle))
        e2e_ms.append((time.perf_counter() - t0) * 1e3)
        if mixed and rank == 0 and world == 1 and not args.no_cpu_baseline:
            # outside the timed region: this step's observation, hashed for the parity check
            e2e_hashes.append((arena_hashes(_active_car_rows(car_pin.numpy(), w.counts), MAX_CARS * CAR_BYTES),
                               arena_hashes(ball_pin.numpy(), BALL_BYTES)))
    torch.cuda.synchronize()
    e2e_s = max_over_ranks(sum(e2e_ms) / 1e3, world)
    e2e = arena_ticks / e2e_s
    h2d = cap * TICKS_PER_STEP * CTRL_BYTES if mixed else 0
    d2h = ENVS * BALL_BYTES + (cap * CAR_BYTES if mixed else 0)
    sim_b.close()

    hbm, peak_kind = peaks()
    line = {
        "metric": METRIC, "value": value, "unit": "arena-ticks/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": dev_s * 1e3 / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic (seeded arenas, bodies, controls and episode resets)" if mixed
        else "synthetic (seeded ball states)",
        "config": {"workload": WORKLOADS[args.workload], "arenas_per_gpu": ENVS, "ticks_per_step": TICKS_PER_STEP,
                   "settle_steps": settle, "l2": "256 MiB flush before every timed step",
                   "parallelism": f"arena shards x{world}", **({"events_per_arena": EVENTS} if EVENTS else {})},
        "latency_ms_per_step": {"p50": float(np.percentile(step_ms, 50)), "p99": float(np.percentile(step_ms, 99)),
                                "max": float(np.max(step_ms)), "e2e_p50": float(np.percentile(e2e_ms, 50)),
                                "e2e_p99": float(np.percentile(e2e_ms, 99))},
        "e2e": {"value": e2e, "unit": "arena-ticks/s", "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h},
        "gpu_launches": args.steps * (TICKS_PER_STEP * KERNELS_PER_TICK + 1) if mixed else args.steps,
        "clocks": clocks.summary(),
    }
    if mixed:
        cars_total = int(w.counts.sum())
        pairs_total = int((w.counts * (w.counts - 1) // 2).sum())
        ticks = max(1, phase_ticks.value)
        per_launch_ms = {name: phase_ms[k] / ticks for k, name in enumerate(KERNEL_NAMES)}
        top = max(per_launch_ms, key=per_launch_ms.get)
        pa, pc, pp = KERNEL_BYTES[top]
        top_bytes = ENVS * pa + cars_total * pc + pairs_total * pp
        achieved = top_bytes / (per_launch_ms[top] / 1e3) / 1e9
        line["config"]["cars_per_gpu"] = cars_total
        line["roofline"] = {
            "bound": "hbm", "kernel": top, "achieved": achieved, "peak": hbm, "unit": "GB/s",
            "frac": achieved / hbm, "peak_source": peak_kind,
            "traffic": KERNEL_TRAFFIC_PER_CAR[top] * cars_total if top in KERNEL_TRAFFIC_PER_CAR else None,
            "traffic_note": "car_vehicle_kernel alone (the phase also holds car_rays_kernel), 4,096-arena ncu capture "
                            "scaled by cars",
            "algorithmic_bytes_per_launch": top_bytes, "avg_launch_ms": per_launch_ms[top],
            "note": "dominant kernel by device time; the tick is bound by latency and FP32 issue of serial per-arena "
                    "work, not by HBM; frac is the HBM fraction of its algorithmic state bytes"}
        line["kernel_ms_per_step"] = {name: ms * TICKS_PER_STEP for name, ms in per_launch_ms.items()}
        # the same digest as the reference CUDA arm's (--impl reference --ref-backend cuda) after the same ticks
        line["final_state_sha"] = hashlib.sha256(final_a[0].tobytes() + final_a[1].tobytes()).hexdigest()[:16]
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        timing, record = cpu_leg(args.workload, args.warmup, args.steps, parity=True)
        line["cpu_baseline"] = timing
        if record is not None:
            line["parity"] = parity_summary(record, e2e_hashes, final_a, mixed)
    return line


def parity_summary(record, e2e_hashes, final_a, mixed):
    from tests import parity
    bad_steps = np.zeros(ENVS, bool)
    for (oc, ob), (gc, gb) in zip(record["hashes"], e2e_hashes):
        bad_steps |= (oc != gc) | (ob != gb)
    oc, ob, oe, op = record["final"]
    gc, gb, ge, gp = final_a
    bad_final = np.zeros(ENVS, bool)
    for o, g in ((oc, gc), (ob, gb), (oe, ge), (op, gp)):
        if o is None:
            continue
        o = o.reshape(ENVS, -1)
        g = g.reshape(ENVS, -1)
        diff = np.nonzero((o != g).any(axis=1))[0]
        for e in diff:
            if not parity.equal(o[e], g[e]):
                bad_final[e] = True
    return {"arenas": ENVS, "ticks_compared": len(e2e_hashes) * TICKS_PER_STEP,
            "compared": ("every arena's active cars and ball after each timed step of the end-to-end pass, and every "
                         "arena's cars, ball, env and pads after the device-timed pass, bitwise (NaN payloads aside)")
            if mixed else "every arena's ball and env after the device-timed pass, bitwise",
            "mismatched_arenas": int((bad_steps | bad_final).sum())}


# ---- serving: many clients through rg_server ----------------------------------------------------------------------
SERVE_CLIENTS = 64
SERVE_BUDGET = 60 * 1024 ** 3


def serve_clients(seed: int, k: int):
    """Client k's arenas: log-uniform count in [64, 1024], 55/27/18 mix, first half of each arena's cars blue."""
    rng = np.random.default_rng(seed * 1000 + k)
    n = int(np.exp(rng.uniform(np.log(64), np.log(1024))))
    counts = rng.choice(np.array([2, 4, 6], np.int32), size=n, p=[0.55, 0.27, 0.18]).astype(np.int32)
    teams = np.zeros(n * MAX_CARS, np.uint8)
    for e in range(n):
        teams[e * MAX_CARS + counts[e] // 2: e * MAX_CARS + counts[e]] = 1
    return counts, teams


def run_serve_policy(srv_policy, rate, seconds, seed, v, i):
    """Poisson step requests (ticks in {1, 4, 8}) at `rate` per second spread over the clients, 1 % of clients closed
    and reopened per second; returns throughput and latency percentiles."""
    from tests import scenarios
    from rocketgpu_b200.server import Busy, Server
    specs = [serve_clients(seed, k) for k in range(SERVE_CLIENTS)]
    cap = int(sum(len(c) for c, _ in specs) * 1.3)
    srv = Server(v, i, max_arenas=cap, hbm_budget_bytes=SERVE_BUDGET, policy=srv_policy, max_cars_per_env=MAX_CARS)
    rng = np.random.default_rng(seed)
    clients = []
    for k, (counts, teams) in enumerate(specs):
        clients.append([srv.open_client(counts, teams, kickoff_seed=seed + k), len(counts), 0])
    ctrl_cache = {}

    def controls(n, ticks):
        key = (n, ticks)
        if key not in ctrl_cache:
            st = scenarios.ControlStream(n * MAX_CARS, seed=n * 10 + ticks, p_jump=0.1, hold_max=30)
            ctrl_cache[key] = np.stack([st.next() for _ in range(ticks)])
        return ctrl_cache[key]

    outstanding = []
    lat, done_ticks, refused = [], 0, 0
    t_start = time.perf_counter()
    next_arrival = t_start + rng.exponential(1.0 / rate)
    next_churn = t_start + rng.exponential(1.0 / (0.01 * SERVE_CLIENTS))
    reopened = 0
    while True:
        now = time.perf_counter()
        if now - t_start >= seconds:
            break
        while next_arrival <= now:
            c = clients[rng.integers(0, SERVE_CLIENTS)]
            ticks = int(rng.choice([1, 4, 8]))
            outstanding.append((srv.submit(c[0], controls(c[1], ticks)), c[1] * ticks))
            next_arrival += rng.exponential(1.0 / rate)
        if next_churn <= now:
            k = int(rng.integers(0, SERVE_CLIENTS))
            counts, teams = serve_clients(seed + 7919 + reopened, k)
            # closing waits for the client's admitted request and drops its queued ones (polling those then reports
            # an unknown request, below)
            srv.close_client(clients[k][0])
            try:
                clients[k] = [srv.open_client(counts, teams, kickoff_seed=reopened), len(counts), 0]
            except Busy:
                refused += 1
                clients[k] = [srv.open_client(specs[k][0], specs[k][1], kickoff_seed=reopened), len(specs[k][0]), 0]
            reopened += 1
            next_churn += rng.exponential(1.0 / (0.01 * SERVE_CLIENTS))
        keep = []
        for req, work in outstanding:
            try:
                res = srv.poll(req)
            except IndexError:
                continue  # its client was closed before it ran
            if res is None:
                keep.append((req, work))
            else:
                lat.append(res[0])
                done_ticks += work
        outstanding = keep
        time.sleep(0.0002)
    elapsed = time.perf_counter() - t_start
    stats = srv.stats()
    srv.close()
    lat_ms = np.array(lat) * 1e3 if lat else np.array([float("nan")])
    return {"policy": srv_policy, "offered_req_per_s": rate, "completed": len(lat),
            "throughput_arena_ticks_per_s": done_ticks / elapsed,
            "p50_ms": float(np.percentile(lat_ms, 50)), "p99_ms": float(np.percentile(lat_ms, 99)),
            "p999_ms": float(np.percentile(lat_ms, 99.9)), "rounds": stats["rounds"],
            "device_busy_frac": stats["busy_s"] / elapsed, "pool_slots": stats["capacity"],
            "slot_bytes": stats["slot_bytes"], "clients_reopened": reopened, "reopen_refused": refused}


def run_serve(args, world, rank, local):
    import torch

    from rocketgpu_b200 import arena
    torch.cuda.set_device(local)
    v, i = arena.generate()
    out = {}
    for policy in ("static", "continuous"):
        out[policy] = run_serve_policy(policy, args.rate, args.serve_seconds, 11 + rank, v, i)
    cont = out["continuous"]
    return {
        "metric": METRIC, "value": cont["throughput_arena_ticks_per_s"] * world, "unit": "arena-ticks/s",
        "n_gpus": world, "steps": 0, "warmup": 0, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded clients, Poisson step requests)",
        "config": {"workload": f"serving: {SERVE_CLIENTS} clients x log-uniform 64..1024 arenas (55/27/18), Poisson "
                               f"requests at {args.rate:g}/s with ticks in {{1,4,8}}, 1%/s client churn, "
                               f"{SERVE_BUDGET / 1024 ** 3:.0f} GiB HBM budget, {args.serve_seconds:g} s per policy"},
        "serving": out,
        "gpu_launches": None,
    }


def run_reference(args, world, rank):
    if rank != 0:
        return None
    cb, _ = cpu_leg(args.workload, args.warmup, args.steps, parity=False)
    line = {
        "impl": "reference", "metric": METRIC, "value": cb["value"], "unit": "arena-ticks/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32",
        "data": "synthetic (seeded arenas, bodies, controls and episode resets)" if args.workload == "mixed"
        else "synthetic (seeded ball states)",
        "config": {"workload": WORKLOADS[args.workload], "arenas_per_gpu": ENVS, "ticks_per_step": TICKS_PER_STEP,
                   "settle_steps": SETTLE_STEPS if args.workload == "mixed" else 0,
                   **({"events_per_arena": EVENTS} if EVENTS else {})},
        "cpu_baseline": cb,
        "e2e": {"value": cb["value"], "unit": "arena-ticks/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    return line


def run_reference_cuda(args, world, rank):
    """The reference's own CUDA build of the path (oracle/_ref/librg_oracle_cuda.so: src/rocketgpu_cuda.cu and the host
    sources compiled here for sm_100 with ROCKETGPU_USE_CUDA) on the same workload, stepped through its BatchSim with
    device-resident controls and commands: the plain GPU bar. Each step is timed host-side with a device
    synchronisation on both sides (the reference launches on its own streams); the episode clock's commands are made
    between steps, outside the timed region, as in the CPU leg."""
    import torch
    if rank != 0:
        return None
    from rocketgpu_b200 import arena
    from tests import oracle_ref, scenarios
    path = os.path.join(ROOT, "oracle", "_ref", "librg_oracle_cuda.so")
    if not os.path.exists(path):
        return {"impl": "reference", "unavailable": "oracle/_ref/librg_oracle_cuda.so not built (make -C oracle cuda)"}
    oracle_ref.LIB_PATH = path
    oracle_ref._lib = None
    v, i = arena.generate()
    w = MixedWorkload(0)
    sim = oracle_ref.OracleSim(ENVS, MAX_CARS, v, i, kickoff_settled=False)
    sim.set_env_car_count(w.counts)
    sim.set_teams(w.teams)
    sim.set_car_configs(w.car_configs(_presets()))
    sim.reset_to_kickoff(w.reset_seed)
    clock = scenarios.EpisodeClock(sim.envs(), sim.cars(), MAX_CARS, NO_TOUCH_TICKS, w.stagger_seed)
    cmds = np.zeros((TICKS_PER_STEP * ENVS, CMD_BYTES), np.uint8)
    ctrl_dev = torch.empty(TICKS_PER_STEP * ENVS * MAX_CARS * CTRL_BYTES, dtype=torch.uint8, device="cuda")
    cmd_dev = torch.empty(TICKS_PER_STEP * ENVS * CMD_BYTES, dtype=torch.uint8, device="cuda")
    flush = torch.empty(256 << 20, dtype=torch.uint8, device="cuda")
    gen = w.controls()
    step_s = []
    for k in range(SETTLE_STEPS + args.warmup + args.steps):
        timed = k >= SETTLE_STEPS + args.warmup
        ctrl_dev.copy_(torch.from_numpy(next(gen).reshape(-1)))
        cmd_dev.copy_(torch.from_numpy(cmds.reshape(-1)))
        flush.zero_()
        torch.cuda.synchronize()
        if timed:
            torch.cuda.nvtx.range_push("timed")
        t0 = time.perf_counter()
        sim.step_with_device_commands(ctrl_dev.data_ptr(), ENVS * MAX_CARS, cmd_dev.data_ptr(), ENVS, TICKS_PER_STEP)
        torch.cuda.synchronize()
        dt = time.perf_counter() - t0
        if timed:
            torch.cuda.nvtx.range_pop()
            step_s.append(dt)
        cmds[:ENVS] = clock.commands(sim.envs(), sim.cars(), w.counts)
    final = (_active_car_rows(sim.cars(), w.counts), sim.balls())
    sim.close()
    value = ENVS * TICKS_PER_STEP * len(step_s) / sum(step_s)
    ms = sorted(1e3 * s for s in step_s)
    return {
        "impl": "reference", "backend": "cuda", "metric": METRIC, "value": value, "unit": "arena-ticks/s",
        "n_gpus": 1, "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * sum(step_s) / len(step_s),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic (seeded arenas, bodies, controls and episode resets)",
        "config": {"workload": WORKLOADS["mixed"], "arenas_per_gpu": ENVS, "ticks_per_step": TICKS_PER_STEP,
                   "settle_steps": SETTLE_STEPS, "l2": "256 MiB flush before every timed step"},
        "latency_ms_per_step": {"p50": ms[len(ms) // 2], "p99": ms[min(len(ms) - 1, int(0.99 * len(ms)))]},
        "final_state_sha": hashlib.sha256(final[0].tobytes() + final[1].tobytes()).hexdigest()[:16],
    }


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--ref-backend", default="cpu", choices=["cpu", "cuda"],
                    help="reference arm: its CPU BatchSim (default) or its own CUDA build (the plain GPU bar)")
    ap.add_argument("--workload", default="mixed", choices=sorted(WORKLOADS))
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--events", type=int, default=0,
                    help="physics event stream on, this many records per arena (mixed workload; 0: off)")
    ap.add_argument("--arenas", type=int, default=ENVS, help="arenas per GPU (smaller cases for profiling)")
    ap.add_argument("--rate", type=float, default=1000.0, help="serving: offered step requests per second")
    ap.add_argument("--serve-seconds", type=float, default=10.0, help="serving: seconds per policy")
    args = ap.parse_args()
    globals()["EVENTS"] = args.events
    if args.arenas != ENVS:
        globals()["ENVS"] = args.arenas
        for k in WORKLOADS:
            WORKLOADS[k] = WORKLOADS[k].replace("16384 arenas", f"{args.arenas} arenas")
    if args.warmup < 3:
        args.warmup = 3
    if args.impl == "reference":
        world = int(os.environ.get("WORLD_SIZE", "1"))
        rank = int(os.environ.get("RANK", "0"))
        line = run_reference_cuda(args, world, rank) if args.ref_backend == "cuda" else run_reference(args, world, rank)
    else:
        world, rank, local = dist_setup(args.gpus)
        line = run_serve(args, world, rank, local) if args.workload == "serve" else run_ours(args, world, rank, local)
        if world > 1:
            import torch.distributed as dist
            dist.destroy_process_group()
    if line is not None and int(os.environ.get("RANK", "0")) == 0:
        print(json.dumps(line), flush=True)


if __name__ == "__main__":
    main()
