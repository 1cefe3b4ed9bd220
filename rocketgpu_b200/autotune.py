"""Launch autotuner: picks threads per block for the per-arena and per-car kernels and whether steps replay CUDA
graphs, by timing the caller's own step on the caller's batch.

Results never depend on the launch config (each arena and each car is one thread whatever the block size, and a
graph replays exactly the launches it captured), so the tuner may time candidates on consecutive steps of a live
batch; run it once the workload is in steady state.
"""
from __future__ import annotations

import ctypes
import itertools

import numpy as np

from . import abi
from .batch_sim import _check

ARENA_THREADS = (32, 64, 128)
CAR_THREADS = (32, 64, 128, 256)


def get_config(sim) -> dict:
    c = abi.rg_launch_config()
    _check(abi.lib().rg_batch_get_launch_config(sim._h, ctypes.byref(c)))
    return {"arena_threads": c.arena_threads, "car_threads": c.car_threads, "use_graphs": bool(c.use_graphs)}


def set_config(sim, arena_threads: int, car_threads: int, use_graphs: bool):
    c = abi.rg_launch_config(arena_threads, car_threads, int(use_graphs), 0)
    _check(abi.lib().rg_batch_set_launch_config(sim._h, ctypes.byref(c)))


def autotune(sim, step, steps: int = 3, graphs=(False, True), arena_threads=ARENA_THREADS, car_threads=CAR_THREADS):
    """`step()` runs one step of the caller's workload on `sim` (on torch's current stream). Each candidate gets one
    untimed step (a graph capture, when graphs are on) and `steps` steps timed with CUDA events; the fastest median
    wins and is left set. Returns (best config, [(config, median ms)])."""
    import torch
    stream = torch.cuda.current_stream()
    results = []
    for at, ct, g in itertools.product(arena_threads, car_threads, graphs):
        set_config(sim, at, ct, g)
        step()
        ms = []
        for _ in range(steps):
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record(stream)
            step()
            b.record(stream)
            b.synchronize()
            ms.append(a.elapsed_time(b))
        results.append(({"arena_threads": at, "car_threads": ct, "use_graphs": g}, float(np.median(ms))))
    best = min(results, key=lambda r: r[1])[0]
    set_config(sim, best["arena_threads"], best["car_threads"], best["use_graphs"])
    return best, results
