"""Generates the golden fixtures under tests/golden/ by running the oracle (the reference's own CPU BatchSim, built
by oracle/Makefile) on the seeded scenarios of tests/scenarios.py.

    make -C oracle && python tests/golden/make_golden.py

Each fixture stores the uploaded inputs and the oracle's full ball / env struct bytes after every tick.
"""
from __future__ import annotations

import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from rocketgpu_b200 import arena  # noqa: E402
from tests import oracle_ref, scenarios  # noqa: E402


def run_ball_case(name: str, states_fn, n: int, seed: int, ticks: int):
    v, i = arena.generate()
    sim = oracle_ref.OracleSim(n, 2, v, i, kickoff_settled=False)
    sim.set_env_car_count([0] * n)
    _, default_ball, _, _, _ = oracle_ref.default_states()
    init = states_fn(default_ball, n, seed)
    sim.upload_balls(init)
    env0 = sim.envs()
    balls, envs = [], []
    for _ in range(ticks):
        sim.step(1)
        balls.append(sim.balls())
        envs.append(sim.envs())
    np.savez_compressed(os.path.join(HERE, name + ".npz"), init_balls=init, init_envs=env0,
                        balls=np.stack(balls), envs=np.stack(envs), seed=seed)
    print(name, n, "arenas", ticks, "ticks")


if __name__ == "__main__":
    run_ball_case("ball_free_flight", scenarios.free_flight_states, 8, 1234, 60)
    run_ball_case("ball_contacts", scenarios.ball_states, 8, 4321, 200)
