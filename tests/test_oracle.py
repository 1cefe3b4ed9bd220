"""The oracle (the reference's own CPU BatchSim, oracle/_ref) against the committed golden fixtures, and the
synthetic arena generator's determinism. CPU only."""
import hashlib
import os

import numpy as np

from tests import oracle_ref, scenarios

HERE = os.path.dirname(os.path.abspath(__file__))


def test_arena_mesh_is_deterministic(arena_mesh):
    v, i = arena_mesh
    assert v.dtype == np.float32 and i.dtype == np.int32
    assert 9000 <= len(i) // 3 <= 12000
    h = hashlib.sha256(v.tobytes() + i.tobytes()).hexdigest()
    from rocketgpu_b200 import arena
    v2, i2 = arena.generate()
    assert hashlib.sha256(v2.tobytes() + i2.tobytes()).hexdigest() == h


def test_oracle_reproduces_golden_free_flight(oracle_available, arena_mesh):
    g = np.load(os.path.join(HERE, "golden", "ball_free_flight.npz"))
    v, i = arena_mesh
    n = g["init_balls"].shape[0]
    sim = oracle_ref.OracleSim(n, 2, v, i, kickoff_settled=False)
    sim.set_env_car_count([0] * n)
    _, default_ball, _, _, _ = oracle_ref.default_states()
    init = scenarios.free_flight_states(default_ball, n, int(g["seed"]))
    assert bytes(init) == bytes(g["init_balls"])
    sim.upload_balls(init)
    for t in range(g["balls"].shape[0]):
        sim.step(1)
        assert bytes(sim.balls()) == bytes(g["balls"][t]), t
        assert bytes(sim.envs()) == bytes(g["envs"][t]), t
