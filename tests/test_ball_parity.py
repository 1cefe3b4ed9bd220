"""GPU parity: the CUDA tick against the oracle (the reference's CPU BatchSim) on the same seeded inputs, compared
bitwise (0 ulp) on the full 288-byte ball struct and 44-byte env struct after every tick."""
import os

import numpy as np
import pytest

from tests import oracle_ref, scenarios

HERE = os.path.dirname(os.path.abspath(__file__))
pytestmark = pytest.mark.gpu


def _pair(n, arena_mesh):
    from rocketgpu_b200.batch_sim import BatchSim, SimConfig
    v, i = arena_mesh
    orc = oracle_ref.OracleSim(n, 2, v, i, kickoff_settled=False)
    orc.set_env_car_count([0] * n)
    gpu = BatchSim(SimConfig(kickoff_settled=0, env_count=n, max_cars_per_env=2), v, i)
    gpu.set_env_car_count([0] * n)
    return orc, gpu


def _first_diff(a, b):
    rows = np.nonzero((a != b).any(1))[0]
    if len(rows) == 0:
        return None
    r = rows[0]
    return int(r), np.nonzero(a[r] != b[r])[0][:16].tolist()


def test_upload_canonicalization_matches(oracle_available, arena_mesh):
    n = 256
    orc, gpu = _pair(n, arena_mesh)
    _, default_ball, _, _, _ = oracle_ref.default_states()
    init = scenarios.ball_states(default_ball, n, seed=5)
    orc.upload_balls(init)
    gpu.upload_ball_states(init)
    assert _first_diff(orc.balls(), gpu.download_ball_states()) is None


def test_free_flight_parity_every_tick(oracle_available, arena_mesh):
    n = 512
    orc, gpu = _pair(n, arena_mesh)
    _, default_ball, _, _, _ = oracle_ref.default_states()
    init = scenarios.free_flight_states(default_ball, n, seed=11)
    orc.upload_balls(init)
    gpu.upload_ball_states(init)
    gpu.upload_env_states(orc.envs())
    for t in range(60):
        orc.step(1)
        gpu.step(1)
        d = _first_diff(orc.balls(), gpu.download_ball_states())
        assert d is None, f"tick {t}: ball {d}"
        d = _first_diff(orc.envs(), gpu.download_env_states())
        assert d is None, f"tick {t}: env {d}"


def test_multi_tick_launch_equals_single_ticks(oracle_available, arena_mesh):
    n = 128
    orc, gpu = _pair(n, arena_mesh)
    _, default_ball, _, _, _ = oracle_ref.default_states()
    init = scenarios.free_flight_states(default_ball, n, seed=3)
    orc.upload_balls(init)
    gpu.upload_ball_states(init)
    gpu.upload_env_states(orc.envs())
    for _ in range(6):
        orc.step(8)
        gpu.step(8)
        assert _first_diff(orc.balls(), gpu.download_ball_states()) is None
        assert _first_diff(orc.envs(), gpu.download_env_states()) is None


def test_golden_free_flight(arena_mesh):
    from rocketgpu_b200.batch_sim import BatchSim, SimConfig
    g = np.load(os.path.join(HERE, "golden", "ball_free_flight.npz"))
    v, i = arena_mesh
    n = g["init_balls"].shape[0]
    gpu = BatchSim(SimConfig(kickoff_settled=0, env_count=n, max_cars_per_env=2), v, i)
    gpu.set_env_car_count([0] * n)
    gpu.upload_ball_states(g["init_balls"])
    gpu.upload_env_states(g["init_envs"])
    for t in range(g["balls"].shape[0]):
        gpu.step(1)
        assert bytes(gpu.download_ball_states()) == bytes(g["balls"][t]), t
        assert bytes(gpu.download_env_states()) == bytes(g["envs"][t]), t


def test_contact_heavy_parity_every_tick(oracle_available, arena_mesh):
    """Balls thrown at up to 6000 uu/s: bounces, rolling, corner and edge contacts, predictive (CCD) contacts."""
    n = 1024
    orc, gpu = _pair(n, arena_mesh)
    _, default_ball, _, _, _ = oracle_ref.default_states()
    init = scenarios.ball_states(default_ball, n, seed=21)
    orc.upload_balls(init)
    gpu.upload_ball_states(init)
    gpu.upload_env_states(orc.envs())
    for t in range(600):
        orc.step(1)
        gpu.step(1)
        d = _first_diff(orc.balls(), gpu.download_ball_states())
        assert d is None, f"tick {t}: ball {d}"
        d = _first_diff(orc.envs(), gpu.download_env_states())
        assert d is None, f"tick {t}: env {d}"


def test_contact_heavy_multi_tick_launches(oracle_available, arena_mesh):
    n = 2048
    orc, gpu = _pair(n, arena_mesh)
    _, default_ball, _, _, _ = oracle_ref.default_states()
    init = scenarios.ball_states(default_ball, n, seed=22)
    orc.upload_balls(init)
    gpu.upload_ball_states(init)
    gpu.upload_env_states(orc.envs())
    for k in range(100):
        orc.step(8)
        gpu.step(8)
        d = _first_diff(orc.balls(), gpu.download_ball_states())
        assert d is None, f"launch {k}: ball {d}"
        d = _first_diff(orc.envs(), gpu.download_env_states())
        assert d is None, f"launch {k}: env {d}"


def test_golden_contacts(arena_mesh):
    from rocketgpu_b200.batch_sim import BatchSim, SimConfig
    g = np.load(os.path.join(HERE, "golden", "ball_contacts.npz"))
    v, i = arena_mesh
    n = g["init_balls"].shape[0]
    gpu = BatchSim(SimConfig(kickoff_settled=0, env_count=n, max_cars_per_env=2), v, i)
    gpu.set_env_car_count([0] * n)
    gpu.upload_ball_states(g["init_balls"])
    gpu.upload_env_states(g["init_envs"])
    for t in range(g["balls"].shape[0]):
        gpu.step(1)
        assert bytes(gpu.download_ball_states()) == bytes(g["balls"][t]), t
        assert bytes(gpu.download_env_states()) == bytes(g["envs"][t]), t
