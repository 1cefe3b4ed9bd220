"""GPU parity of the car path: the CUDA tick against the oracle (the reference's CPU BatchSim) on the same seeded car
states and control streams, compared bitwise (0 ulp) on the full 880-byte car struct, the ball, the env and the 34
boost pads of every arena.

Scope of this build: cars in the air and on their wheels (controls, jumps, dodges, boost, air control, suspension,
tyre friction, sticky force, pads), the car body's contacts with the arena mesh (landings on the roof or a side,
wall hits) with the broadphase manifold list that orders the solver, and car-ball contacts (the retained car-ball
manifold, the two-body rows in the unified solve, the ball-hit records and the game's extra hit impulse). These
scenarios run one car per arena; arenas with several cars are covered by test_car_car_parity.py.
"""
import numpy as np
import pytest

from tests import oracle_ref, parity, scenarios

pytestmark = pytest.mark.gpu
MC = 2  # car slots per arena; one car per arena is active
PADS = 34
OFF_LAST_BALL_CONTACT = 440  # CarState.last_ball_contact_start (u64, ~0 until the car first touches the ball)


def _pair(n, arena_mesh, cars_init):
    from rocketgpu_b200.batch_sim import BatchSim, SimConfig
    v, i = arena_mesh
    orc = oracle_ref.OracleSim(n, MC, v, i, kickoff_settled=False)
    orc.set_env_car_count([1] * n)
    gpu = BatchSim(SimConfig(env_count=n, max_cars_per_env=MC, kickoff_settled=0), v, i)
    gpu.set_env_car_count([1] * n)
    cars = orc.cars().copy()
    cars[0::MC] = cars_init
    orc.upload_cars(cars)
    gpu.upload_car_states(cars)
    return orc, gpu


def _touched_ball(cars):
    return cars[0::MC, OFF_LAST_BALL_CONTACT:OFF_LAST_BALL_CONTACT + 8].copy().view(np.uint64).ravel() != np.uint64(~0 & (2**64 - 1))


def _compare(orc, gpu, n):
    oc, gc = orc.cars(), gpu.download_car_states()
    ob, gb = orc.balls(), gpu.download_ball_states()
    oe, ge = orc.envs(), gpu.download_env_states()
    op, gp = orc.pads().reshape(n, -1), gpu.download_boost_pad_states().reshape(n, -1)
    for e in range(n):
        d = parity.first_mismatch((("car", oc[MC * e], gc[MC * e]), ("ball", ob[e], gb[e]), ("env", oe[e], ge[e]),
                                   ("pads", op[e], gp[e])))
        if d:
            return f"arena {e} {d}"
    return None


def test_car_upload_canonicalization_matches(oracle_available, arena_mesh):
    n = 128
    car0, _, _, _, _ = oracle_ref.default_states()
    init = np.concatenate([scenarios.airborne_cars(car0, n // 2, seed=1), scenarios.grounded_cars(car0, n // 2, seed=2)])
    orc, gpu = _pair(n, arena_mesh, init)
    oc, gc = orc.cars(), gpu.download_car_states()
    assert (oc == gc).all(), np.nonzero((oc != gc).any(1))[0][:8]


def test_airborne_cars_every_tick(oracle_available, arena_mesh):
    import torch
    n = 256
    car0, _, _, _, _ = oracle_ref.default_states()
    orc, gpu = _pair(n, arena_mesh, scenarios.airborne_cars(car0, n, seed=3))
    stream = scenarios.ControlStream(n * MC, seed=103, p_jump=0.1)
    for t in range(60):
        ctrl = stream.next()
        orc.step_with_controls(ctrl, 1, 0)
        dev = torch.from_numpy(ctrl).cuda()
        gpu.step_with_device_controls(dev.data_ptr(), 1, 0)
        gpu.synchronize()
        d = _compare(orc, gpu, n)
        assert d is None, f"tick {t}: {d}"


@pytest.mark.parametrize("seed", [2, 5])
def test_grounded_cars_multi_tick_launches(oracle_available, arena_mesh, seed):
    """Cars driving on the floor, stepped in launches of 8 ticks with a per-tick control block (stride = capacity)."""
    import torch
    n, k, launches = 256, 8, 30
    car0, _, _, _, _ = oracle_ref.default_states()
    orc, gpu = _pair(n, arena_mesh, scenarios.grounded_cars(car0, n, seed=seed))
    stream = scenarios.ControlStream(n * MC, seed=seed + 100, p_jump=0.05, hold_max=20)
    for launch in range(launches):
        block = np.stack([stream.next() for _ in range(k)])  # [k, capacity, 24]
        orc.step_with_controls(block.reshape(-1, 24), k, n * MC)
        dev = torch.from_numpy(block.reshape(-1, 24).copy()).cuda()
        gpu.step_with_device_controls(dev.data_ptr(), k, n * MC)
        gpu.synchronize()
        d = _compare(orc, gpu, n)
        assert d is None, f"launch {launch}: {d}"


def test_cars_landing_on_the_arena(oracle_available, arena_mesh):
    """Cars dropped from 300 uu in random orientations land on wheels, roof or side; the body's mesh contacts,
    their retained manifold and the unified solve must match every tick."""
    import torch
    n, ticks = 128, 360
    car0, _, _, _, _ = oracle_ref.default_states()
    orc, gpu = _pair(n, arena_mesh, scenarios.airborne_cars(car0, n, seed=7, z=300.0))
    stream = scenarios.ControlStream(n * MC, seed=107, p_jump=0.05, hold_max=10)
    for t in range(ticks):
        ctrl = stream.next()
        orc.step_with_controls(ctrl, 1, 0)
        dev = torch.from_numpy(ctrl).cuda()
        gpu.step_with_device_controls(dev.data_ptr(), 1, 0)
        gpu.synchronize()
        d = _compare(orc, gpu, n)
        assert d is None, f"tick {t}: {d}"


def test_kickoff_reset_matches(oracle_available, arena_mesh):
    """reset_to_kickoff with seeded team layouts: every car at its team's kickoff spot, ball, pads and env bookkeeping."""
    from rocketgpu_b200.batch_sim import BatchSim, SimConfig
    v, i = arena_mesh
    n, mc = 64, 6
    orc = oracle_ref.OracleSim(n, mc, v, i, kickoff_settled=False)
    gpu = BatchSim(SimConfig(env_count=n, max_cars_per_env=mc, kickoff_settled=0), v, i)
    for what, a, b in (("ball", orc.balls(), gpu.download_ball_states()), ("env", orc.envs(), gpu.download_env_states()),
                       ("pads", orc.pads(), gpu.download_boost_pad_states())):
        assert (a == b).all(), f"after create: {what}"
    rng = np.random.default_rng(7)
    counts = rng.integers(1, mc + 1, n).astype(np.int32)
    teams = rng.integers(0, 2, n * mc).astype(np.uint8)
    for sim in (orc, gpu):
        sim.set_env_car_count(counts)
        sim.set_teams(teams)
    active = np.concatenate([np.arange(e * mc, e * mc + counts[e]) for e in range(n)])
    for seed in (0, 0, 987654321):
        orc.reset_to_kickoff(seed)
        gpu.reset_to_kickoff(seed)
        gpu.synchronize()
        assert (orc.cars()[active] == gpu.download_car_states()[active]).all(), seed
        assert (orc.balls() == gpu.download_ball_states()).all(), seed
        assert (orc.envs() == gpu.download_env_states()).all(), seed
        assert (orc.pads() == gpu.download_boost_pad_states()).all(), seed


@pytest.mark.parametrize("seed", [11, 12])
def test_kickoff_ball_chase(oracle_available, arena_mesh, seed):
    """reset_to_kickoff, then each arena's car chases the ball with boost (steering toward it, rare jumps, air-control
    noise), in launches of 8 ticks with controls chosen from the state at each launch's start: first touches,
    repeated hits, dribbles and aerial touches (car-ball manifold, two-body rows, hit records, the extra hit impulse)
    must match every launch, and nearly every car must reach the ball."""
    import torch
    from rocketgpu_b200.batch_sim import BatchSim, SimConfig
    v, i = arena_mesh
    n, k, launches = 96, 8, 70
    orc = oracle_ref.OracleSim(n, MC, v, i, kickoff_settled=False)
    gpu = BatchSim(SimConfig(env_count=n, max_cars_per_env=MC, kickoff_settled=0), v, i)
    teams = np.random.default_rng(seed).integers(0, 2, n * MC).astype(np.uint8)
    for sim in (orc, gpu):
        sim.set_env_car_count([1] * n)
        sim.set_teams(teams)
        sim.reset_to_kickoff(seed)
    gpu.synchronize()
    rng = np.random.default_rng(seed + 300)
    for launch in range(launches):
        ctrl = scenarios.chase_ball_controls(orc.cars(), orc.balls(), MC, rng, p_jump=0.05)
        orc.step_with_controls(ctrl, k, 0)
        dev = torch.from_numpy(ctrl).cuda()
        gpu.step_with_device_controls(dev.data_ptr(), k, 0)
        gpu.synchronize()
        d = _compare(orc, gpu, n)
        assert d is None, f"launch {launch}: {d}"
    assert _touched_ball(orc.cars()).mean() >= 0.8, _touched_ball(orc.cars()).mean()
