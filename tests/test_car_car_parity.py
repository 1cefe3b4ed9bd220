"""GPU parity of arenas with several cars: contacts between cars (the box/box contact points, the retained pair
manifold, the pair rows in the unified solves), bumps, demolitions and respawns, against the oracle (the reference's
CPU BatchSim) on the same seeded inputs, compared bitwise (0 ulp) on every active car's 880-byte state, the ball, the
env and the arena's 34 pads after every tick or launch. No arena leaves the comparison; the only allowance is a NaN
word's payload (tests/parity.py).
"""
import numpy as np
import pytest

from tests import oracle_ref, parity, scenarios

pytestmark = pytest.mark.gpu
MC = 6


def _arenas(n, seed):
    rng = np.random.default_rng(seed)
    counts = rng.choice(np.array([2, 4, 6], np.int32), size=n, p=[0.4, 0.3, 0.3]).astype(np.int32)
    teams = np.zeros(n * MC, np.uint8)
    for e in range(n):
        teams[e * MC + counts[e] // 2: e * MC + counts[e]] = 1
    return counts, teams


def _pair(n, arena_mesh, counts, teams, seed):
    from rocketgpu_b200.batch_sim import BatchSim, SimConfig
    v, i = arena_mesh
    orc = oracle_ref.OracleSim(n, MC, v, i, kickoff_settled=False)
    gpu = BatchSim(SimConfig(env_count=n, max_cars_per_env=MC, kickoff_settled=0), v, i)
    for sim in (orc, gpu):
        sim.set_env_car_count(counts)
        sim.set_teams(teams)
        sim.reset_to_kickoff(seed)
    gpu.synchronize()
    return orc, gpu


def _compare(orc, gpu, counts):
    n = len(counts)
    oc, gc = orc.cars(), gpu.download_car_states()
    ob, gb = orc.balls(), gpu.download_ball_states()
    oe, ge = orc.envs(), gpu.download_env_states()
    op, gp = orc.pads().reshape(n, -1), gpu.download_boost_pad_states().reshape(n, -1)
    for e in range(n):
        d = parity.first_mismatch((("cars", oc[e * MC: e * MC + counts[e]], gc[e * MC: e * MC + counts[e]]),
                                   ("ball", ob[e], gb[e]), ("env", oe[e], ge[e]), ("pads", op[e], gp[e])),
                                  {"cars": 880})
        if d:
            return f"arena {e} ({counts[e]} cars) {d}"
    return None


OFF_BUMP_BUMPS, OFF_BUMP_DEMOS, OFF_IS_DEMOED = 412, 419, 135  # CarState.bump_event_bumps / _demos, is_demoed


def _events(cars, counts):
    """(bumps, demolitions) the active cars' bump-event counters hold, and how many cars are demolished now."""
    act = np.concatenate([np.arange(e * MC, e * MC + counts[e]) for e in range(len(counts))])
    c = cars[act]
    return (int(c[:, OFF_BUMP_BUMPS:OFF_BUMP_BUMPS + 7].astype(np.int64).sum()),
            int(c[:, OFF_BUMP_DEMOS:OFF_BUMP_DEMOS + 7].astype(np.int64).sum()), int(c[:, OFF_IS_DEMOED].sum()))


@pytest.mark.parametrize("seed", [21, 22])
def test_kickoff_chase_with_car_contacts(oracle_available, arena_mesh, seed):
    """Every car chases the ball from kickoff with boost: cars meet at the ball and bump, push and demolish each
    other, demolished cars respawn after three seconds; compared after every tick."""
    import torch
    n, k, launches = 96, 8, 70
    counts, teams = _arenas(n, seed)
    orc, gpu = _pair(n, arena_mesh, counts, teams, seed)
    rng = np.random.default_rng(seed + 500)
    bumps = demos = 0
    for launch in range(launches):
        b, dm, _ = _events(orc.cars(), counts)
        bumps, demos = max(bumps, b), max(demos, dm)
        ctrl = scenarios.chase_ball_controls(orc.cars(), orc.balls(), MC, rng, p_jump=0.03)
        dev = torch.from_numpy(ctrl).cuda()
        for t in range(k):  # one tick per step: every tick is compared
            orc.step_with_controls(ctrl, 1, 0)
            gpu.step_with_device_controls(dev.data_ptr(), 1, 0)
            gpu.synchronize()
            d = _compare(orc, gpu, counts)
            assert d is None, f"launch {launch} tick {t}: {d} (bumps so far {bumps}, demolitions {demos})"
    assert bumps > 0 and demos > 0, (bumps, demos)
    print(f"bump events {bumps}, demolition events {demos}, every arena compared every tick")


def test_mixed_random_controls(oracle_available, arena_mesh):
    """The benchmark's workload at small scale: mixed 1v1/2v2/3v3 arenas from kickoff with the seeded held random
    controls (jumps, boost, handbrake, air control), 400 ticks in launches of 8 with per-tick control blocks."""
    import torch
    n, k, launches = 64, 8, 50
    counts, teams = _arenas(n, 31)
    orc, gpu = _pair(n, arena_mesh, counts, teams, 31)
    stream = scenarios.ControlStream(n * MC, seed=131, p_jump=0.1, hold_max=30)
    for launch in range(launches):
        block = np.stack([stream.next() for _ in range(k)]).reshape(-1, 24)
        orc.step_with_controls(block, k, n * MC)
        dev = torch.from_numpy(block.copy()).cuda()
        gpu.step_with_device_controls(dev.data_ptr(), k, n * MC)
        gpu.synchronize()
        d = _compare(orc, gpu, counts)
        assert d is None, f"launch {launch}: {d}"


def test_one_arena_1v1_1200_ticks(oracle_available, arena_mesh):
    """The CPU-runnable workload: one 1v1 arena (default car body) from kickoff for 1,200 ticks at 120 Hz, each car's
    seeded controls (axes U[-1, 1], jump / boost / handbrake Bernoulli 0.1 / 0.3 / 0.1) held U{1..30} ticks, compared
    after every tick."""
    import torch
    from rocketgpu_b200.batch_sim import BatchSim, SimConfig
    v, i = arena_mesh
    orc = oracle_ref.OracleSim(1, 2, v, i, kickoff_settled=False)
    gpu = BatchSim(SimConfig(env_count=1, max_cars_per_env=2, kickoff_settled=0), v, i)
    for sim in (orc, gpu):
        sim.set_env_car_count([2])
        sim.set_teams(np.array([0, 1], np.uint8))
        sim.reset_to_kickoff(1200)
    gpu.synchronize()
    stream = scenarios.ControlStream(2, seed=1201, p_jump=0.1, hold_max=30)
    ctrl_dev = torch.zeros((2, 24), dtype=torch.uint8, device="cuda")
    for t in range(1200):
        ctrl = stream.next()
        orc.step_with_controls(ctrl, 1, 0)
        ctrl_dev.copy_(torch.from_numpy(ctrl))
        gpu.step_with_device_controls(ctrl_dev.data_ptr(), 1, 0)
        gpu.synchronize()
        d = _compare(orc, gpu, np.array([2]))
        assert d is None, f"tick {t}: {d}"


def test_six_hitbox_presets(oracle_available, arena_mesh):
    """Car bodies drawn uniformly from the six hitbox presets (Octane, Dominus, Plank, Breakout, Hybrid, Merc) in
    mixed 1v1 / 2v2 / 3v3 arenas where every car chases the ball: different boxes, wheel offsets, wheel radii and
    suspension rests in the wheel rays, the car/mesh and car/car contacts and the bumps; compared after every tick."""
    import torch
    n, k, launches = 64, 8, 50
    counts, teams = _arenas(n, 41)
    rng = np.random.default_rng(41)
    bodies = rng.integers(0, 6, n * MC)
    cfgs = np.stack([oracle_ref.car_preset(int(p)) for p in bodies])
    from rocketgpu_b200.batch_sim import BatchSim, SimConfig
    v, i = arena_mesh
    orc = oracle_ref.OracleSim(n, MC, v, i, kickoff_settled=False)
    gpu = BatchSim(SimConfig(env_count=n, max_cars_per_env=MC, kickoff_settled=0), v, i)
    for sim in (orc, gpu):
        sim.set_env_car_count(counts)
        sim.set_teams(teams)
        sim.set_car_configs(cfgs)
        sim.reset_to_kickoff(41)
    gpu.synchronize()
    assert len(set(bodies.tolist())) == 6
    crng = np.random.default_rng(541)
    for launch in range(launches):
        ctrl = scenarios.chase_ball_controls(orc.cars(), orc.balls(), MC, crng, p_jump=0.03)
        dev = torch.from_numpy(ctrl).cuda()
        for t in range(k):
            orc.step_with_controls(ctrl, 1, 0)
            gpu.step_with_device_controls(dev.data_ptr(), 1, 0)
            gpu.synchronize()
            d = _compare(orc, gpu, counts)
            assert d is None, f"launch {launch} tick {t}: {d}"


OFF_RESPAWN_OVERRIDE = 138  # CarState.respawn_slot_override_plus1


def test_respawn_spot_picks_1600_ticks(oracle_available, arena_mesh):
    """Long chase with the six hitbox presets, so demolished cars come back many times: each one's respawn spot is
    picked a tick ahead, walking the arena's spot order and the eight moved spots around each, clear of the other cars
    (where they are, or where they come back, by their bodies' mesh bounds) and of the ball; 1,600 ticks compared after
    every tick, the picks counted."""
    import torch
    from rocketgpu_b200.batch_sim import BatchSim, SimConfig
    n, k, launches = 96, 8, 200
    counts, teams = _arenas(n, 23)
    rng = np.random.default_rng(30)
    cfgs = np.stack([oracle_ref.car_preset(int(p)) for p in rng.integers(0, 6, n * MC)])
    v, i = arena_mesh
    orc = oracle_ref.OracleSim(n, MC, v, i, kickoff_settled=False)
    gpu = BatchSim(SimConfig(env_count=n, max_cars_per_env=MC, kickoff_settled=0), v, i)
    for sim in (orc, gpu):
        sim.set_env_car_count(counts)
        sim.set_teams(teams)
        sim.set_car_configs(cfgs)
        sim.reset_to_kickoff(23)
    gpu.synchronize()
    act = np.concatenate([np.arange(e * MC, e * MC + counts[e]) for e in range(n)])
    crng = np.random.default_rng(523)
    prev = np.zeros(len(act), np.uint8)
    picks = moved = 0
    for launch in range(launches):
        ctrl = scenarios.chase_ball_controls(orc.cars(), orc.balls(), MC, crng, p_jump=0.03)
        dev = torch.from_numpy(ctrl).cuda()
        for t in range(k):
            orc.step_with_controls(ctrl, 1, 0)
            gpu.step_with_device_controls(dev.data_ptr(), 1, 0)
            gpu.synchronize()
            d = _compare(orc, gpu, counts)
            assert d is None, f"launch {launch} tick {t}: {d} ({picks} respawn picks so far)"
            cur = orc.cars()[act, OFF_RESPAWN_OVERRIDE]
            new = (prev == 0) & (cur != 0)
            picks += int(new.sum())
            moved += int((new & (cur >= 128)).sum())
            prev = cur.copy()
    assert picks > 10, picks
    print(f"{picks} respawn spot picks, {moved} of them moved off a taken spot")
