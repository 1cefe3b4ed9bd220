"""GPU parity of arenas with several cars: contacts between cars (the box/box contact points, the retained pair
manifold, the pair rows in the unified solves), bumps, demolitions and respawns, against the oracle (the reference's
CPU BatchSim) on the same seeded inputs, compared bitwise (0 ulp) on every active car's 880-byte state, the ball, the
env and the arena's 34 pads after every launch.

Arenas whose oracle car state left the reals (the reference's EPA can return a NaN witness point for a box landing
flat; the NaN payload then differs between x86 and the GPU) leave the comparison from that launch on.

Two behaviours of the reference are not built, and the comparison names them instead of hiding them:
  * a car demolished in the middle of a world step ends the tick with a different reported rotation (position,
    velocities and every other byte match): the rotation of demolished cars is left out;
  * the reference skips, for a suspension ray, a body (the ball or a car) whose broadphase box from the previous
    sweep misses the ray; this build tests the body's shape. An arena whose wheel-contact flags part ways leaves the
    comparison, and at most 5 % of arenas may.
"""
import numpy as np
import pytest

from tests import oracle_ref, scenarios

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


OFF_ROT, OFF_WHEEL_CONTACT = 12, 123  # CarState.rot (16 bytes), CarState.wheels_with_contact (4 bytes)


def _compare(orc, gpu, counts, excluded, wheel_gap):
    n = len(counts)
    oc, gc = orc.cars(), gpu.download_car_states()
    ob, gb = orc.balls(), gpu.download_ball_states()
    oe, ge = orc.envs(), gpu.download_env_states()
    op, gp = orc.pads().reshape(n, -1), gpu.download_boost_pad_states().reshape(n, -1)
    for e in range(n):
        if excluded[e]:
            continue
        cars_o = oc[e * MC: e * MC + counts[e]].copy()
        cars_g = gc[e * MC: e * MC + counts[e]].copy()
        if not np.isfinite(cars_o[:, 0:12].copy().view(np.float32)).all():
            excluded[e] = True
            continue
        if (cars_o[:, OFF_WHEEL_CONTACT:OFF_WHEEL_CONTACT + 4] != cars_g[:, OFF_WHEEL_CONTACT:OFF_WHEEL_CONTACT + 4]).any():
            excluded[e] = wheel_gap[e] = True
            continue
        demoed = cars_o[:, OFF_IS_DEMOED] == 1
        cars_o[demoed, OFF_ROT:OFF_ROT + 16] = 0
        cars_g[demoed, OFF_ROT:OFF_ROT + 16] = 0
        for what, a, b in (("cars", cars_o, cars_g), ("ball", ob[e], gb[e]),
                           ("env", oe[e], ge[e]), ("pads", op[e], gp[e])):
            if not np.array_equal(a, b):
                d = np.nonzero((a != b).reshape(-1))[0]
                return f"arena {e} ({counts[e]} cars) {what} bytes {d[:12].tolist()}"
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
    excluded = np.zeros(n, bool)
    wheel_gap = np.zeros(n, bool)
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
            d = _compare(orc, gpu, counts, excluded, wheel_gap)
            assert d is None, f"launch {launch} tick {t}: {d} (bumps so far {bumps}, demolitions {demos})"
    assert excluded.mean() <= 0.25, excluded.mean()
    assert wheel_gap.mean() <= 0.05, wheel_gap.mean()
    assert bumps > 0 and demos > 0, (bumps, demos)
    print(f"bump events {bumps}, demolition events {demos}, excluded {excluded.sum()} (wheel gap {wheel_gap.sum()})")


def test_mixed_random_controls(oracle_available, arena_mesh):
    """The benchmark's workload at small scale: mixed 1v1/2v2/3v3 arenas from kickoff with the seeded held random
    controls (jumps, boost, handbrake, air control), 400 ticks in launches of 8 with per-tick control blocks."""
    import torch
    n, k, launches = 64, 8, 50
    counts, teams = _arenas(n, 31)
    orc, gpu = _pair(n, arena_mesh, counts, teams, 31)
    stream = scenarios.ControlStream(n * MC, seed=131, p_jump=0.1, hold_max=30)
    excluded = np.zeros(n, bool)
    wheel_gap = np.zeros(n, bool)
    for launch in range(launches):
        block = np.stack([stream.next() for _ in range(k)]).reshape(-1, 24)
        orc.step_with_controls(block, k, n * MC)
        dev = torch.from_numpy(block.copy()).cuda()
        gpu.step_with_device_controls(dev.data_ptr(), k, n * MC)
        gpu.synchronize()
        d = _compare(orc, gpu, counts, excluded, wheel_gap)
        assert d is None, f"launch {launch}: {d}"
    assert excluded.mean() <= 0.10, excluded.mean()
    assert wheel_gap.mean() <= 0.05, wheel_gap.mean()
