"""A custom ArenaLayout's rules and pads (reference ArenaLayout goals / kickoff_spawns / respawn_spawns / ball_spawn /
boost_pads, rocketgpu.h:943-959; ArenaRules, detail/constants.hpp:57-67): moved goals with bounded mouths, moved and
turned kickoff and respawn spots, a moved ball spawn and a layout of its own pads, against the oracle built from the
same layout, compared bitwise on every active car, ball, env and pad after every tick, through goal and no-touch
resets, bumps, demolitions and respawns. GPU tests, except the validation one."""
import numpy as np
import pytest

from tests import oracle_ref, parity, scenarios

MC = 6


def _rules():
    from rocketgpu_b200.batch_sim import arena_rules
    r = arena_rules()
    for t, sign in ((0, -1.0), (1, 1.0)):
        g = r.goals[t]
        g.point.y = -4700.0 if t == 0 else 200.0  # orange's goal line just past the ball spawn: goals come often
        g.normal.x, g.normal.y, g.normal.z = 0.05 * sign, 2.0 * sign, 0.0  # normalized by the layout
        g.min.x, g.min.z = -3000.0, -1.0e30
        g.max.x, g.max.z = 3000.0, 900.0
        for k in range(5):
            s = r.kickoff_spawns[t][k]
            s.pos.x += 96.0 * (k - 2)
            s.pos.y -= sign * 180.0
            s.yaw += 0.125 * (k + 1)
        for k in range(4):
            s = r.respawn_spawns[t][k]
            s.pos.x *= 0.75
            s.pos.y -= sign * 300.0
            s.pos.z = 40.0
            s.yaw -= 0.3
    r.ball_spawn.y, r.ball_spawn.z = 256.0, 140.0
    return r


def _rules_floats(r):
    import ctypes
    return np.frombuffer(ctypes.string_at(ctypes.addressof(r), ctypes.sizeof(r)), np.float32).copy()


def _pads(seed):
    rng = np.random.default_rng(seed)
    pads = []
    for k in range(22):
        x, y = rng.uniform(-3500, 3500), rng.uniform(-4400, 4400)
        big = 1 if k % 5 == 0 else 0
        pads.append((float(np.float32(x)), float(np.float32(y)), 73.0 if big else 70.0, big))
    return pads


def test_layout_rules_and_pads_are_validated_before_any_device_call(arena_mesh):
    from rocketgpu_b200.batch_sim import BatchSim, SimConfig, arena_rules
    v, i = arena_mesh
    r = arena_rules()
    r.kickoff_spawns[0][1].yaw = 30.0  # beyond 8 pi
    with pytest.raises(ValueError, match="yaw"):
        BatchSim(SimConfig(kickoff_settled=0, env_count=2), v, i, rules=r)
    r = arena_rules()
    r.goals[1].min.y = float("nan")
    with pytest.raises(ValueError, match="NaN"):
        BatchSim(SimConfig(kickoff_settled=0, env_count=2), v, i, rules=r)
    r = arena_rules()
    r.ball_spawn.x = 12000.0
    with pytest.raises(ValueError, match="ball spawn"):
        BatchSim(SimConfig(kickoff_settled=0, env_count=2), v, i, rules=r)
    with pytest.raises(ValueError, match="kMaxBoostPads"):
        BatchSim(SimConfig(kickoff_settled=0, env_count=2), v, i, boost_pads=[(0.0, 0.0, 70.0, 0)] * 49)
    with pytest.raises(ValueError, match="boost pad position"):
        BatchSim(SimConfig(kickoff_settled=0, env_count=2), v, i, boost_pads=[(0.0, float("inf"), 70.0, 0)])


def _run(arena_mesh, rules, pads, n, ticks, seed):
    import torch
    from rocketgpu_b200.batch_sim import BatchSim, SimConfig
    v, i = arena_mesh
    rng = np.random.default_rng(seed)
    counts = rng.choice(np.array([2, 4, 6], np.int32), size=n, p=[0.4, 0.3, 0.3]).astype(np.int32)
    teams = np.zeros(n * MC, np.uint8)
    for e in range(n):
        teams[e * MC + counts[e] // 2: e * MC + counts[e]] = 1
    orc = oracle_ref.OracleSim(n, MC, v, i, kickoff_settled=False,
                               rules=None if rules is None else _rules_floats(rules),
                               pad_layout=None if pads is None else np.array(pads, np.float32))
    gpu = BatchSim(SimConfig(kickoff_settled=0, env_count=n, max_cars_per_env=MC), v, i, rules=rules, boost_pads=pads)
    assert gpu.pad_capacity() == orc.pad_capacity
    for sim in (orc, gpu):
        sim.set_env_car_count(counts)
        sim.set_teams(teams)
        sim.reset_to_kickoff(seed)
    gpu.synchronize()
    clock = scenarios.EpisodeClock(orc.envs(), orc.cars(), MC, 600)
    crng = np.random.default_rng(seed + 1)
    cmds = np.zeros((n, 16), np.uint8)
    goals = resets = 0
    per = orc.pad_capacity // n
    for t in range(ticks):
        if t % 8 == 0:
            ctrl = scenarios.chase_ball_controls(orc.cars(), orc.balls(), MC, crng, p_jump=0.04)
            dev_ctrl = torch.from_numpy(ctrl).cuda()
        dev_cmds = torch.from_numpy(cmds.copy()).cuda()
        orc.step_with_commands(ctrl, 0, cmds, n, 1)
        gpu.step_with_device_commands(dev_ctrl.data_ptr(), 0, dev_cmds.data_ptr(), n, 1)
        gpu.synchronize()
        oc, gc = orc.cars(), gpu.download_car_states()
        ob, gb = orc.balls(), gpu.download_ball_states()
        oe, ge = orc.envs(), gpu.download_env_states()
        op, gp = orc.pads().reshape(n, per, -1), gpu.download_boost_pad_states().reshape(n, per, -1)
        for e in range(n):
            d = parity.first_mismatch((("cars", oc[e * MC: e * MC + counts[e]], gc[e * MC: e * MC + counts[e]]),
                                       ("ball", ob[e], gb[e]), ("env", oe[e], ge[e]), ("pads", op[e], gp[e])),
                                      {"cars": 880})
            assert d is None, f"tick {t} arena {e} ({counts[e]} cars) {d}"
        score = oe[:, scenarios.ENV_BLUE:scenarios.ENV_BLUE + 4].copy().view(np.uint32).ravel() | \
            oe[:, scenarios.ENV_ORANGE:scenarios.ENV_ORANGE + 4].copy().view(np.uint32).ravel()
        goals += int((score != 0).sum())
        cmds = clock.commands(oe, oc, counts)
        resets += int(cmds[:, 0].sum())
    return goals, resets


@pytest.mark.gpu
def test_custom_goals_spawns_ball_spawn_and_pads(oracle_available, arena_mesh):
    goals, resets = _run(arena_mesh, _rules(), _pads(3), n=64, ticks=900, seed=31)
    assert resets > 20 and goals > 0, (goals, resets)


@pytest.mark.gpu
def test_official_rules_given_explicitly_behave_as_none(oracle_available, arena_mesh):
    from rocketgpu_b200.batch_sim import arena_rules
    _run(arena_mesh, arena_rules(), None, n=32, ticks=240, seed=32)
