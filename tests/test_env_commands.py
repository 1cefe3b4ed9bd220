"""GPU parity of env commands against the oracle (the reference's CPU BatchSim), compared bitwise (0 ulp, NaN
payloads aside) on every active car, ball, env and pad:

  * apply_env_commands between steps with every field combination the build runs (kickoff reset with and without the
    scoreboard, tick counter, the four kickoff seed modes, explicit and zero seeds, new-round bodies alone, kept pads);
  * step_with_device_commands with commands on random ticks inside each launch;
  * the mixed 55 % 1v1 / 27 % 2v2 / 18 % 3v3 workload with goal / 300-tick no-touch resets for 2,000 ticks: the
    device's rg_batch_episode_commands against its host statement (tests/scenarios.EpisodeClock) on the oracle.
"""
import numpy as np
import pytest

from tests import oracle_ref, parity, scenarios

pytestmark = pytest.mark.gpu
MC = 6


def _arenas(n, seed, p=(0.4, 0.3, 0.3)):
    rng = np.random.default_rng(seed)
    counts = rng.choice(np.array([2, 4, 6], np.int32), size=n, p=list(p)).astype(np.int32)
    teams = np.zeros(n * MC, np.uint8)
    for e in range(n):
        teams[e * MC + counts[e] // 2: e * MC + counts[e]] = 1
    return counts, teams


def _pair(n, arena_mesh, counts, teams, seed):
    from rocketgpu_b200.batch_sim import BatchSim, SimConfig
    v, i = arena_mesh
    orc = oracle_ref.OracleSim(n, MC, v, i, kickoff_settled=False)
    gpu = BatchSim(SimConfig(kickoff_settled=0, env_count=n, max_cars_per_env=MC), v, i)
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


def _random_commands(rng, n):
    cmds = np.zeros((n, 16), np.uint8)
    cmds[:, 0] = rng.random(n) < 0.7
    cmds[:, 1] = rng.random(n) < 0.5
    cmds[:, 2] = rng.random(n) < 0.5
    cmds[:, 3] = rng.choice([0, 0, 1, 2, 3], n)
    cmds[:, 4] = rng.random(n) < 0.3
    cmds[:, 5] = rng.random(n) < 0.3
    seeds = np.where(rng.random(n) < 0.5, 0, rng.integers(1, 2**62, n)).astype(np.uint64)
    cmds[:, 8:16] = seeds.view(np.uint8).reshape(n, 8)
    return cmds


def test_apply_env_commands_between_steps(oracle_available, arena_mesh):
    import torch
    n = 96
    counts, teams = _arenas(n, 61)
    orc, gpu = _pair(n, arena_mesh, counts, teams, 61)
    rng = np.random.default_rng(61)
    crng = np.random.default_rng(62)
    for rnd in range(12):
        for t in range(40):
            ctrl = scenarios.chase_ball_controls(orc.cars(), orc.balls(), MC, crng, p_jump=0.03)
            orc.step_with_controls(ctrl, 1, 0)
            gpu.step_with_device_controls(torch.from_numpy(ctrl).cuda().data_ptr(), 1, 0)
            gpu.synchronize()
        d = _compare(orc, gpu, counts)
        assert d is None, f"round {rnd} before commands: {d}"
        cmds = _random_commands(rng, n)
        orc.apply_env_commands(cmds)
        if rnd % 2:
            gpu.apply_env_commands(cmds)
        else:
            dev = torch.from_numpy(cmds).cuda()
            gpu.apply_env_commands_device(dev.data_ptr(), n)
            gpu.synchronize()
        d = _compare(orc, gpu, counts)
        assert d is None, f"round {rnd} after commands: {d}"


def test_step_with_device_commands(oracle_available, arena_mesh):
    import torch
    n, k, steps = 96, 8, 60
    counts, teams = _arenas(n, 71)
    orc, gpu = _pair(n, arena_mesh, counts, teams, 71)
    rng = np.random.default_rng(71)
    crng = np.random.default_rng(72)
    for step in range(steps):
        ctrl = scenarios.chase_ball_controls(orc.cars(), orc.balls(), MC, crng, p_jump=0.03)
        cmds = np.zeros((k, n, 16), np.uint8)
        sel = np.nonzero(rng.random(n) < 0.08)[0]
        cmds[rng.integers(0, k, len(sel)), sel] = _random_commands(rng, len(sel))
        cmds[:, :, 6:8] = 0
        orc.step_with_commands(ctrl, 0, cmds.reshape(-1, 16), n, k)
        # both device buffers stay referenced until the step has run (a temporary's memory could be handed to the
        # next allocation before the stream reads it)
        dev_ctrl = torch.from_numpy(ctrl).cuda()
        dev_cmds = torch.from_numpy(cmds.reshape(-1, 16).copy()).cuda()
        gpu.step_with_device_commands(dev_ctrl.data_ptr(), 0, dev_cmds.data_ptr(), n, k)
        gpu.synchronize()
        d = _compare(orc, gpu, counts)
        assert d is None, f"step {step}: {d}"


def test_goal_and_no_touch_resets_2000_ticks(oracle_available, arena_mesh):
    """The batched workload with episode resets: 1,024 arenas mixed 55/27/18, seeded held random controls, a reset on a
    goal or after 300 ticks without a touch (staggered clocks), 2,000 ticks in launches of 8 with every launch
    compared; the device's reset decisions must equal the host statement's."""
    import torch
    n, k, steps = 1024, 8, 250
    counts, teams = _arenas(n, 81, p=(0.55, 0.27, 0.18))
    orc, gpu = _pair(n, arena_mesh, counts, teams, 81)
    clock = scenarios.EpisodeClock(orc.envs(), orc.cars(), MC, 300, stagger_seed=81)
    dev_cmds = torch.zeros((k, n, 16), dtype=torch.uint8, device="cuda")
    gpu.episode_commands(300, dev_cmds.data_ptr(), stagger_seed=81, init=True)
    host_cmds = np.zeros((k, n, 16), np.uint8)
    stream = scenarios.ControlStream(n * MC, seed=181, p_jump=0.1, hold_max=30)
    ctrl_dev = torch.zeros((k * n * MC, 24), dtype=torch.uint8, device="cuda")
    resets = 0
    for step in range(steps):
        block = np.stack([stream.next() for _ in range(k)]).reshape(-1, 24)
        ctrl_dev.copy_(torch.from_numpy(block))
        orc.step_with_commands(block, n * MC, host_cmds.reshape(-1, 16), n, k)
        gpu.step_with_device_commands(ctrl_dev.data_ptr(), n * MC, dev_cmds.data_ptr(), n, k)
        gpu.synchronize()
        d = _compare(orc, gpu, counts)
        assert d is None, f"step {step}: {d} (resets so far {resets})"
        host_cmds[:] = 0
        host_cmds[0] = clock.commands(orc.envs(), orc.cars(), counts)
        dev_cmds.zero_()
        gpu.episode_commands(300, dev_cmds.data_ptr())
        gpu.synchronize()
        assert np.array_equal(dev_cmds[0].cpu().numpy(), host_cmds[0]), f"step {step}: reset decisions differ"
        resets += int(host_cmds[0, :, 0].sum())
    assert resets > n, resets  # about one reset per arena per 300-400 ticks
    print(f"{resets} episode resets over {steps * k} ticks of {n} arenas")


def test_countdown_kickoffs(oracle_available, arena_mesh):
    """Countdown kickoffs (kickoff_countdown_ticks: 480 ticks, and 0xFFFF, until the game's countdown timers end it):
    cars wait a tick and a half then appear at their spots, driving stays off, the ball drops from the game's height;
    between steps (host and device arrays) and inside launches, through the end of the countdown."""
    import torch
    n, k = 48, 8
    counts, teams = _arenas(n, 91)
    orc, gpu = _pair(n, arena_mesh, counts, teams, 91)
    rng = np.random.default_rng(91)
    crng = np.random.default_rng(92)
    for rnd in range(3):
        cmds = np.zeros((n, 16), np.uint8)
        sel = rng.random(n) < 0.6
        cmds[sel, 0] = 1
        cmds[sel, 1] = rng.random(sel.sum()) < 0.5
        ticks = np.where(rng.random(n) < 0.5, 480, 0xFFFF).astype(np.uint16)
        cmds[:, 6:8] = ticks.view(np.uint8).reshape(n, 2)
        cmds[:, 3] = rng.choice([0, 3], n)
        orc.apply_env_commands(cmds)
        if rnd == 1:
            dev = torch.from_numpy(cmds).cuda()
            gpu.apply_env_commands_device(dev.data_ptr(), n)
        else:
            gpu.apply_env_commands(cmds)
        gpu.synchronize()
        d = _compare(orc, gpu, counts)
        assert d is None, f"round {rnd} after commands: {d}"
        for step in range(70):  # 560 ticks: past the countdown's end
            ctrl = scenarios.chase_ball_controls(orc.cars(), orc.balls(), MC, crng, p_jump=0.05)
            cm = np.zeros((k, n, 16), np.uint8)
            if rnd == 2 and step == 3:  # a countdown kickoff inside a launch
                cm[5, :, 0] = 1
                cm[5, :, 6:8] = np.full(n, 480, np.uint16).view(np.uint8).reshape(n, 2)
            dev_ctrl = torch.from_numpy(ctrl).cuda()
            dev_cmds = torch.from_numpy(cm.reshape(-1, 16).copy()).cuda()
            orc.step_with_commands(ctrl, 0, cm.reshape(-1, 16), n, k)
            gpu.step_with_device_commands(dev_ctrl.data_ptr(), 0, dev_cmds.data_ptr(), n, k)
            gpu.synchronize()
            d = _compare(orc, gpu, counts)
            assert d is None, f"round {rnd} step {step}: {d}"
