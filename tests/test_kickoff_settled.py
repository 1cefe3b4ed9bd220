"""GPU parity of settled kickoffs (kickoff_settled = 1, the reference's default: MutatorConfig::kickoff_settled,
rocketgpu.h:831; recorded by record_kickoff_settled, src/rocketgpu.cpp:1538-1612, applied by SettleKickoffCar and
ResetKickoffBall, arena_ball.hpp:2756-2767, 2959-2975) against the oracle with the same flag: the batch as created,
kickoffs after new car configs and teams, play from the settled state, and env-command resets with and without a
countdown (a countdown kickoff is never settled), compared bitwise on every active car, ball, env and pad."""
import numpy as np
import pytest

from tests import oracle_ref, parity, scenarios

pytestmark = pytest.mark.gpu
MC = 6


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


def test_settled_kickoffs_through_play_and_commands(oracle_available, arena_mesh):
    import torch
    from rocketgpu_b200.batch_sim import BatchSim, SimConfig
    v, i = arena_mesh
    n, k = 64, 8
    orc = oracle_ref.OracleSim(n, MC, v, i, kickoff_settled=True)
    gpu = BatchSim(SimConfig(env_count=n, max_cars_per_env=MC), v, i)  # kickoff_settled defaults to 1
    assert gpu.config.c.kickoff_settled == 1
    zero = np.zeros(n, np.int32)
    d = _compare(orc, gpu, zero)  # created and reset with no cars: the settled ball
    assert d is None, f"after create: {d}"
    rng = np.random.default_rng(5)
    counts = rng.choice(np.array([2, 4, 6], np.int32), size=n, p=[0.4, 0.3, 0.3]).astype(np.int32)
    teams = np.zeros(n * MC, np.uint8)
    for e in range(n):
        teams[e * MC + counts[e] // 2: e * MC + counts[e]] = 1
    cfgs = np.stack([oracle_ref.car_preset(int(p)) for p in rng.integers(0, 6, n * MC)])
    for sim in (orc, gpu):
        sim.set_env_car_count(counts)
        sim.set_teams(teams)
        sim.set_car_configs(cfgs)
        sim.reset_to_kickoff(17)
    gpu.synchronize()
    d = _compare(orc, gpu, counts)
    assert d is None, f"after the settled kickoff: {d}"
    crng = np.random.default_rng(6)
    for rnd in range(3):
        for step in range(25):
            ctrl = scenarios.chase_ball_controls(orc.cars(), orc.balls(), MC, crng, p_jump=0.03)
            dev_ctrl = torch.from_numpy(ctrl).cuda()
            cm = np.zeros((k, n, 16), np.uint8)
            if step == 12:  # resets inside a launch: half plain (settled), half with a countdown (not settled)
                cm[3, :, 0] = 1
                cm[3, 1::2, 6:8] = np.full(n // 2, 480, np.uint16).view(np.uint8).reshape(-1, 2)
            dev_cmds = torch.from_numpy(cm.reshape(-1, 16).copy()).cuda()
            orc.step_with_commands(ctrl, 0, cm.reshape(-1, 16), n, k)
            gpu.step_with_device_commands(dev_ctrl.data_ptr(), 0, dev_cmds.data_ptr(), n, k)
            gpu.synchronize()
            d = _compare(orc, gpu, counts)
            assert d is None, f"round {rnd} step {step}: {d}"
        # new bodies and swapped teams between rounds: new entries are recorded before the next reset
        cfgs = np.stack([oracle_ref.car_preset(int(p)) for p in rng.integers(0, 6, n * MC)])
        teams = 1 - teams if rnd == 0 else teams
        cmds = np.zeros((n, 16), np.uint8)
        cmds[:, 0] = 1
        cmds[:, 1] = rng.random(n) < 0.5
        cmds[:, 3] = rng.choice([0, 3], n)
        for sim in (orc, gpu):
            sim.set_car_configs(cfgs)
            sim.set_teams(teams)
            sim.apply_env_commands(cmds)
        gpu.synchronize()
        d = _compare(orc, gpu, counts)
        assert d is None, f"round {rnd} after commands: {d}"
