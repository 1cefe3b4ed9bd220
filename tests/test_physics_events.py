"""Physics events (reference PhysicsEventStream, rocketgpu.h:44-98, set_physics_event_stream rocketgpu.h:1015): the
device stream against the oracle's (the reference's CPU BatchSim writing the same records into host arrays) on the same
seeded inputs: every window (tick, count, overflow) and every record field compared bitwise (padding aside), in order,
after every launch; ball touches, ball-world and car-world contacts, boost pickups, bumps and demolitions, goals; the
goal-only filter and a full window's overflow flag."""
import ctypes

import numpy as np
import pytest

from tests import oracle_ref, scenarios

MC = 6


def _dtypes():
    from rocketgpu_b200.batch_sim import PHYSICS_EVENT_DTYPE, PHYSICS_EVENT_WINDOW_DTYPE
    return PHYSICS_EVENT_DTYPE, PHYSICS_EVENT_WINDOW_DTYPE


def test_event_layout_matches_the_reference(oracle_available):
    ev, win = _dtypes()
    out = np.zeros(4, np.int64)
    oracle_ref.lib().orc_physics_event_sizes(out.ctypes.data_as(ctypes.c_void_p))
    assert out.tolist() == [ev.itemsize, win.itemsize, ev.fields["position"][1], ev.fields["boost_after"][1]]


def _field_bits(rec):
    """Each field of the records as raw integers (floats by their bits), padding left out."""
    out = {}
    for name in rec.dtype.names:
        a = rec[name]
        if a.dtype.kind == "f":
            a = np.ascontiguousarray(a).view(np.uint32)
        out[name] = a
    return out


def _compare_events(orc_events, gpu_records, gpu_windows, n, cap):
    ev, win = _dtypes()
    ow = orc_events[1].view(win)
    gw = gpu_windows.cpu().numpy().view(win)
    for name in ("tick", "count", "overflow"):
        bad = np.nonzero(ow[name] != gw[name])[0]
        assert len(bad) == 0, f"window {name} differs in arena {bad[0]}: oracle {ow[bad[0]]} device {gw[bad[0]]}"
    orec = orc_events[0].view(ev).reshape(n, cap)
    grec = gpu_records.cpu().numpy().view(ev).reshape(n, cap)
    types = np.zeros(6, np.int64)
    for e in range(n):
        k = int(ow["count"][e])
        if k == 0:
            continue
        a, b = _field_bits(orec[e, :k]), _field_bits(grec[e, :k])
        for name in a:
            diff = np.nonzero(np.any((a[name] != b[name]).reshape(k, -1), axis=1))[0]
            assert len(diff) == 0, (f"arena {e} event {diff[0]} of {k} field {name}: oracle {orec[e, diff[0]]} "
                                    f"device {grec[e, diff[0]]}")
        types += np.bincount(orec[e, :k]["type"], minlength=6)[:6]
    return types


def _clear(orc_events, gpu_windows):
    _, win = _dtypes()
    orc_events[1].view(win)["count"] = 0
    orc_events[1].view(win)["overflow"] = 0
    gpu_windows.zero_()  # tick is rewritten by the next tick


def _run(arena_mesh, n, ticks_per_launch, launches, cap, seed, goal_only=False, rules=None, pads=None):
    import torch
    from rocketgpu_b200.batch_sim import BatchSim, SimConfig
    v, i = arena_mesh
    rng = np.random.default_rng(seed)
    counts = rng.choice(np.array([2, 4, 6], np.int32), size=n, p=[0.4, 0.3, 0.3]).astype(np.int32)
    teams = np.zeros(n * MC, np.uint8)
    for e in range(n):
        teams[e * MC + counts[e] // 2: e * MC + counts[e]] = 1
    cfgs = np.stack([oracle_ref.car_preset(int(p)) for p in rng.integers(0, 6, n * MC)])
    kw = {}
    if rules is not None:
        from tests.test_arena_rules import _rules_floats
        kw = {"rules": _rules_floats(rules), "pad_layout": np.array(pads, np.float32)}
    orc = oracle_ref.OracleSim(n, MC, v, i, kickoff_settled=False, **kw)
    gpu = BatchSim(SimConfig(kickoff_settled=0, env_count=n, max_cars_per_env=MC), v, i, rules=rules, boost_pads=pads)
    for sim in (orc, gpu):
        sim.set_env_car_count(counts)
        sim.set_teams(teams)
        sim.set_car_configs(cfgs)
        sim.reset_to_kickoff(seed)
    orc_events = orc.set_physics_event_stream(cap, goal_only)
    records = torch.zeros(n * cap * 104, dtype=torch.uint8, device="cuda")
    windows = torch.zeros(n * 16, dtype=torch.uint8, device="cuda")
    gpu.set_physics_event_stream(records.data_ptr(), windows.data_ptr(), cap, goal_only)
    clock = scenarios.EpisodeClock(orc.envs(), orc.cars(), MC, 400)
    crng = np.random.default_rng(seed + 1)
    cmds = np.zeros((ticks_per_launch, n, 16), np.uint8)
    types = np.zeros(6, np.int64)
    overflows = 0
    for launch in range(launches):
        ctrl = scenarios.chase_ball_controls(orc.cars(), orc.balls(), MC, crng, p_jump=0.04)
        dev_ctrl = torch.from_numpy(ctrl).cuda()
        dev_cmds = torch.from_numpy(cmds.reshape(-1, 16).copy()).cuda()
        orc.step_with_commands(ctrl, 0, cmds.reshape(-1, 16), n, ticks_per_launch)
        gpu.step_with_device_commands(dev_ctrl.data_ptr(), 0, dev_cmds.data_ptr(), n, ticks_per_launch)
        gpu.synchronize()
        types += _compare_events(orc_events, records, windows, n, cap)
        overflows += int(orc_events[1].view(_dtypes()[1])["overflow"].sum())
        _clear(orc_events, windows)
        cmds[:] = 0
        cmds[0] = clock.commands(orc.envs(), orc.cars(), counts)
    gpu.set_physics_event_stream(0, 0, 0)
    gpu.synchronize()
    return types, overflows


@pytest.mark.gpu
def test_events_match_the_reference_through_play(oracle_available, arena_mesh):
    types, overflows = _run(arena_mesh, n=64, ticks_per_launch=4, launches=90, cap=512, seed=41)
    print("events by type", dict(zip(("touch", "ball-world", "car-world", "pickup", "bump", "goal"), types.tolist())))
    assert overflows == 0
    assert types[0] > 0 and types[1] > 0 and types[2] > 0 and types[3] > 0 and types[4] > 0, types


@pytest.mark.gpu
def test_goal_events_and_goal_only_and_overflow(oracle_available, arena_mesh):
    from tests.test_arena_rules import _pads, _rules
    types, _ = _run(arena_mesh, n=48, ticks_per_launch=8, launches=60, cap=512, seed=43, rules=_rules(),
                    pads=_pads(3))
    assert types[5] > 0, types  # goals (the moved goal line is just past the ball spawn)
    types, _ = _run(arena_mesh, n=48, ticks_per_launch=8, launches=40, cap=4, seed=44, goal_only=True,
                    rules=_rules(), pads=_pads(3))
    assert types[5] > 0 and types[:5].sum() == 0, types
    _, overflows = _run(arena_mesh, n=32, ticks_per_launch=8, launches=10, cap=3, seed=45)
    assert overflows > 0
