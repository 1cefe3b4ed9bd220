"""The state-array boundary of the reference's Python binding: arrays by name (upload_state_array /
download_state_array, PublicState and PreserveInternal uploads) and zero-copy device_arrays, checked against the
oracle and against the typed calls. GPU tests."""
import ctypes

import numpy as np
import pytest

from tests import oracle_ref, parity, scenarios

pytestmark = pytest.mark.gpu
MC = 2


class _Bytes:
    """A uint8 view of one device_arrays entry, for torch.as_tensor."""

    def __init__(self, entry):
        cai = entry["__cuda_array_interface__"]
        self.__cuda_array_interface__ = {"data": cai["data"], "shape": (entry["count"] * entry["itemsize"],),
                                         "typestr": "|u1", "strides": None, "version": 3}


def test_state_arrays_by_name_and_device_arrays(oracle_available, arena_mesh):
    import torch
    from rocketgpu_b200.batch_sim import BatchSim, SimConfig
    v, i = arena_mesh
    n = 64
    orc = oracle_ref.OracleSim(n, MC, v, i, kickoff_settled=False)
    gpu = BatchSim(SimConfig(kickoff_settled=0, env_count=n, max_cars_per_env=MC), v, i)
    for sim in (orc, gpu):
        sim.set_env_car_count([2] * n)
        sim.set_teams(np.tile(np.array([0, 1], np.uint8), n))
        sim.reset_to_kickoff(5)
    gpu.synchronize()
    crng = np.random.default_rng(5)
    for _ in range(40):
        ctrl = scenarios.chase_ball_controls(orc.cars(), orc.balls(), MC, crng)
        orc.step_with_controls(ctrl, 1, 0)
        gpu.step_with_device_controls(torch.from_numpy(ctrl).cuda().data_ptr(), 1, 0)
    gpu.synchronize()
    # by name == typed
    for name, typed, size, count in (("car_states", gpu.download_car_states, 880, n * MC),
                                     ("ball_states", gpu.download_ball_states, 288, n),
                                     ("env_states", gpu.download_env_states, 44, n),
                                     ("boost_pad_states", gpu.download_boost_pad_states, 16, n * 34)):
        buf = np.zeros((count, size), np.uint8)
        gpu.download_state_array(name, buf.ctypes.data, count)
        assert np.array_equal(buf, typed()), name
    with pytest.raises(ValueError):
        gpu.download_state_array("solver_scratch", buf.ctypes.data, 1)
    # zero-copy views see the same bytes
    arrays = gpu.device_arrays()
    for name, typed in (("car_states", gpu.download_car_states), ("ball_states", gpu.download_ball_states),
                        ("env_states", gpu.download_env_states)):
        t = torch.as_tensor(_Bytes(arrays[name]), device="cuda")
        assert np.array_equal(t.cpu().numpy().reshape(typed().shape), typed()), name
    assert arrays["car_states"]["per_env"] == MC and arrays["boost_pad_states"]["per_env"] == 34
    # PreserveInternal: raw states in, then stepping matches the oracle fed the same raw states
    cars = orc.cars()
    cars[:, 28:40] = (cars[:, 28:40].copy().view(np.float32) * np.float32(1.5)).view(np.uint8)  # velocities
    balls = orc.balls()
    for preserve in (True, False):
        orc.upload_cars(cars, preserve_internal=preserve)
        orc.upload_balls(balls, preserve_internal=preserve)
        gpu.upload_state_array("car_states", cars.ctypes.data, len(cars), preserve)
        gpu.upload_state_array("ball_states", balls.ctypes.data, len(balls), preserve)
        gc = gpu.download_car_states()
        assert np.array_equal(gc, orc.cars()), preserve
        if preserve:
            assert np.array_equal(gc, cars)
        for _ in range(30):
            ctrl = scenarios.chase_ball_controls(orc.cars(), orc.balls(), MC, crng)
            orc.step_with_controls(ctrl, 1, 0)
            gpu.step_with_device_controls(torch.from_numpy(ctrl).cuda().data_ptr(), 1, 0)
        gpu.synchronize()
        assert parity.equal(orc.cars(), gpu.download_car_states()), preserve
        assert parity.equal(orc.balls(), gpu.download_ball_states()), preserve


def test_internal_state_snapshot_restores_a_batch(arena_mesh):
    """Public arrays (PreserveInternal) plus the internal state blob are a whole snapshot: restoring one into the
    batch and replaying the same controls repeats the same ticks byte for byte (reference download/upload_internal_
    state, python/rocketgpu_bindings.cpp:1002-1060)."""
    import torch
    from rocketgpu_b200.batch_sim import BatchSim, SimConfig
    v, i = arena_mesh
    n, mc = 48, 4
    gpu = BatchSim(SimConfig(kickoff_settled=0, env_count=n, max_cars_per_env=mc), v, i)
    counts = np.array([2, 4, 3] * (n // 3), np.int32)
    gpu.set_env_car_count(counts)
    gpu.set_teams(np.tile(np.array([0, 1, 0, 1], np.uint8), n))
    gpu.reset_to_kickoff(9)
    crng = np.random.default_rng(9)
    for _ in range(60):
        ctrl = scenarios.chase_ball_controls(gpu.download_car_states(), gpu.download_ball_states(), mc, crng)
        gpu.step_with_device_controls(torch.from_numpy(ctrl).cuda().data_ptr(), 1, 0)
    gpu.synchronize()
    layout = gpu.internal_state_layout()
    assert [name for name, _ in layout] == ["wheel_runtime", "ball_world", "broadphase", "car_world", "ball_car",
                                            "car_pairs", "car_stages"]
    public = {name: getattr(gpu, f"download_{name}")() for name in ("car_states", "ball_states", "env_states",
                                                                    "boost_pad_states")}
    blob = gpu.download_internal_state()
    replay = [scenarios.chase_ball_controls(public["car_states"], public["ball_states"], mc, crng) for _ in range(8)]

    def run():
        outs = []
        for k in range(40):
            gpu.step_with_device_controls(torch.from_numpy(replay[k % 8]).cuda().data_ptr(), 1, 0)
        gpu.synchronize()
        for name in public:
            outs.append(getattr(gpu, f"download_{name}")())
        outs.append(gpu.download_internal_state())
        return outs
    first = run()
    for name, arr in public.items():
        gpu.upload_state_array(name, arr.ctypes.data, len(arr), True)
    gpu.upload_internal_state(blob)
    assert np.array_equal(gpu.download_internal_state(), blob)
    second = run()
    for a, b in zip(first, second):
        assert np.array_equal(a, b)
    assert not np.array_equal(first[0], public["car_states"])


def test_pybind_module_steps_like_the_oracle(oracle_available, arena_mesh):
    """The pybind11 module with the reference binding's names: a mixed batch driven through it matches the oracle."""
    import importlib
    import os
    import sys

    import torch
    from rocketgpu_b200 import abi
    sys.path.insert(0, os.path.join(abi.HERE, "_lib"))
    m = importlib.import_module("rocketgpu_py_b200")
    v, i = arena_mesh
    n, mc = 32, 6
    cfg = m.SimConfig()
    cfg.env_count, cfg.max_cars_per_env, cfg.kickoff_settled = n, mc, 0
    layout = m.ArenaLayout()
    layout.meshes = [m.ArenaMesh(v, i)]
    sim = m.BatchSim(cfg, layout)
    orc = oracle_ref.OracleSim(n, mc, v, i, kickoff_settled=False)
    counts = np.random.default_rng(2).choice(np.array([2, 4, 6], np.int32), n).astype(np.int32)
    teams = np.tile(np.array([0, 1, 0, 1, 0, 1], np.uint8), n)
    for s in (sim, orc):
        s.set_env_car_count(counts.tolist() if s is sim else counts)
        s.set_teams(teams.tolist() if s is sim else teams)
        s.reset_to_kickoff(2)
    stream = scenarios.ControlStream(n * mc, seed=3, p_jump=0.1, hold_max=20)
    dev = torch.zeros((8 * n * mc, 24), dtype=torch.uint8, device="cuda")
    for _ in range(20):
        block = np.stack([stream.next() for _ in range(8)]).reshape(-1, 24)
        orc.step_with_controls(block, 8, n * mc)
        dev.copy_(torch.from_numpy(block))
        sim.step_with_device_controls(dev.data_ptr(), 8, n * mc)
    sim.synchronize()
    assert parity.equal(sim.download_car_states(), orc.cars())
    assert parity.equal(sim.download_ball_states(), orc.balls())
    assert np.array_equal(sim.download_env_states(), orc.envs())
    assert sim.device_view()["car_states"] != 0
