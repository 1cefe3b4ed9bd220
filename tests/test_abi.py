"""CPU tests of the C ABI boundary: the library loads, exports every declared symbol, its structs are byte-identical
to the reference's, and argument validation fails the way the reference's BatchSim does. No GPU calls."""
import ctypes
import re

import numpy as np
import pytest

from rocketgpu_b200 import abi


def test_library_exports_every_declared_symbol():
    lib = abi.lib()
    header = open(abi.os.path.join(abi.HERE, "..", "include", "rocketgpu_b200.h")).read()
    declared = set(re.findall(r"RG_API\s+[\w\s\*]+?\b(rg_\w+)\s*\(", header))
    assert declared == set(abi.EXPORTS), declared ^ set(abi.EXPORTS)
    for name in declared:
        assert hasattr(lib, name), name


def test_defaults_match_reference_structs(oracle_available):
    from tests import oracle_ref
    lib = abi.lib()
    car, ball, env, pad, cfg = oracle_ref.default_states()
    my_ball = np.zeros(288, np.uint8)
    my_env = np.zeros(44, np.uint8)
    lib.rg_default_ball_state(my_ball.ctypes.data)
    lib.rg_default_env_state(my_env.ctypes.data)
    assert bytes(my_ball) == bytes(ball)
    assert bytes(my_env) == bytes(env)
    my_car = np.zeros(880, np.uint8)
    my_cfg = np.zeros(120, np.uint8)
    lib.rg_default_car_state(my_car.ctypes.data)
    lib.rg_default_car_config(my_cfg.ctypes.data)
    assert bytes(my_car) == bytes(car), np.nonzero(my_car != car)[0]
    pad_byte = 81  # CarConfig's padding between three_wheels (u8 at 80) and body (u16 at 82)
    keep = np.arange(120) != pad_byte
    assert (my_cfg[keep] == cfg[keep]).all(), np.nonzero(my_cfg != cfg)[0]


def test_car_presets_match_reference(oracle_available):
    from rocketgpu_b200.batch_sim import car_preset
    from tests import oracle_ref
    keep = np.arange(120) != 81  # CarConfig's padding byte
    for k in range(6):
        assert (car_preset(k)[keep] == oracle_ref.car_preset(k)[keep]).all(), k
    assert (car_preset("merc") == car_preset(5)).all()
    with pytest.raises(IndexError):
        car_preset(6)


def test_ucrt_math_matches_reference(oracle_available):
    from tests import oracle_ref
    L = oracle_ref.lib()
    for f in (L.orc_ucrt_powf, L.orc_ucrt_atan2f):
        f.restype = ctypes.c_float
        f.argtypes = [ctypes.c_float, ctypes.c_float]
    for f in (L.orc_ucrt_sinf, L.orc_ucrt_cosf):
        f.restype = ctypes.c_float
        f.argtypes = [ctypes.c_float]
    lib = abi.lib()
    rng = np.random.default_rng(7)
    xs = np.concatenate([rng.uniform(-10, 10, 3000), rng.normal(0, 1e3, 1000), [0.0, -0.0, 1e-30, 1.0, -1.0]])
    ys = np.concatenate([rng.uniform(-10, 10, 3000), rng.normal(0, 1e3, 1000), [0.0, 1.0, -2.0, 0.5, 3.0]])
    def bits(v):
        return np.float32(v).view(np.uint32)
    for x, y in zip(xs.astype(np.float32), ys.astype(np.float32)):
        assert bits(lib.rg_ucrt_sinf(x)) == bits(L.orc_ucrt_sinf(x)), x
        assert bits(lib.rg_ucrt_cosf(x)) == bits(L.orc_ucrt_cosf(x)), x
        assert bits(lib.rg_ucrt_atan2f(y, x)) == bits(L.orc_ucrt_atan2f(y, x)), (y, x)
        ax = abs(x) % 4.0
        assert bits(lib.rg_ucrt_powf(ax, y)) == bits(L.orc_ucrt_powf(ax, y)), (ax, y)


def test_invalid_config_is_rejected_before_any_device_call(arena_mesh):
    from rocketgpu_b200.batch_sim import BatchSim, SimConfig
    v, i = arena_mesh
    with pytest.raises(ValueError):
        BatchSim(SimConfig(env_count=0), v, i)
    with pytest.raises(ValueError):
        BatchSim(SimConfig(env_count=4, max_cars_per_env=9), v, i)
    # 7- and 8-car arenas would overflow the car-car pair rows; kickoff settling is not built
    with pytest.raises(ValueError):
        BatchSim(SimConfig(env_count=4, max_cars_per_env=7), v, i)
    with pytest.raises(ValueError, match="kickoff_settled"):
        BatchSim(SimConfig(env_count=4, kickoff_settled=2), v, i)
    assert SimConfig().c.kickoff_settled == 1  # the reference's default
    with pytest.raises(ValueError):
        BatchSim(SimConfig(env_count=4), v, i[:-1])
    bad = v.copy()
    bad[0, 0] = 12000.0
    with pytest.raises(ValueError):
        BatchSim(SimConfig(env_count=4), bad, i)


def test_parity_compare_allows_only_nan_payloads():
    from tests import parity
    a = np.zeros(16, np.uint8)
    a[0:4] = np.frombuffer(np.float32(1.5).tobytes(), np.uint8)
    a[4:8] = np.frombuffer(np.uint32(0xffc00000).tobytes(), np.uint8)  # x86 NaN
    b = a.copy()
    b[4:8] = np.frombuffer(np.uint32(0x7fffffff).tobytes(), np.uint8)  # GPU NaN
    assert parity.equal(a, b)
    c = b.copy()
    c[0:4] = np.frombuffer(np.float32(1.5000001).tobytes(), np.uint8)  # one ulp
    assert parity.mismatched_bytes(a, c).tolist() == [0]
    d = a.copy()
    d[4:8] = np.frombuffer(np.float32(2.0).tobytes(), np.uint8)  # NaN on one side only
    assert not parity.equal(a, d)
    e = a.copy()
    e[15] = 1
    assert parity.mismatched_bytes(a, e).tolist() == [15]


def test_server_rejects_bad_config_before_any_device_call(arena_mesh):
    from rocketgpu_b200.server import Server
    v, i = arena_mesh
    with pytest.raises(ValueError):
        Server(v, i)  # neither max_arenas nor an HBM budget
    with pytest.raises(ValueError):
        Server(v, i, max_arenas=8, max_cars_per_env=7)
    with pytest.raises(KeyError):
        Server(v, i, max_arenas=8, policy="fifo")


def test_pybind_module_mirrors_the_reference_binding(arena_mesh):
    """rocketgpu_py_b200 (pybind11 over the C ABI) exposes the reference's rocketgpu_py.BatchSim method names; config
    errors surface as the reference's exception types before any device call."""
    import importlib
    import sys
    sys.path.insert(0, abi.os.path.join(abi.HERE, "_lib"))
    m = importlib.import_module("rocketgpu_py_b200")
    for name in ("env_count", "car_capacity", "boost_pad_capacity", "device_view", "set_env_car_count", "set_teams",
                 "set_car_configs", "upload_car_states", "upload_ball_states", "upload_env_states",
                 "upload_boost_pad_states", "upload_controls", "download_car_states", "download_ball_states",
                 "download_env_states", "download_boost_pad_states", "upload_state_array", "download_state_array",
                 "apply_env_commands", "apply_env_commands_device", "step", "step_with_device_controls",
                 "step_with_device_commands", "reset_to_kickoff", "synchronize", "internal_state_layout",
                 "download_internal_state", "upload_internal_state", "set_physics_event_stream"):
        assert hasattr(m.BatchSim, name), name
    assert m.physics_event_layout() == {"record_size": 104, "window_size": 16, "type_offset": 8,
                                        "velocity_offset": 80, "count_offset": 8, "overflow_offset": 12,
                                        "goal_type": 5}
    layout = m.ArenaLayout()
    for name in ("meshes", "boost_pads", "goals", "kickoff_spawns", "respawn_spawns", "ball_spawn"):
        assert hasattr(layout, name), name
    assert layout.goals[1].point.y == layout.goals[1].point.y and len(layout.respawn_spawns[1]) == 4
    cfg = m.SimConfig()
    assert cfg.kickoff_settled == 1 and cfg.max_cars_per_env == 6
    v, i = arena_mesh
    layout = m.ArenaLayout()
    layout.meshes = [m.ArenaMesh(v, i)]
    cfg.kickoff_settled = 2
    with pytest.raises(ValueError, match="kickoff_settled"):
        m.BatchSim(cfg, layout)
    cfg.kickoff_settled = 0
    cfg.max_cars_per_env = 7
    with pytest.raises(ValueError):
        m.BatchSim(cfg, layout)
