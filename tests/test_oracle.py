"""The oracle (the reference's own CPU BatchSim, oracle/_ref) against the committed golden fixtures, and the
synthetic arena generator's determinism. CPU only."""
import hashlib
import os

import numpy as np

from tests import oracle_ref, scenarios

HERE = os.path.dirname(os.path.abspath(__file__))


def test_arena_mesh_is_deterministic(arena_mesh):
    v, i = arena_mesh
    assert v.dtype == np.float32 and i.dtype == np.int32
    assert 9000 <= len(i) // 3 <= 12000
    h = hashlib.sha256(v.tobytes() + i.tobytes()).hexdigest()
    from rocketgpu_b200 import arena
    v2, i2 = arena.generate()
    assert hashlib.sha256(v2.tobytes() + i2.tobytes()).hexdigest() == h


def test_oracle_reproduces_golden_free_flight(oracle_available, arena_mesh):
    g = np.load(os.path.join(HERE, "golden", "ball_free_flight.npz"))
    v, i = arena_mesh
    n = g["init_balls"].shape[0]
    sim = oracle_ref.OracleSim(n, 2, v, i, kickoff_settled=False)
    sim.set_env_car_count([0] * n)
    _, default_ball, _, _, _ = oracle_ref.default_states()
    init = scenarios.free_flight_states(default_ball, n, int(g["seed"]))
    assert bytes(init) == bytes(g["init_balls"])
    sim.upload_balls(init)
    for t in range(g["balls"].shape[0]):
        sim.step(1)
        assert bytes(sim.balls()) == bytes(g["balls"][t]), t
        assert bytes(sim.envs()) == bytes(g["envs"][t]), t


def test_oracle_reproduces_golden_contacts(oracle_available, arena_mesh):
    g = np.load(os.path.join(HERE, "golden", "ball_contacts.npz"))
    v, i = arena_mesh
    n = g["init_balls"].shape[0]
    sim = oracle_ref.OracleSim(n, 2, v, i, kickoff_settled=False)
    sim.set_env_car_count([0] * n)
    _, default_ball, _, _, _ = oracle_ref.default_states()
    init = scenarios.ball_states(default_ball, n, int(g["seed"]))
    assert bytes(init) == bytes(g["init_balls"])
    sim.upload_balls(init)
    for t in range(g["balls"].shape[0]):
        sim.step(1)
        assert bytes(sim.balls()) == bytes(g["balls"][t]), t


def test_mesh_tables_match_reference(oracle_available, arena_mesh):
    """The product's arena build (triangles, internal-edge angles, BVH leaf order) equals the reference loader's."""
    import ctypes

    from rocketgpu_b200 import abi, arena
    L = oracle_ref.lib()
    L.orc_mesh_tables.restype = ctypes.c_int64
    L.orc_mesh_tables.argtypes = [ctypes.c_void_p, ctypes.c_int64, ctypes.c_void_p, ctypes.c_int64,
                                  ctypes.c_void_p, ctypes.c_int64]
    L.orc_mesh_nodes.restype = ctypes.c_int64
    L.orc_mesh_nodes.argtypes = [ctypes.c_void_p, ctypes.c_int64]
    for v, i in (arena_mesh, arena.generate_dense()):
        nt = len(i) // 3
        ref = np.zeros((nt, 16), np.float32)
        assert L.orc_mesh_tables(v.ctypes.data, len(v), i.ctypes.data, len(i), ref.ctypes.data, nt) == nt
        nodes = np.zeros((2 * nt, 7), np.int32)
        nn = L.orc_mesh_nodes(nodes.ctypes.data, 2 * nt)
        ref_leaf = nodes[:nn][nodes[:nn, 6] >= 0, 6]
        lay = abi.rg_arena_layout()
        lay.vertices_uu = v.ctypes.data_as(ctypes.POINTER(ctypes.c_float))
        lay.vertex_count = len(v)
        lay.indices = i.ctypes.data_as(ctypes.POINTER(ctypes.c_int32))
        lay.index_count = len(i)
        mine = np.zeros((nt, 16), np.float32)
        leaf = np.zeros(nt, np.int32)
        assert abi.lib().rg_arena_mesh_tables(ctypes.byref(lay), mine.ctypes.data, leaf.ctypes.data, nt) == nt
        assert bytes(mine) == bytes(ref)
        assert (leaf == ref_leaf).all()


def _run_mixed(n, ticks, seed, arena_mesh):
    v, i = arena_mesh
    rng = np.random.default_rng(seed)
    counts = rng.choice(np.array([2, 4, 6], np.int32), size=n).astype(np.int32)
    sim = oracle_ref.OracleSim(n, 6, v, i, kickoff_settled=False)
    sim.set_env_car_count(counts)
    sim.reset_to_kickoff(seed)
    stream = scenarios.ControlStream(n * 6, seed=seed, p_jump=0.1, hold_max=30)
    for _ in range(ticks // 8):
        block = np.stack([stream.next() for _ in range(8)]).reshape(-1, 24)
        sim.step_with_controls(block, 8, n * 6)
    out = (sim.cars(), sim.balls(), sim.envs(), sim.pads())
    sim.close()
    return out


def test_native_oracle_build_matches_portable(oracle_available, arena_mesh):
    """The timed CPU baseline uses an x86-64-v3 build of the reference; with -ffp-contract=off it must step exactly
    like the portable build the parity tests use."""
    import ctypes
    import pytest
    native = os.path.join(os.path.dirname(oracle_ref.LIB_PATH), "librg_oracle_native.so")
    if not os.path.exists(native):
        pytest.skip("native oracle not built")
    try:
        ctypes.CDLL(native)
    except OSError:
        pytest.skip("native oracle does not load on this host")
    portable = _run_mixed(48, 240, 5, arena_mesh)
    saved = (oracle_ref.LIB_PATH, oracle_ref._lib)
    try:
        oracle_ref.LIB_PATH, oracle_ref._lib = native, None
        fast = _run_mixed(48, 240, 5, arena_mesh)
    finally:
        oracle_ref.LIB_PATH, oracle_ref._lib = saved
    for a, b in zip(portable, fast):
        assert np.array_equal(a, b)
