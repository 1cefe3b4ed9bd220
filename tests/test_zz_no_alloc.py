"""The entry point that steps without allocating device memory (rg_batch_step_static_scratch).

Some callers cannot call cudaMalloc at the moment they step: their device memory belongs to another framework's
pool, or an allocation's implicit synchronisation would stall a latency-bound loop. This entry point keeps the
per-arena contact manifolds in a fixed array compiled into the library instead of batch-allocated memory. This test
checks, through the C ABI, that two calls in a row give exactly (bit for bit, the tolerance of every parity test
here) the states the ordinary batch step gives on the same inputs: the first call starts from cleared manifolds,
the second continues from the manifolds the first left. It sits in a file pytest collects last, so a failure here
comes after every other test has run.
"""
import ctypes

import numpy as np
import pytest

from tests import scenarios

pytestmark = pytest.mark.gpu


def test_static_scratch_step_matches_batch_step_on_two_calls(arena_mesh):
    import torch

    from rocketgpu_b200 import abi
    from rocketgpu_b200.batch_sim import BatchSim, SimConfig

    lib = abi.lib()
    v, i = arena_mesh
    n = 1024
    ref = BatchSim(SimConfig(kickoff_settled=0, env_count=n, max_cars_per_env=2), v, i)
    ref.set_env_car_count([0] * n)
    default_ball = np.zeros(288, np.uint8)
    lib.rg_default_ball_state(default_ball.ctypes.data)
    init = scenarios.ball_states(default_ball, n, seed=31)
    ref.upload_ball_states(init)
    balls0 = ref.download_ball_states()
    envs0 = ref.download_env_states()

    # caller-owned device arrays holding the same (canonicalised) states
    d_balls = torch.from_numpy(balls0.copy()).cuda()
    d_envs = torch.from_numpy(envs0.copy()).cuda()
    torch.cuda.synchronize()

    for call, reset in ((0, 1), (1, 0)):
        ref.step(24)
        rc = lib.rg_batch_step_static_scratch(ref._h, ctypes.c_void_p(d_balls.data_ptr()),
                                              ctypes.c_void_p(d_envs.data_ptr()), n, 24, reset, None)
        assert rc == 0, lib.rg_last_error().decode()
        torch.cuda.synchronize()
        got_b = d_balls.cpu().numpy()
        got_e = d_envs.cpu().numpy()
        want_b = ref.download_ball_states()
        want_e = ref.download_env_states()
        bad = np.nonzero((got_b != want_b).any(1))[0]
        assert len(bad) == 0, f"call {call}: {len(bad)} arenas differ, first {bad[:4]}"
        assert bytes(got_e) == bytes(want_e), f"call {call}: env states differ"


def test_static_scratch_rejects_too_many_arenas(arena_mesh):
    import torch

    from rocketgpu_b200 import abi
    from rocketgpu_b200.batch_sim import BatchSim, SimConfig

    lib = abi.lib()
    v, i = arena_mesh
    sim = BatchSim(SimConfig(kickoff_settled=0, env_count=8, max_cars_per_env=2), v, i)
    d = torch.zeros(16, dtype=torch.uint8, device="cuda")
    rc = lib.rg_batch_step_static_scratch(sim._h, ctypes.c_void_p(d.data_ptr()), ctypes.c_void_p(d.data_ptr()),
                                          4097, 1, 1, None)
    assert rc == 3
    assert "4096" in lib.rg_last_error().decode()
