"""Launch configurations do not change results: the mixed workload with episode resets stepped with different block
sizes and with CUDA-graph replay gives, bitwise, the states of the default launches; the autotuner leaves a valid
configuration set. GPU tests."""
import numpy as np
import pytest

from tests import scenarios

pytestmark = pytest.mark.gpu
MC = 6


def _run(arena_mesh, config, steps=24, n=512):
    import torch
    from rocketgpu_b200 import autotune
    from rocketgpu_b200.batch_sim import BatchSim, SimConfig
    v, i = arena_mesh
    rng = np.random.default_rng(3)
    counts = rng.choice(np.array([2, 4, 6], np.int32), size=n, p=[0.55, 0.27, 0.18]).astype(np.int32)
    sim = BatchSim(SimConfig(kickoff_settled=0, env_count=n, max_cars_per_env=MC), v, i)
    sim.set_env_car_count(counts)
    sim.reset_to_kickoff(3)
    if config is not None:
        autotune.set_config(sim, *config)
    cmds = torch.zeros((8, n, 16), dtype=torch.uint8, device="cuda")
    sim.episode_commands(120, cmds.data_ptr(), stagger_seed=9, init=True)
    stream = scenarios.ControlStream(n * MC, seed=4, p_jump=0.1, hold_max=30)
    ctrl = torch.zeros((8 * n * MC, 24), dtype=torch.uint8, device="cuda")  # one buffer: graphs replay
    for _ in range(steps):
        ctrl.copy_(torch.from_numpy(np.stack([stream.next() for _ in range(8)]).reshape(-1, 24)))
        sim.step_with_device_commands(ctrl.data_ptr(), n * MC, cmds.data_ptr(), n, 8)
        sim.episode_commands(120, cmds.data_ptr())
    sim.synchronize()
    out = (sim.download_car_states(), sim.download_ball_states(), sim.download_env_states(),
           sim.download_boost_pad_states())
    sim.close()
    return out


def test_block_sizes_and_graphs_do_not_change_results(arena_mesh):
    base = _run(arena_mesh, None)
    for cfg in ((128, 256, False), (64, 32, True), (32, 64, True)):
        got = _run(arena_mesh, cfg)
        for a, b in zip(base, got):
            assert np.array_equal(a, b), cfg


def test_autotune_picks_a_candidate(arena_mesh):
    import torch
    from rocketgpu_b200 import autotune
    from rocketgpu_b200.batch_sim import BatchSim, SimConfig
    v, i = arena_mesh
    n = 256
    sim = BatchSim(SimConfig(kickoff_settled=0, env_count=n, max_cars_per_env=MC), v, i)
    sim.set_env_car_count(np.full(n, 4, np.int32))
    sim.reset_to_kickoff(1)
    ctrl = torch.zeros((8 * n * MC, 24), dtype=torch.uint8, device="cuda")
    best, results = autotune.autotune(sim, lambda: sim.step_with_device_controls(ctrl.data_ptr(), 8, n * MC),
                                      steps=2, arena_threads=(32, 64), car_threads=(64, 128))
    assert len(results) == 8 and best == autotune.get_config(sim)
    with pytest.raises(ValueError):
        autotune.set_config(sim, 48, 64, False)
