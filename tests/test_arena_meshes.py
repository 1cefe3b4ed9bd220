"""Two arena geometries in one batch (rg_batch_add_mesh / rg_batch_set_arena_meshes): the procedural ~11k-triangle
arena and its ~42k-triangle variant with 64-segment fillets, arenas alternating between them, started contact-heavy
(the ball at up to 6000 uu/s, 2v2 and 3v3 cars within 600 uu of it), demolitions and pads on. The reference takes one
geometry per BatchSim, so the oracle side is two BatchSims, each stepping every arena on its own mesh; arena e is
compared with the oracle of its mesh after every tick, bitwise (NaN payloads aside)."""
import numpy as np
import pytest

from tests import oracle_ref, parity, scenarios

pytestmark = pytest.mark.gpu
MC = 6


def test_two_geometries_in_one_batch(oracle_available, arena_mesh):
    import torch
    from rocketgpu_b200 import arena
    from rocketgpu_b200.batch_sim import BatchSim, SimConfig
    n, ticks = 64, 240
    meshes = [arena_mesh, arena.generate_fine()]
    rng = np.random.default_rng(17)
    counts = rng.choice(np.array([4, 6], np.int32), size=n, p=[0.3, 0.7]).astype(np.int32)
    teams = np.zeros(n * MC, np.uint8)
    for e in range(n):
        teams[e * MC + counts[e] // 2: e * MC + counts[e]] = 1
    mesh_of = (np.arange(n) % 2).astype(np.uint8)
    orcs = []
    for v, i in meshes:
        o = oracle_ref.OracleSim(n, MC, v, i, kickoff_settled=False)
        o.set_env_car_count(counts)
        o.set_teams(teams)
        o.reset_to_kickoff(17)
        orcs.append(o)
    gpu = BatchSim(SimConfig(kickoff_settled=0, env_count=n, max_cars_per_env=MC), *meshes[0])
    assert gpu.add_mesh(*meshes[1]) == 1
    gpu.set_arena_meshes(mesh_of)
    gpu.set_env_car_count(counts)
    gpu.set_teams(teams)
    gpu.reset_to_kickoff(17)
    cars, balls = scenarios.contact_heavy(orcs[0].cars(), orcs[0].balls(), counts, MC, seed=18)
    for sim in orcs:
        sim.upload_cars(cars)
        sim.upload_balls(balls)
    gpu.upload_car_states(cars)
    gpu.upload_ball_states(balls)
    gpu.synchronize()
    crng = np.random.default_rng(19)
    dev = torch.zeros((n * MC, 24), dtype=torch.uint8, device="cuda")
    bumps = 0
    for t in range(ticks):
        ctrl = scenarios.chase_ball_controls(orcs[0].cars(), orcs[0].balls(), MC, crng, p_jump=0.05)
        for o in orcs:
            o.step_with_controls(ctrl, 1, 0)
        dev.copy_(torch.from_numpy(ctrl))
        gpu.step_with_device_controls(dev.data_ptr(), 1, 0)
        gpu.synchronize()
        gc, gb, ge = gpu.download_car_states(), gpu.download_ball_states(), gpu.download_env_states()
        gp = gpu.download_boost_pad_states().reshape(n, -1)
        oc = [o.cars() for o in orcs]
        ob = [o.balls() for o in orcs]
        oe = [o.envs() for o in orcs]
        op = [o.pads().reshape(n, -1) for o in orcs]
        for e in range(n):
            m = mesh_of[e]
            rows = slice(e * MC, e * MC + counts[e])
            d = parity.first_mismatch((("cars", oc[m][rows], gc[rows]), ("ball", ob[m][e], gb[e]),
                                       ("env", oe[m][e], ge[e]), ("pads", op[m][e], gp[e])), {"cars": 880})
            assert d is None, f"tick {t} arena {e} (mesh {m}): {d}"
        bumps = max(bumps, int(gc[:, 412:426].astype(np.int64).sum()))  # bump and demolition event counters
    assert bumps > 0
