"""The serving loop (rg_server_*): results of every client bitwise equal to its arenas stepped alone in a BatchSim
with the same controls, whatever else shares the GPU; admission against the pool's capacity; a client that dies
with requests in flight. GPU tests; the argument checks that need no GPU are in test_abi.py."""
import threading

import numpy as np
import pytest

from tests import oracle_ref, scenarios

pytestmark = pytest.mark.gpu
MC = 6


def _client_spec(n, seed):
    rng = np.random.default_rng(seed)
    counts = rng.choice(np.array([2, 4, 6], np.int32), size=n, p=[0.55, 0.27, 0.18]).astype(np.int32)
    teams = np.zeros(n * MC, np.uint8)
    for e in range(n):
        teams[e * MC + counts[e] // 2: e * MC + counts[e]] = 1
    cfgs = np.stack([oracle_ref.car_preset(int(p)) for p in rng.integers(0, 6, n * MC)])
    stream = scenarios.ControlStream(n * MC, seed=seed + 1, p_jump=0.1, hold_max=30)
    reqs = []
    for _ in range(12):
        t = int(rng.choice([1, 4, 8]))
        reqs.append(np.stack([stream.next() for _ in range(t)]))
    return counts, teams, cfgs, seed * 7 + 3, reqs


def _alone(arena_mesh, spec):
    import torch
    from rocketgpu_b200.batch_sim import BatchSim, SimConfig
    counts, teams, cfgs, seed, reqs = spec
    n = len(counts)
    v, i = arena_mesh
    sim = BatchSim(SimConfig(kickoff_settled=0, env_count=n, max_cars_per_env=MC), v, i)
    sim.set_env_car_count(counts)
    sim.set_teams(teams)
    sim.set_car_configs(cfgs)
    sim.reset_to_kickoff(seed)
    out = []
    for r in reqs:
        dev = torch.from_numpy(r.reshape(-1, 24).copy()).cuda()
        sim.step_with_device_controls(dev.data_ptr(), r.shape[0], n * MC)
        sim.synchronize()
        out.append((sim.download_car_states(), sim.download_ball_states(), sim.download_env_states()))
    sim.close()
    return out


def _served(arena_mesh, specs, policy, order_seed):
    from rocketgpu_b200.server import Server
    v, i = arena_mesh
    srv = Server(v, i, max_arenas=sum(len(s[0]) for s in specs) + 10, policy=policy, max_cars_per_env=MC)
    clients = [srv.open_client(s[0], s[1], s[2], s[3]) for s in specs]
    # submissions interleaved in a seeded order, several requests of a client queued at once
    rng = np.random.default_rng(order_seed)
    order = np.concatenate([np.full(len(s[4]), k) for k, s in enumerate(specs)])
    rng.shuffle(order)
    nxt = [0] * len(specs)
    pending = []
    results = [[None] * len(s[4]) for s in specs]
    for k in order:
        r = specs[k][4][nxt[k]]
        pending.append((k, nxt[k], srv.submit(clients[k], r)))
        nxt[k] += 1
        if rng.random() < 0.3:
            kk, j, req = pending.pop(0)
            res = srv.poll(req, clients[kk], wait_ms=60000)
            assert res is not None
            results[kk][j] = res
    for kk, j, req in pending:
        res = srv.poll(req, clients[kk], wait_ms=60000)
        assert res is not None
        results[kk][j] = res
    stats = srv.stats()
    srv.close()
    return results, stats


@pytest.mark.parametrize("policy", ["continuous", "static"])
def test_each_client_alone_and_in_the_mix(oracle_available, arena_mesh, policy):
    specs = [_client_spec(n, 90 + n) for n in (16, 40, 7, 64)]
    alone = [_alone(arena_mesh, s) for s in specs]
    served, stats = _served(arena_mesh, specs, policy, order_seed=5)
    for k, s in enumerate(specs):
        counts = s[0]
        act = np.concatenate([np.arange(e * MC, e * MC + counts[e]) for e in range(len(counts))])
        for j in range(len(s[4])):
            lat, cars, balls, envs = served[k][j]
            ac, ab, ae = alone[k][j]
            assert np.array_equal(cars[act], ac[act]), (policy, k, j, "cars")
            assert np.array_equal(balls, ab), (policy, k, j, "balls")
            assert np.array_equal(envs, ae), (policy, k, j, "envs")
            assert lat > 0
    assert stats["completed"] == sum(len(s[4]) for s in specs)
    assert stats["arena_ticks"] == sum(len(s[0]) * sum(r.shape[0] for r in s[4]) for s in specs)


def test_admission_against_capacity(arena_mesh):
    from rocketgpu_b200.server import Busy, Server
    v, i = arena_mesh
    srv = Server(v, i, max_arenas=100, max_cars_per_env=MC)
    a = srv.open_client(np.full(60, 2, np.int32))
    with pytest.raises(Busy):
        srv.open_client(np.full(50, 2, np.int32))
    b = srv.open_client(np.full(40, 2, np.int32))
    assert srv.stats()["used"] == 100
    srv.close_client(a)
    c = srv.open_client(np.full(50, 4, np.int32))
    st = srv.stats()
    assert st["used"] == 90 and st["clients"] == 2
    srv.close_client(b)
    srv.close_client(c)
    srv.close()
    # the HBM budget alone sizes the pool
    probe = Server(v, i, max_arenas=1, max_cars_per_env=MC)
    slot = probe.stats()["slot_bytes"]
    probe.close()
    small = Server(v, i, hbm_budget_bytes=slot * 10 + slot // 2, max_cars_per_env=MC)
    assert small.stats()["capacity"] == 10
    small.close()


def test_client_that_dies_mid_request(arena_mesh):
    """A client thread submits and dies without polling or closing; the other client keeps being served, and closing
    the dead client afterwards frees its slots."""
    from rocketgpu_b200.server import Server
    v, i = arena_mesh
    srv = Server(v, i, max_arenas=64, max_cars_per_env=MC)
    dead = srv.open_client(np.full(24, 4, np.int32))
    live = srv.open_client(np.full(16, 2, np.int32))
    ctrl_dead = np.zeros((8, 24 * MC, 24), np.uint8)
    ctrl_live = np.zeros((4, 16 * MC, 24), np.uint8)

    def doomed():
        for _ in range(3):
            srv.submit(dead, ctrl_dead)
        raise SystemExit  # the thread ends with its requests in flight

    t = threading.Thread(target=doomed)
    t.start()
    t.join()
    for _ in range(5):
        req = srv.submit(live, ctrl_live)
        assert srv.poll(req, wait_ms=60000) is not None
    srv.close_client(dead)
    st = srv.stats()
    assert st["used"] == 16 and st["clients"] == 1
    req = srv.submit(live, ctrl_live)
    assert srv.poll(req, wait_ms=60000) is not None
    srv.close()
