"""The multi-GPU path's host logic as two `gloo` ranks on CPU: every rank steps its own shard of arenas (weak
scaling, no data-path collective), the timed duration is the max over ranks, and the reference arm runs on rank 0
alone. No GPU."""
import os

import numpy as np
import torch.multiprocessing as mp


def _rank(rank, world, port, out):
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world))
    import datetime
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    import bench
    w = bench.MixedWorkload(rank)
    bench.barrier(world)
    t = bench.max_over_ranks(1.5 + rank, world)
    ref = bench.run_reference(type("A", (), {"workload": "mixed", "warmup": 3, "steps": 1})(), world, rank) \
        if rank != 0 else "rank0"
    out.put((rank, t, w.counts.sum(), int(w.counts[:64].sum()), w.reset_seed, ref))
    dist.destroy_process_group()


def test_two_gloo_ranks_shard_arenas_and_take_the_max_time():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = 29000 + os.getpid() % 1000
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = sorted(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    (r0, t0, total0, head0, seed0, ref0), (r1, t1, total1, head1, seed1, ref1) = res
    assert t0 == t1 == 2.5                      # the max over ranks
    assert seed0 != seed1 and head0 != head1   # each rank draws its own shard
    assert 2 * 16384 <= total0 <= 6 * 16384 and 2 * 16384 <= total1 <= 6 * 16384
    assert ref0 == "rank0" and ref1 is None    # the reference arm runs on rank 0 only
    assert np.isfinite(t0)
