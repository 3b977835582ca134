"""The multi-rank plumbing (aerosim_b200.distributed) with world size 2 on the gloo
backend, on CPU: every work item assigned exactly once, the slowest rank's time and
the totals reduced across ranks, a barrier that both ranks pass, and the weak-scaling
aggregate the benchmark forms from them."""
import os

import pytest
import torch.multiprocessing as mp

from aerosim_b200 import distributed


def _worker(rank, world, port, q):
    os.environ.update({"RANK": str(rank), "WORLD_SIZE": str(world), "LOCAL_RANK": str(rank),
                       "MASTER_ADDR": "127.0.0.1", "MASTER_PORT": str(port)})
    try:
        distributed.init("gloo", timeout_s=60)
        ws, r, _ = distributed.env()
        items = list(range(32))
        mine = distributed.shard(items, r, ws)
        total = distributed.sum_over_ranks(len(mine))
        t = distributed.max_over_ranks(1.0 + r)  # the slower rank takes 2.0
        distributed.barrier()
        cells, steps = 1000, 10
        mlups = ws * cells * steps / (t * 1e-3) / 1e6
        q.put((r, mine, total, t, mlups))
    finally:
        import torch.distributed as dist
        if dist.is_initialized():
            dist.destroy_process_group()


def test_world_size_two_on_gloo():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = 29500 + os.getpid() % 1000
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = sorted(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    (r0, m0, tot0, t0, v0), (r1, m1, tot1, t1, v1) = res
    assert sorted(m0 + m1) == list(range(32)) and not set(m0) & set(m1)
    assert tot0 == tot1 == 32
    assert t0 == t1 == 2.0
    assert v0 == v1 == pytest.approx(2 * 1000 * 10 / 2.0e-3 / 1e6)


def test_single_process_fallbacks():
    assert distributed.env()[0] >= 1
    assert distributed.shard([1, 2, 3], 0, 1) == [1, 2, 3]
    assert distributed.max_over_ranks(3.5) == 3.5
