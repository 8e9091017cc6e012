"""The multi-rank plumbing of bench.py (mercury_b200/dist.py) with the gloo
backend on CPU, world size 2: sharding, per-rank seeds, max/sum over ranks
and the per-robot all-gather."""
import os
import socket

import pytest
import torch.multiprocessing as mp


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, out):
    os.environ.update(RANK=str(rank), LOCAL_RANK=str(rank), WORLD_SIZE=str(world),
                      MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    import torch

    from mercury_b200 import dist
    assert dist.init("gloo", timeout_s=60)
    r, lr, w = dist.env_rank()
    mine = dist.shard(10, r, w)
    t = dist.max_over_ranks(1.0 + r)
    s = dist.sum_over_ranks(float(len(mine)))
    g = dist.gather_fitness(torch.full((3,), float(r)))
    dist.barrier()
    out.put((r, list(mine), t, s, g.tolist(), dist.seed_base(1000, r)))
    dist.finalize()


def test_two_ranks_gloo():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    ps = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in ps:
        p.start()
    res = sorted(q.get(timeout=120) for _ in ps)
    for p in ps:
        p.join(60)
        assert p.exitcode == 0
    (r0, m0, t0, s0, g0, seed0), (r1, m1, t1, s1, g1, seed1) = res
    assert m0 == [0, 1, 2, 3, 4] and m1 == [5, 6, 7, 8, 9]
    assert t0 == t1 == 2.0 and s0 == s1 == 10.0
    assert g0 == g1 == [0.0, 0.0, 0.0, 1.0, 1.0, 1.0]
    assert seed0 != seed1


def test_shard_covers_everything():
    from mercury_b200 import dist
    for n in (0, 1, 7, 512, 513):
        for w in (1, 2, 3, 8):
            idx = [i for r in range(w) for i in dist.shard(n, r, w)]
            assert idx == list(range(n))
