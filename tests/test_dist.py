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


def _shard_worker(rank, world, port, out):
    """Each rank steps its shard of an 11-robot population with the oracle
    (the CPU stand-in for the CUDA step on its GPU) and all-gathers the
    per-robot centres of mass and fitness."""
    os.environ.update(RANK=str(rank), LOCAL_RANK=str(rank), WORLD_SIZE=str(world),
                      MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    import numpy as np
    import torch

    import mercury_b200 as mb
    from mercury_b200 import dist, robots
    from oracle import core
    assert dist.init("gloo", timeout_s=60)
    full = robots.population_batch("uneven", 11, seed_base=777)
    mine = dist.shard(full.n_robots, rank, world)
    b = dist.shard_batch(full, mine)
    p, v = b.pos.copy(), b.vel.copy()
    s = np.zeros(b.n_springs, np.float32)
    core.xpbd_run(b, p, v, s, mb.material_table(), np.float32(1e-3), 0.0, 200, True, 1)
    com = torch.from_numpy(core.com_device(b, p))
    base = torch.from_numpy(core.com_device(b, b.pos))
    fit = torch.from_numpy(mb.fitness(com.numpy(), base.numpy(), mb.body_length(b)))
    g_com = dist.gather_per_robot(com, full.n_robots)
    g_fit = dist.gather_per_robot(fit, full.n_robots)
    out.put((rank, len(mine), g_com.numpy().tobytes(), g_fit.numpy().tobytes()))
    dist.barrier()
    dist.finalize()


def test_sharded_population_equals_one_process():
    """Population sharding over 2 gloo ranks: the gathered per-robot COM and
    fitness equal, bit for bit, those of the whole population stepped in one
    process."""
    import numpy as np

    import mercury_b200 as mb
    from mercury_b200 import robots
    from oracle import core
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    ps = [ctx.Process(target=_shard_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in ps:
        p.start()
    res = sorted(q.get(timeout=180) for _ in ps)
    for p in ps:
        p.join(60)
        assert p.exitcode == 0
    full = robots.population_batch("uneven", 11, seed_base=777)
    p, v = full.pos.copy(), full.vel.copy()
    s = np.zeros(full.n_springs, np.float32)
    core.xpbd_run(full, p, v, s, mb.material_table(), np.float32(1e-3), 0.0, 200, True, 1)
    com = core.com_device(full, p)
    fit = mb.fitness(com, core.com_device(full, full.pos), mb.body_length(full))
    assert [r[1] for r in res] == [6, 5]
    for _, _, g_com, g_fit in res:
        assert g_com == com.tobytes()
        assert g_fit == fit.tobytes()
