"""Multi-process plumbing for running one population per GPU.

Robots are independent, so a population shards across ranks with no data
exchange during the step: every rank simulates its own robots and only
timings (and, for evolution, per-robot fitness) cross ranks, through
torch.distributed.  Scaling is weak: each rank keeps the per-GPU workload.
"""
from __future__ import annotations

import datetime
import os

import torch
import torch.distributed as dist


def env_rank() -> tuple[int, int, int]:
    """(rank, local_rank, world_size) from the torchrun environment."""
    return (int(os.environ.get("RANK", 0)), int(os.environ.get("LOCAL_RANK", 0)),
            int(os.environ.get("WORLD_SIZE", 1)))


def init(backend: str, timeout_s: float = 120.0) -> bool:
    """Initialises the default process group when WORLD_SIZE > 1."""
    rank, _, world = env_rank()
    if world <= 1 or dist.is_initialized():
        return dist.is_initialized()
    os.environ.setdefault("MASTER_ADDR", "127.0.0.1")
    dist.init_process_group(backend, rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=timeout_s))
    return True


def shard(n_total: int, rank: int, world: int) -> range:
    """Contiguous block of robot indices owned by `rank`."""
    per, extra = divmod(n_total, world)
    start = rank * per + min(rank, extra)
    return range(start, start + per + (1 if rank < extra else 0))


def seed_base(population_seed: int, rank: int) -> int:
    """Seed of the first robot of a rank's own population (weak scaling:
    every rank simulates a distinct population of the same shape)."""
    return population_seed + 1_000_000 * rank


def max_over_ranks(x: float, device: torch.device | None = None) -> float:
    if not dist.is_initialized():
        return float(x)
    t = torch.tensor([float(x)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def sum_over_ranks(x: float, device: torch.device | None = None) -> float:
    if not dist.is_initialized():
        return float(x)
    t = torch.tensor([float(x)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.SUM)
    return float(t.item())


def gather_fitness(local: torch.Tensor) -> torch.Tensor:
    """All-gathers per-robot values of equal-sized shards (4 B per robot)."""
    if not dist.is_initialized():
        return local
    out = [torch.empty_like(local) for _ in range(dist.get_world_size())]
    dist.all_gather(out, local)
    return torch.cat(out)


def gather_per_robot(local: torch.Tensor, n_total: int) -> torch.Tensor:
    """All-gathers per-robot rows (shape (k, ...)) of the contiguous shards of
    shard(n_total, rank, world), which may differ in size by one: each rank
    pads its rows to the largest shard, and the padding is dropped after the
    gather.  Returns the (n_total, ...) rows in robot order on every rank."""
    if not dist.is_initialized():
        return local
    world = dist.get_world_size()
    sizes = [len(shard(n_total, r, world)) for r in range(world)]
    if local.shape[0] != sizes[dist.get_rank()]:
        raise ValueError(f"rank {dist.get_rank()} holds {local.shape[0]} rows, its shard has {sizes[dist.get_rank()]}")
    padded = torch.zeros((max(sizes), *local.shape[1:]), dtype=local.dtype, device=local.device)
    padded[: local.shape[0]] = local
    out = [torch.empty_like(padded) for _ in range(world)]
    dist.all_gather(out, padded)
    return torch.cat([o[:n] for o, n in zip(out, sizes)])


def shard_batch(batch, robots: range):
    """The robots `robots` (a contiguous range) of a packed population, as a
    population of their own (offsets rebased; faces kept)."""
    from .element import Batch
    r0, r1 = robots.start, robots.stop
    m0, m1 = int(batch.mass_offsets[r0]), int(batch.mass_offsets[r1])
    s0, s1 = int(batch.spring_offsets[r0]), int(batch.spring_offsets[r1])
    out = Batch(batch.mass_offsets[r0:r1 + 1] - m0, batch.pos[m0:m1].copy(), batch.vel[m0:m1].copy(),
                batch.mass_material[m0:m1].copy(), batch.spring_offsets[r0:r1 + 1] - s0,
                batch.pairs[s0:s1].copy(), batch.spring_material[s0:s1].copy(), batch.lbar[s0:s1].copy())
    if batch.face_offsets is not None:
        f0, f1 = int(batch.face_offsets[r0]), int(batch.face_offsets[r1])
        out.face_offsets = batch.face_offsets[r0:r1 + 1] - f0
        out.faces = batch.faces[f0:f1].copy()
    return out


def barrier() -> None:
    if dist.is_initialized():
        dist.barrier()


def finalize() -> None:
    if dist.is_initialized():
        dist.destroy_process_group()
