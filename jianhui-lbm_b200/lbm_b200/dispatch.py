"""Host-side dispatch of independent solves over one process per GPU.

The batched and serving workloads are independent permeability solves, so a
multi-GPU run needs no data-path collective: every rank takes a fixed share of
the solves, runs it in its own node pool, and only the timing is combined
(max over ranks).  This replaces the reference's one batch job per sample
(CPP_SCRIPT/HPC_SUBDOMAIN_INPUT.cpp:240-270 writes an INPUT file and a PBS
script with one ``mpiexec`` per subdomain); the reference's x-slab halo
exchange is the single-domain decomposition, which is not used here (single
domains run as replicas).
"""
from __future__ import annotations

import datetime
import os

__all__ = ["shard", "dist_env", "init_process_group", "max_over_ranks", "barrier"]


def shard(weights, world, rank):
    """Indices of the items that ``rank`` runs: greedy longest-first
    assignment by weight (fluid nodes), ties to the lowest rank.  Every rank
    computes the same assignment from the same weights, so no message is
    exchanged; the shares are disjoint and cover every item."""
    if world < 1 or not 0 <= rank < world:
        raise ValueError(f"rank {rank} out of range for world size {world}")
    order = sorted(range(len(weights)), key=lambda i: (-float(weights[i]), i))
    load = [0.0] * world
    mine = []
    for i in order:
        r = min(range(world), key=lambda k: (load[k], k))
        load[r] += float(weights[i])
        if r == rank:
            mine.append(i)
    return sorted(mine)


def dist_env():
    """(world, rank, local_rank) from the torchrun environment."""
    return (int(os.environ.get("WORLD_SIZE", "1")), int(os.environ.get("RANK", "0")),
            int(os.environ.get("LOCAL_RANK", "0")))


def init_process_group(timeout_s=600):
    """Host process group for barriers and the max-over-ranks timing (gloo:
    nothing but a few scalars crosses it).  None at world size 1."""
    world, _, _ = dist_env()
    if world <= 1:
        return None
    import torch.distributed as dist

    if not dist.is_initialized():
        dist.init_process_group("gloo", timeout=datetime.timedelta(seconds=timeout_s))
    return dist


def max_over_ranks(pg, x):
    if pg is None:
        return float(x)
    import torch

    t = torch.tensor([float(x)], dtype=torch.float64)
    pg.all_reduce(t, op=pg.ReduceOp.MAX)
    return float(t.item())


def barrier(pg):
    if pg is not None:
        pg.barrier()
