"""Source sharding across ranks: one process per GPU, each holding a replica
of the graph and running its own slice of the sources.  No data-path
collective: sources are independent, so the only cross-rank traffic is the
max-over-ranks timing reduction and an optional gather of results."""
from __future__ import annotations

import numpy as np

import hc


def rank_sources(host: "hc.HostCSR", per_rank: int, rank: int) -> np.ndarray:
    """Rank r runs picks [r*k, (r+1)*k) of the SourcePicker sequence, so every
    rank's sources are distinct and the union equals a single-process run of
    world*k picks."""
    return hc.pick_sources(host, per_rank * (rank + 1))[per_rank * rank:]


def split_batch(sources: np.ndarray, rank: int, world: int) -> np.ndarray:
    """Contiguous near-equal split of one batch of sources (strong scaling)."""
    bounds = np.linspace(0, len(sources), world + 1).round().astype(int)
    return sources[bounds[rank]:bounds[rank + 1]]


def run_sharded(run, sources: np.ndarray, rank: int, world: int) -> np.ndarray:
    """One batch of sources over all ranks (strong scaling): this rank runs `run` on its contiguous share
    (split_batch) -- a batched BFS / SSSP call returning [k_r, N] rows -- and every rank receives all rows in
    the batch's source order."""
    return gather_rows(np.asarray(run(split_batch(sources, rank, world))), world)


def max_over_ranks(value: float, device=None) -> float:
    """Max of a per-rank scalar (the timing rule for multi-GPU numbers)."""
    import torch
    import torch.distributed as dist
    if not dist.is_available() or not dist.is_initialized() or dist.get_world_size() == 1:
        return float(value)
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def gather_rows(rows: np.ndarray, world: int) -> np.ndarray | None:
    """Gathers each rank's [k_r, N] result block on every rank, in rank order."""
    import torch.distributed as dist
    if world == 1:
        return rows
    out = [None] * world
    dist.all_gather_object(out, rows)
    return np.concatenate(out, axis=0)
