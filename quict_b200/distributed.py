"""Batch sharding across GPUs (one process per GPU, torch.distributed).

The state-vector path does not shard: a 30-qubit complex128 state (16 GiB) and
even 32 qubits in complex64 (32 GiB) fit one 180 GB B200, so several GPUs run
independent replicas.  Batches of independent instances (parameter sets,
QAOA instances) partition across ranks with no collective on the data path;
the only exchange is gathering the per-instance results (KB-sized) at the
end, which works on NCCL (GPU tensors) and gloo (CPU tensors).
"""
from __future__ import annotations

import heapq
from typing import Callable, List, Sequence, Tuple

import torch
import torch.distributed as dist


def block_shard(count: int, world: int, rank: int) -> range:
    """Contiguous block of [0, count) for `rank` (sizes differ by at most one)."""
    base, extra = divmod(count, world)
    start = rank * base + min(rank, extra)
    return range(start, start + base + (1 if rank < extra else 0))


def balanced_shard(costs: Sequence[float], world: int) -> List[List[int]]:
    """Longest-processing-time assignment of items to ranks by cost (e.g. 2^n
    amplitudes x circuit depth for uneven QAOA instances); deterministic."""
    order = sorted(range(len(costs)), key=lambda i: (-costs[i], i))
    heap = [(0.0, r) for r in range(world)]
    out: List[List[int]] = [[] for _ in range(world)]
    for i in order:
        load, r = heapq.heappop(heap)
        out[r].append(i)
        heapq.heappush(heap, (load + costs[i], r))
    return [sorted(s) for s in out]


def gather_rows(local: torch.Tensor, indices: Sequence[int], total: int) -> torch.Tensor:
    """All-gather per-instance result rows computed on each rank into one
    (total, ...) tensor in global instance order (on every rank)."""
    world = dist.get_world_size() if dist.is_initialized() else 1
    if world == 1:
        out = torch.empty((total,) + tuple(local.shape[1:]), dtype=local.dtype, device=local.device)
        out[list(indices)] = local
        return out
    idx = torch.tensor(list(indices), dtype=torch.long, device=local.device)
    # pad to the largest shard so every rank sends the same shape
    n = torch.tensor([idx.numel()], device=local.device)
    sizes = [torch.zeros_like(n) for _ in range(world)]
    dist.all_gather(sizes, n)
    m = int(max(s.item() for s in sizes))
    pad_rows = torch.zeros((m,) + tuple(local.shape[1:]), dtype=local.dtype, device=local.device)
    pad_rows[: idx.numel()] = local
    pad_idx = torch.full((m,), -1, dtype=torch.long, device=local.device)
    pad_idx[: idx.numel()] = idx
    rows = [torch.empty_like(pad_rows) for _ in range(world)]
    idxs = [torch.empty_like(pad_idx) for _ in range(world)]
    dist.all_gather(rows, pad_rows)
    dist.all_gather(idxs, pad_idx)
    out = torch.empty((total,) + tuple(local.shape[1:]), dtype=local.dtype, device=local.device)
    for r, ix in zip(rows, idxs):
        keep = ix >= 0
        out[ix[keep]] = r[keep]
    return out


def run_sharded(fn: Callable[[List[int]], torch.Tensor], costs: Sequence[float]) -> torch.Tensor:
    """Evaluate fn on this rank's instances (chosen by cost balance) and gather
    the rows of every rank in global order."""
    world = dist.get_world_size() if dist.is_initialized() else 1
    rank = dist.get_rank() if dist.is_initialized() else 0
    mine = balanced_shard(costs, world)[rank]
    local = fn(mine)
    return gather_rows(local, mine, len(costs))
