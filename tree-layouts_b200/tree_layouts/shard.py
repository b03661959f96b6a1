"""Sharding of the hot path over ranks (one process per GPU).

A single array's permutation does not shard (its tiles' destinations span the
whole array), so multi-GPU runs of it are replicas.  Two workloads do shard,
with no collective on the data path:

- a query batch against a layout replicated on every rank: each rank answers a
  contiguous slice of the batch;
- the batched mode: instances are dealt to ranks so that every rank permutes
  about the same number of keys (longest-processing-time greedy), each rank
  building its own offset table over its own instances.

Collectives appear only to assemble results for checking (gather_answers)."""
from __future__ import annotations

import heapq

import numpy as np


def query_slice(q: int, rank: int, world: int) -> tuple[int, int]:
    """[lo, hi) of the batch answered by `rank`; slices differ by at most one."""
    base, extra = divmod(q, world)
    lo = rank * base + min(rank, extra)
    return lo, lo + base + (1 if rank < extra else 0)


def assign_instances(sizes, world: int) -> np.ndarray:
    """owner[j] = rank that permutes instance j; greedy by decreasing size onto
    the least-loaded rank (ties to the lowest rank), deterministic."""
    sizes = np.asarray(sizes, dtype=np.int64)
    order = sorted(range(len(sizes)), key=lambda j: (-int(sizes[j]), j))
    heap = [(0, r) for r in range(world)]
    owner = np.empty(len(sizes), dtype=np.int64)
    for j in order:
        load, r = heapq.heappop(heap)
        owner[j] = r
        heapq.heappush(heap, (load + int(sizes[j]), r))
    return owner


def local_batch(sizes, owner, rank: int):
    """Instance ids of `rank` (ascending) and their local offset table."""
    sizes = np.asarray(sizes, dtype=np.int64)
    mine = np.nonzero(np.asarray(owner) == rank)[0]
    offsets = np.zeros(len(mine) + 1, dtype=np.int64)
    np.cumsum(sizes[mine], out=offsets[1:])
    return mine, offsets


def gather_answers(local, q: int, world: int):
    """All-gather the per-rank answer slices into the whole batch (result
    assembly, not part of the data path).  `local` is a 1-D int64 torch tensor."""
    import torch
    import torch.distributed as dist
    slices = [query_slice(q, r, world) for r in range(world)]
    width = max(hi - lo for lo, hi in slices)
    buf = torch.zeros(width, dtype=torch.int64, device=local.device)
    buf[:local.numel()] = local
    parts = [torch.empty_like(buf) for _ in range(world)]
    dist.all_gather(parts, buf)
    return torch.cat([p[:hi - lo] for p, (lo, hi) in zip(parts, slices)])
