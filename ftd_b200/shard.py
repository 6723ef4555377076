"""Multi-GPU plumbing for the correlator: channels are independent HERKs, so
N GPUs run N replicas (one process and one handle per GPU) over disjoint
channel sets, with no exchange step.

* ``partition_channels`` balances a channel list over ranks by the work of
  each channel, 8 N_f (N_f + 1) / 2 K_f, longest first (LPT), as the
  batched entry point orders its tiles.
* ``max_over_ranks`` is the timing reduction of a multi-rank measurement (the
  slowest rank sets the step time).
* ``gather_to_rank0`` collects per-rank results on rank 0 (host objects).

All of it is host logic over ``torch.distributed``; it runs with the ``nccl``
backend on GPUs and with ``gloo`` on CPU.
"""
from __future__ import annotations

import heapq
from typing import Sequence


def channel_cost(n_inputs: int, k: int) -> float:
    """Work of one channel: 8 N(N+1)/2 K real operations."""
    return 8.0 * n_inputs * (n_inputs + 1) / 2.0 * k


def partition_channels(shapes: Sequence[tuple[int, int]], world: int) -> list[list[int]]:
    """Assign channel indices to ``world`` ranks, largest first to the least
    loaded rank (LPT).  ``shapes`` holds (n_inputs, K) per channel.  Returns one
    sorted index list per rank; together they cover every channel once."""
    if world < 1:
        raise ValueError("world must be >= 1")
    order = sorted(range(len(shapes)), key=lambda c: (-channel_cost(*shapes[c]), c))
    heap = [(0.0, r) for r in range(world)]
    heapq.heapify(heap)
    parts: list[list[int]] = [[] for _ in range(world)]
    for c in order:
        load, r = heapq.heappop(heap)
        parts[r].append(c)
        heapq.heappush(heap, (load + channel_cost(*shapes[c]), r))
    return [sorted(p) for p in parts]


def rank_load(shapes: Sequence[tuple[int, int]], part: Sequence[int]) -> float:
    return sum(channel_cost(*shapes[c]) for c in part)


def max_over_ranks(value: float, dist=None, device=None) -> float:
    """Maximum of a per-rank scalar over all ranks (the value itself without a
    process group)."""
    if dist is None or not dist.is_initialized():
        return float(value)
    import torch
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def gather_to_rank0(obj, dist=None):
    """List of every rank's ``obj`` on rank 0 (None elsewhere); [obj] alone."""
    if dist is None or not dist.is_initialized():
        return [obj]
    out = [None] * dist.get_world_size() if dist.get_rank() == 0 else None
    dist.gather_object(obj, out, dst=0)
    return out
