"""Multi-GPU plumbing for batches of mask clips.

Clips are independent, so a batch shards across GPUs with no exchange on the
imaging path: each rank images its own clips (one process per GPU, launched by
torchrun).  The only reduction the path has is the source-weight gradient of
the adjoint, a sum over clips of srcSize^2 floats, done with one all-reduce.
Kernel sets are computed per rank (a few milliseconds) or broadcast once.
"""
from __future__ import annotations

import heapq


def partition(clip_pixels: list[int], world: int) -> list[list[int]]:
    """Assign clip indices to `world` ranks, balancing total pixels (longest
    processing time first).  Deterministic: equal loads break ties by rank."""
    if world <= 0:
        raise ValueError("world must be positive")
    order = sorted(range(len(clip_pixels)), key=lambda i: (-clip_pixels[i], i))
    heap = [(0, r) for r in range(world)]
    heapq.heapify(heap)
    shards: list[list[int]] = [[] for _ in range(world)]
    for i in order:
        load, r = heapq.heappop(heap)
        shards[r].append(i)
        heapq.heappush(heap, (load + clip_pixels[i], r))
    for s in shards:
        s.sort()
    return shards


def shard_for_rank(clip_pixels: list[int], rank: int, world: int) -> list[int]:
    return partition(clip_pixels, world)[rank]


def allreduce_source_gradient(grad, group=None):
    """Sum the per-rank source-weight gradients (torch tensor, in place)."""
    import torch.distributed as dist
    if dist.is_available() and dist.is_initialized() and dist.get_world_size(group) > 1:
        dist.all_reduce(grad, op=dist.ReduceOp.SUM, group=group)
    return grad


def broadcast_kernels(tensor, src: int = 0, group=None):
    """Share a kernel set computed on one rank with the others."""
    import torch.distributed as dist
    if dist.is_available() and dist.is_initialized() and dist.get_world_size(group) > 1:
        dist.broadcast(tensor, src=src, group=group)
    return tensor
