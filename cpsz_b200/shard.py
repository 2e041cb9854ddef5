"""Multi-GPU batched compression: fields sharded across ranks.

Fields of a batch are independent, so a batch shards by field with no data
exchange: one process per GPU compresses the fields it owns into ordinary
2D offline blobs (each byte-identical to the single-field call), and the
only collective is a sum-all-reduce of the per-field blob sizes, after which
every rank knows where each blob sits in the batch's concatenation (field
order).  Writing that concatenation needs no further communication: each
rank writes its own blobs at their offsets into one file.

A single field does not shard: its Lorenzo recurrence is serial across the
whole field, so one field runs on one GPU (replicas at the job level).

Ownership is the greedy longest-processing-time rule over field sizes (points):
fields in decreasing size, ties by index, each to the least-loaded rank, ties
to the lowest rank.  It is a pure function of the shapes, so every rank
computes the same partition without communicating.
"""
from __future__ import annotations

import heapq
import os
from dataclasses import dataclass

import numpy as np


def partition(sizes, world: int) -> list[list[int]]:
    """Field indices owned by each of `world` ranks (each list ascending)."""
    if world < 1:
        raise ValueError("world must be >= 1")
    order = sorted(range(len(sizes)), key=lambda k: (-int(sizes[k]), k))
    heap = [(0, r) for r in range(world)]
    own: list[list[int]] = [[] for _ in range(world)]
    for k in order:
        load, r = heapq.heappop(heap)
        own[r].append(k)
        heapq.heappush(heap, (load + int(sizes[k]), r))
    return [sorted(o) for o in own]


@dataclass
class ShardResult:
    own: list            # field indices this rank compressed
    blobs: dict          # field index -> blob (bytes) of this rank's fields
    sizes: np.ndarray    # blob size of every field of the batch (after the all-reduce)
    offsets: np.ndarray  # n + 1 offsets of the blobs in the batch's concatenation


def _default_compress(ctx):
    from . import compress_2d_batch

    return lambda fields, ebs: compress_2d_batch(fields, ebs, ctx=ctx)


def compress_2d_batch_sharded(shapes, ebs, get_field, *, group=None, ctx=None, compress=None,
                              out_path: str | None = None) -> ShardResult:
    """Compresses this rank's share of a batch of 2D fields.

    shapes: (r1, r2) of every field of the batch (the same list on every rank);
    ebs: the fields' bounds; get_field(k) -> (U, V) for a field this rank owns
    (host arrays or device tensors, as ``compress_2d_batch`` takes them).
    The rank and world come from ``torch.distributed`` (group ``group``) when it
    is initialised, else the call is the whole batch on one rank.  With
    ``out_path`` every rank writes its blobs at their offsets into that file,
    which then holds the concatenation of all blobs in field order.
    """
    import torch
    import torch.distributed as dist

    distributed = dist.is_available() and dist.is_initialized()
    rank = dist.get_rank(group) if distributed else 0
    world = dist.get_world_size(group) if distributed else 1
    n = len(shapes)
    if len(ebs) != n:
        raise ValueError("shapes and ebs differ in length")
    own = partition([int(r1) * int(r2) for r1, r2 in shapes], world)[rank]
    compress = compress or _default_compress(ctx)
    blobs = dict(zip(own, compress([get_field(k) for k in own], [ebs[k] for k in own]))) if own else {}
    local = np.zeros(n, np.int64)
    for k, b in blobs.items():
        local[k] = len(b)
    if distributed:
        dev = "cuda" if dist.get_backend(group) == "nccl" else "cpu"
        t = torch.from_numpy(local).to(dev)
        dist.all_reduce(t, op=dist.ReduceOp.SUM, group=group)
        sizes = t.cpu().numpy()
    else:
        sizes = local
    offsets = np.zeros(n + 1, np.int64)
    np.cumsum(sizes, out=offsets[1:])
    if out_path is not None:
        fd = os.open(out_path, os.O_WRONLY | os.O_CREAT, 0o644)
        try:
            if rank == 0:
                os.ftruncate(fd, int(offsets[-1]))
            for k, b in blobs.items():
                os.pwrite(fd, b, int(offsets[k]))
        finally:
            os.close(fd)
        if distributed:
            dist.barrier(group)
    return ShardResult(own, blobs, sizes, offsets)
