"""Box sharding for batched boxes on several GPUs (one process per GPU).

Boxes are independent, so a batch shards with no collective in the step:
each rank steps the boxes assigned to it as one batch (fluid_batch_*), and
only the per-box statistics (and timings) are combined at the end. Boxes go
to ranks by LPT (longest processing time first): boxes in order of falling
particle count, each to the rank with the least particles so far (ties to
the lowest rank), which bounds the largest rank's load by 4/3 of the optimum.
"""
import heapq

import numpy as np


def lpt_shards(counts, world):
    """Box indices per rank: LPT on particle counts, each list ascending."""
    if world < 1:
        raise ValueError("world must be >= 1")
    order = sorted(range(len(counts)), key=lambda b: (-int(counts[b]), b))
    heap = [(0, r) for r in range(world)]
    shards = [[] for _ in range(world)]
    for b in order:
        load, r = heapq.heappop(heap)
        shards[r].append(b)
        heapq.heappush(heap, (load + int(counts[b]), r))
    return [sorted(s) for s in shards]


def shard_loads(counts, shards):
    return [int(sum(int(counts[b]) for b in s)) for s in shards]


def gather_box_values(local_boxes, local_values, nboxes, group=None, device="cpu"):
    """Every rank's per-box rows (local_values[k] belongs to box
    local_boxes[k]) assembled into one [nboxes, width] float64 array on
    every rank: each rank fills its boxes' rows of a zero array and the
    ranks sum them (one all_reduce; a box lives on exactly one rank)."""
    import torch
    import torch.distributed as dist
    vals = np.asarray(local_values, np.float64)
    width = vals.shape[1] if vals.ndim == 2 else 1
    full = torch.zeros((nboxes, width), dtype=torch.float64, device=device)
    if len(local_boxes):
        idx = torch.as_tensor(np.asarray(local_boxes, np.int64), device=device)
        full[idx] = torch.as_tensor(vals.reshape(len(local_boxes), width), device=device)
    if dist.is_available() and dist.is_initialized():
        dist.all_reduce(full, op=dist.ReduceOp.SUM, group=group)
    return full.cpu().numpy()
