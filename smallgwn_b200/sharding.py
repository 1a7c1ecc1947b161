"""Work division for several GPUs (one process per GPU).

Queries are independent, so the forward path runs as replicas (every rank builds the same BVH;
the build is deterministic) or with the query batch split into contiguous ranges. Two steps do
exchange data:

- the adjoint's dL/dV is a sum over all queries; with the queries of one mesh split over ranks
  each rank holds a partial sum and one all-reduce (sum) of the packed V x 3 buffer completes it
  (dL/dq stays with the rank that owns the query);
- batched dynamic meshes are divided whole among ranks by a longest-processing-time-first
  assignment on a cost model of the per-frame work (refit and moments ~ T log T, queries
  ~ Q x tree depth), with no exchange at all.
"""
from __future__ import annotations

import math
from typing import Sequence


def shard_range(n: int, rank: int, world: int) -> tuple[int, int]:
    """[start, stop) of rank's contiguous share of n items; shares differ by at most one item and
    the lower ranks take the larger ones."""
    if world < 1 or not 0 <= rank < world:
        raise ValueError(f"rank {rank} outside a world of {world}")
    if n < 0:
        raise ValueError("negative item count")
    base, extra = divmod(n, world)
    start = rank * base + min(rank, extra)
    return start, start + base + (1 if rank < extra else 0)


def bvh4_depth(triangles: int, leaf_size: float = 2.0) -> float:
    """Expected depth of a BVH4 over `triangles` primitives (levels of a 4-ary tree over the leaves)."""
    leaves = max(triangles / leaf_size, 1.0)
    return max(math.log(leaves, 4.0), 0.0) + 1.0


def mesh_cost(triangles: int, queries: int) -> float:
    """Per-frame cost model of one mesh: T log2 T (refit + moment refit) + Q x depth (queries)."""
    t = max(int(triangles), 1)
    return t * math.log2(t + 1) + max(int(queries), 0) * bvh4_depth(t)


def lpt_partition(costs: Sequence[float], world: int) -> list[list[int]]:
    """Longest processing time first: items by decreasing cost (ties by index) each go to the rank
    with the least load so far (ties to the lower rank). Deterministic, so every rank computes the
    same partition without communicating. The makespan is at most 4/3 - 1/(3 world) of the optimum
    (Graham 1969). Returns each rank's item indices in ascending order."""
    if world < 1:
        raise ValueError("world must be positive")
    order = sorted(range(len(costs)), key=lambda i: (-float(costs[i]), i))
    load = [0.0] * world
    parts: list[list[int]] = [[] for _ in range(world)]
    for i in order:
        r = min(range(world), key=lambda k: (load[k], k))
        parts[r].append(i)
        load[r] += float(costs[i])
    return [sorted(p) for p in parts]


def allreduce_sum_(tensors, group=None) -> None:
    """Sums each tensor over the ranks of `group`, in place, with one all-reduce of a packed
    buffer (a single launch and a single message instead of one per tensor)."""
    import torch
    import torch.distributed as dist

    tensors = list(tensors)
    if not tensors or not dist.is_initialized() or dist.get_world_size(group) == 1:
        return
    if len(tensors) == 1 and tensors[0].is_contiguous():
        dist.all_reduce(tensors[0], op=dist.ReduceOp.SUM, group=group)
        return
    flat = torch.cat([t.reshape(-1) for t in tensors])
    dist.all_reduce(flat, op=dist.ReduceOp.SUM, group=group)
    off = 0
    for t in tensors:
        n = t.numel()
        t.copy_(flat[off:off + n].view_as(t))
        off += n


def _device_for(group):
    import torch
    import torch.distributed as dist

    return torch.device("cuda", torch.cuda.current_device()) if dist.get_backend(group) == "nccl" else torch.device("cpu")


def max_over_ranks(values, group=None) -> list[float]:
    """Element-wise maximum of a list of floats over the ranks of `group` (device times: the job
    takes as long as its slowest rank). Identity without an initialised process group."""
    import torch
    import torch.distributed as dist

    vals = [float(v) for v in values]
    if not dist.is_initialized() or dist.get_world_size(group) == 1:
        return vals
    t = torch.tensor(vals, dtype=torch.float64, device=_device_for(group))
    dist.all_reduce(t, op=dist.ReduceOp.MAX, group=group)
    return [float(x) for x in t.cpu().tolist()]


def sum_over_ranks(values, group=None) -> list[float]:
    """Element-wise sum of a list of floats over the ranks of `group` (whole-job counts).
    Identity without an initialised process group."""
    import torch
    import torch.distributed as dist

    vals = [float(v) for v in values]
    if not dist.is_initialized() or dist.get_world_size(group) == 1:
        return vals
    t = torch.tensor(vals, dtype=torch.float64, device=_device_for(group))
    dist.all_reduce(t, op=dist.ReduceOp.SUM, group=group)
    return [float(x) for x in t.cpu().tolist()]
