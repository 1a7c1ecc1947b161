"""Work division over several ranks, on the CPU: contiguous query ranges, the longest-processing-
time-first mesh partition, the packed all-reduce that completes a split adjoint's dL/dV, and the
max-over-ranks of device times -- single-process properties plus world-size-2 `gloo` runs."""
from __future__ import annotations

import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

from smallgwn_b200 import sharding


@pytest.mark.parametrize("n, world", [(0, 1), (0, 3), (1, 2), (7, 3), (10_000_000, 8), (5, 8)])
def test_shard_ranges_cover_once_in_order(n, world):
    ranges = [sharding.shard_range(n, r, world) for r in range(world)]
    assert ranges[0][0] == 0 and ranges[-1][1] == n
    for (a, b), (c, d) in zip(ranges, ranges[1:]):
        assert b == c and a <= b
    sizes = [b - a for a, b in ranges]
    assert max(sizes) - min(sizes) <= 1 and sizes == sorted(sizes, reverse=True)


def test_shard_range_refuses_bad_arguments():
    with pytest.raises(ValueError):
        sharding.shard_range(10, 2, 2)
    with pytest.raises(ValueError):
        sharding.shard_range(-1, 0, 1)
    with pytest.raises(ValueError):
        sharding.lpt_partition([1.0], 0)


def test_lpt_partition_properties():
    rng = np.random.default_rng(4)
    tris = np.exp(rng.uniform(np.log(1e3), np.log(2e5), 256))
    nqs = np.exp(rng.uniform(np.log(1e4), np.log(1e6), 256)).astype(np.int64)
    costs = [sharding.mesh_cost(int(t), int(q)) for t, q in zip(tris, nqs)]
    for world in (1, 2, 3, 4, 8):
        parts = sharding.lpt_partition(costs, world)
        assert sorted(i for p in parts for i in p) == list(range(256))
        assert all(p == sorted(p) for p in parts)
        loads = [sum(costs[i] for i in p) for p in parts]
        lower = max(max(costs), sum(costs) / world)  # no partition does better than this
        # greedy list scheduling: the last item on the busiest rank started below the mean load
        assert lower <= max(loads) <= sum(costs) / world + max(costs)
        assert max(loads) <= 1.05 * lower  # many small items: LPT lands within a few percent
        assert sharding.lpt_partition(costs, world) == parts  # deterministic


def test_lpt_on_a_known_case():
    # Graham's tight example for two machines: 3, 3, 2, 2, 2 -> LPT makespan 7, optimum 6
    parts = sharding.lpt_partition([3, 3, 2, 2, 2], 2)
    loads = sorted(sum([3, 3, 2, 2, 2][i] for i in p) for p in parts)
    assert loads == [5, 7]
    assert sharding.lpt_partition([5.0, 1.0, 1.0], 4) == [[0], [1], [2], []]


def test_mesh_cost_is_monotone():
    assert sharding.mesh_cost(2000, 10) < sharding.mesh_cost(4000, 10) < sharding.mesh_cost(4000, 10_000)
    assert sharding.bvh4_depth(1) == 1.0 and sharding.bvh4_depth(2 * 4 ** 5) == pytest.approx(6.0)


def test_single_process_helpers_are_identities():
    import torch

    t = torch.arange(6, dtype=torch.float32)
    sharding.allreduce_sum_([t])
    assert t.tolist() == list(range(6))
    assert sharding.max_over_ranks([1.5, 2.0]) == [1.5, 2.0]
    assert sharding.sum_over_ranks([3.0]) == [3.0]


# ---- world size 2 over gloo -------------------------------------------------------------------------

def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _per_query_vertex_gradient(V: np.ndarray, Q: np.ndarray, g: np.ndarray) -> np.ndarray:
    """A stand-in adjoint with the same structure as dL/dV: each query adds g_q times a smooth
    function of (vertex, query) to every vertex (sum over queries)."""
    d = V[:, None, :] - Q[None, :, :]
    r2 = (d * d).sum(-1) + 1.0
    return ((g[None, :, None] * d) / r2[..., None] ** 1.5).sum(1)


def _worker(rank: int, world: int, port: int, out_dir: str) -> None:
    import torch
    import torch.distributed as dist
    from datetime import timedelta

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=60))
    try:
        rng = np.random.default_rng(11)
        V = rng.normal(size=(40, 3))
        Q = rng.normal(size=(1001, 3)) * 2
        g = rng.normal(size=1001)
        lo, hi = sharding.shard_range(Q.shape[0], rank, world)
        part = _per_query_vertex_gradient(V, Q[lo:hi], g[lo:hi])
        dV = [torch.from_numpy(np.ascontiguousarray(part[:, k])) for k in range(3)]
        sharding.allreduce_sum_(dV)  # packed: one all-reduce for the three columns
        got = torch.stack(dV, -1).numpy()
        full = _per_query_vertex_gradient(V, Q, g)
        np.testing.assert_allclose(got, full, rtol=1e-12, atol=1e-12)
        # a single contiguous tensor takes the direct path
        single = torch.from_numpy(part.copy())
        sharding.allreduce_sum_([single])
        np.testing.assert_allclose(single.numpy(), full, rtol=1e-12, atol=1e-12)

        # every rank derives the same partition by itself
        costs = [sharding.mesh_cost(1000 * (i % 7 + 1), 5000 * (i % 5 + 1)) for i in range(37)]
        parts = sharding.lpt_partition(costs, world)
        gathered = [None] * world
        dist.all_gather_object(gathered, (rank, parts[rank], parts))
        assert all(p == parts for _, _, p in gathered)
        mine = sorted(i for _, m, _ in gathered for i in m)
        assert mine == list(range(37))

        # the job's time is its slowest rank's
        mx = sharding.max_over_ranks([10.0 + rank, 5.0 - rank])
        assert mx == [10.0 + world - 1, 5.0]
        # and its launch count is every rank's
        assert sharding.sum_over_ranks([7.0, float(rank)]) == [7.0 * world, float(sum(range(world)))]
        with open(os.path.join(out_dir, f"ok{rank}"), "w") as f:
            f.write("ok")
    finally:
        dist.destroy_process_group()


def test_two_ranks_over_gloo(tmp_path):
    world = 2
    mp.start_processes(_worker, args=(world, _free_port(), str(tmp_path)), nprocs=world, join=True,
                       start_method="spawn")
    assert sorted(p.name for p in tmp_path.iterdir()) == ["ok0", "ok1"]
