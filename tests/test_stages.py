"""The benchmark-stage harness (smallgwn_b200/stages.py) against smallgwn's harness definitions:
the CSV header and stage names (read from smallgwn's sources when they are present here), the
latency summary (mean and linearly interpolated p50 / p95, tests/benchmark_utils.cuh:64-90), the
CSV row layout, and the seeded query and ray mixes (tests/benchmark_utils.cuh:136-370)."""
from __future__ import annotations

import csv
import io
import re

import numpy as np
import pytest

from oracle.build import REFERENCE_ROOT
from smallgwn_b200 import meshes, stages

BENCH_CSV = REFERENCE_ROOT / "tests" / "benchmark_csv.cuh"
BENCH_MAIN = REFERENCE_ROOT / "tests" / "benchmark_main.cu"


@pytest.mark.skipif(not BENCH_CSV.exists(), reason="smallgwn's sources are not present")
def test_csv_header_is_smallgwns():
    text = BENCH_CSV.read_text()
    body = text[text.index("void write_header()"):]
    body = body[:body.index(";")]
    header = "".join(re.findall(r'"((?:[^"\\]|\\.)*)"', body)).replace("\\n", "")
    assert stages.CSV_HEADER == header


@pytest.mark.skipif(not BENCH_MAIN.exists(), reason="smallgwn's sources are not present")
def test_stage_names_are_smallgwns():
    text = BENCH_MAIN.read_text()
    named = re.findall(r'run_stage\(\s*"([a-z0-9_]+)"', text)
    named += ["bvh_build_{builder}"] if 'std::string("bvh_build_")' in text else []
    assert set(named) == set(stages.STAGES)


def test_latency_summary():
    samples = [4.0, 1.0, 3.0, 2.0]
    mean, p50, p95 = stages.summarize(samples)
    assert mean == 2.5 and p50 == pytest.approx(2.5) and p95 == pytest.approx(3.85)
    assert stages.percentile_ms([7.0], 0.95) == 7.0 and stages.summarize([]) == (0.0, 0.0, 0.0)
    assert stages.percentile_ms(samples, 1.5) == 4.0  # q clamped to [0, 1]


def test_csv_rows_layout():
    opts = stages.options(query_count=10, warmup_iters=1, measure_iters=2)
    ok = stages.stage_result("query_taylor_o2", "queries/s", 1, 2, 8, 12, 10, success=True, latency_mean_ms=1.5,
                             latency_p50_ms=1.25, latency_p95_ms=2.0, throughput_per_s=6666.6667)
    bad = stages._unavailable("query_antipodal_boundary", "queries/s", opts, 8, 12, stages.FUSED_ANTIPODAL)
    text = stages.csv_rows([ok, bad], {"boundary_edge_count": 3}, "m.ply", opts, "B200", 12090, "t")
    rows = list(csv.reader(io.StringIO(text)))
    header = rows[0]
    assert ",".join(header) == stages.CSV_HEADER and all(len(r) == len(header) for r in rows)
    a = dict(zip(header, rows[1]))
    b = dict(zip(header, rows[2]))
    assert (a["stage"], a["success"], a["boundary_edge_count"], a["latency_p50_ms"]) == ("query_taylor_o2", "1", "3",
                                                                                           "1.250000")
    assert (b["success"], b["error_message"]) == ("0", stages.FUSED_ANTIPODAL)
    assert a["stream_sync_per_iter"] == "1" and a["seed"] == str(0xB3A9E5D4) and a["builder"] == "hploc"


def test_query_mix():
    mesh = meshes.small_mesh()
    q = np.stack(meshes.reference_mixed_queries(mesh, 10_001, seed=5), axis=1)
    P = np.stack([mesh["x"], mesh["y"], mesh["z"]], axis=1)
    lo, hi = P.min(axis=0), P.max(axis=0)
    ctr, ext = (lo + hi) / 2, hi - lo
    assert np.allclose(q[0], ctr)
    ids = np.arange(1, q.shape[0])
    near = (ids % 10) < 7
    r = np.abs(q[1:] - ctr) / ext
    assert np.all(r[near] <= 0.85 + 1e-6)
    assert np.all((r[~near] >= 1.25 - 1e-6) & (r[~near] <= 3.25 + 1e-6))
    assert abs(near.mean() - 0.7) < 1e-3


def test_ray_mix():
    mesh = meshes.small_mesh()
    n = 4000
    ox, oy, oz, dx, dy, dz = meshes.reference_mixed_rays(mesh, n, seed=7)
    o = np.stack([ox, oy, oz], axis=1).astype(np.float64)
    d = np.stack([dx, dy, dz], axis=1).astype(np.float64)
    assert np.allclose(np.linalg.norm(d, axis=1), 1.0, atol=1e-6)
    P = np.stack([mesh["x"], mesh["y"], mesh["z"]], axis=1).astype(np.float64)
    lo, hi = P.min(axis=0), P.max(axis=0)
    ctr, ext = (lo + hi) / 2, hi - lo
    ids = np.arange(n)
    tri = (ids % 4) < 2
    t = ids[tri] % mesh["i0"].size
    cen = sum(P[mesh[f"i{j}"][t].astype(np.int64)] for j in range(3)) / 3
    dist = np.linalg.norm(o[tri] - cen, axis=1) / ext.max()
    assert np.all((dist >= 0.2 - 1e-5) & (dist <= 0.45 + 1e-5))
    towards = np.einsum("ij,ij->i", d[tri], cen - o[tri]) > 0
    assert np.all(towards[(ids[tri] % 4) == 0]) and not np.any(towards[(ids[tri] % 4) == 1])
    shell = np.abs(o[~tri] - ctr) / ext
    assert np.all(shell.max(axis=1) <= 3.2 + 1e-5)
    inward = np.einsum("ij,ij->i", d[~tri], ctr - o[~tri]) > 0
    assert np.all(inward)
