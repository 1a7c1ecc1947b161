"""Benchmark: Taylor winding queries/s on a 1M-triangle mesh (one JSON line on rank 0).

Workload (per rank): displaced UV sphere 1024 x 512 (1,046,528 triangles, seed 2), 10M mixed
queries (half uniform in the 1.2x bounding box, half at surface samples offset along the normal by
N(0, 1e-3), seed 2 + rank), H-PLOC (radius 8) BVH4, Taylor order 2 at accuracy scale 3.5,
compensated near field. A step is one call of the Taylor batch on the 10M device-resident queries
(Morton ordering of the queries included).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

For N > 1 run one process per GPU with torch.distributed.run; every rank processes its own 10M
queries against its own copy of the BVH (queries are independent: weak scaling, no data-path
collective; the only collective is the max over ranks of the measured time).
``--impl reference`` times the CPU implementation of the same path (the oracle's port of the
reference traversal, all host threads) on bounded samples of the same workload.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

METRIC = "Winding queries/s at 1M tris (chosen vs plain form, max err ≤1e-3 vs FP64)"
ORDER = 2
# Order 2 needs accuracy scale >= 3.25 for max |err| <= 1e-3 against FP64 on this workload
# (2.0: 9.2e-3, 3.0: 1.5e-3, 3.25: 9.8e-4, 3.5: 6.4e-4 on the 100k-query subset).
BETA = 3.5
N_QUERIES = 10_000_000
ERROR_SUBSET = 100_000
MOMENT_BYTES = {0: 112, 1: 208, 2: 368}


def parse() -> argparse.Namespace:
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--queries", type=int, default=N_QUERIES)
    ap.add_argument("--order", type=int, default=ORDER)
    ap.add_argument("--beta", type=float, default=BETA)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--profile", choices=["taylor", "taylor-plain", "taylor-thread", "build", "exact"], default=None,
                    help="run one small workload for a profiler (no JSON): 2 launches of the kernel")
    return ap.parse_args()


def run_profile(args) -> None:
    """Self-contained launches for ncu: the traversal kernel over pre-ordered queries (`taylor`:
    the timed form, warp-cooperative with the compensated near field; `taylor-plain`: FP32 near
    field; `taylor-thread`: one traversal per thread, FP32 near field), one H-PLOC build (`build`)
    or the exact batch on the small icosphere (`exact`). Uses --queries and --order / --beta."""
    import torch

    import smallgwn_b200 as g
    from smallgwn_b200 import api, meshes

    stream = torch.cuda.current_stream()
    if args.profile == "exact":
        mesh = meshes.small_mesh()
        q = meshes.small_queries(100_000)
    else:
        mesh = meshes.sphere_mesh()
        q = meshes.mixed_queries(mesh, args.queries, seed=2)
    geo = g.gwn_geometry_object()
    assert g.gwn_upload_geometry(geo, mesh["x"], mesh["y"], mesh["z"], mesh["i0"], mesh["i1"], mesh["i2"]).is_ok()
    bvh = g.gwn_bvh4_object()
    method = 1 if args.profile == "exact" else 0
    assert g.gwn_build_bvh(geo, bvh, g.gwn_bvh_build_options(method=method, hploc_search_radius=8)).is_ok()
    if args.profile == "build":
        for _ in range(2):
            assert g.gwn_build_bvh(geo, bvh, g.gwn_bvh_build_options(method=0, hploc_search_radius=8)).is_ok()
        torch.cuda.synchronize()
        print("profile build ok")
        return
    dq = [torch.from_numpy(v).to("cuda") for v in q]
    out = torch.empty_like(dq[0])
    if args.profile == "exact":
        for _ in range(2):
            assert g.gwn_compute_winding_number_exact_batch(bvh, *dq, out).is_ok()
        torch.cuda.synchronize()
        print("profile exact ok")
        return
    mom = g.gwn_bvh4_moment_object(args.order)
    assert g.gwn_refit_bvh_moment(args.order, bvh, mom).is_ok()
    order = torch.empty(dq[0].numel(), dtype=torch.int32, device="cuda")
    assert api.query_order(bvh, *dq, order).is_ok()
    sq = [d[order.long()].contiguous() for d in dq]
    precision = g.near_precision.compensated if args.profile == "taylor" else g.near_precision.plain
    for _ in range(2):
        assert g.gwn_compute_winding_number_taylor_batch(args.order, bvh, mom, *sq, out, accuracy_scale=args.beta,
                                                         stream=stream, sort_queries=False, precision=precision,
                                                         per_thread=args.profile == "taylor-thread").is_ok()
    torch.cuda.synchronize()
    print(f"profile {args.profile} ok")


def dist_setup(n: int):
    import torch
    import torch.distributed as dist

    if n <= 1 or "RANK" not in os.environ:
        return 0, 1, None
    rank = int(os.environ["RANK"])
    world = int(os.environ["WORLD_SIZE"])
    local = int(os.environ.get("LOCAL_RANK", rank))
    torch.cuda.set_device(local)
    from datetime import timedelta

    dist.init_process_group("nccl", timeout=timedelta(seconds=300), device_id=torch.device("cuda", local))
    return rank, world, dist


class ClockSampler:
    """nvidia-smi clock / throttle sampling during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int):
        self.device = device
        self.proc = None
        self.file = None

    def __enter__(self):
        try:
            self.file = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.device}", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "200"], stdout=self.file, stderr=subprocess.DEVNULL)
        except (OSError, FileNotFoundError):
            self.proc = None
        return self

    def __exit__(self, *exc):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self) -> dict:
        if self.file is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.file.flush()
        rows = [ln.split(",") for ln in Path(self.file.name).read_text().splitlines() if ln.count(",") >= 8]
        os.unlink(self.file.name)
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["no samples"]}
        sm = [float(r[1]) for r in rows]
        mx = max(float(r[2]) for r in rows)
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[k] for r in rows for k in range(4) if r[5 + k].strip().lower().startswith("active")})
        loaded = [s for s in sm if s > 0.5 * mx] or sm
        return {"sm_mhz": statistics.median(loaded), "sm_max_mhz": mx, "reasons": reasons, "samples": len(rows)}


def peaks() -> dict:
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        d = json.loads(p.read_text())
        return {"hbm_gbs": float(d["hbm_gbs"]), "source": "measured"}
    return {"hbm_gbs": 6650.0, "source": "fallback"}


def profiled_traffic(order: int, beta: float, n: int) -> float | None:
    """DRAM bytes (read + write) of one traversal launch over this workload, from the committed
    ncu summary of the same launch (profiles/taylor_warp_o{order}_sphere1m.md); None when no
    capture of this exact configuration is recorded."""
    path = ROOT / "profiles" / f"taylor_warp_o{order}_sphere1m.md"
    if not path.exists():
        return None
    key = f"dram_bytes_per_launch[order={order},beta={beta:g},queries={n}]:"
    for line in path.read_text().splitlines():
        if line.startswith(key):
            return float(line.split(":", 1)[1].split()[0])
    return None


def make_workload(rank: int, n_queries: int):
    from smallgwn_b200 import meshes

    mesh = meshes.sphere_mesh()
    q = meshes.mixed_queries(mesh, n_queries, seed=2 + rank)
    return mesh, q


def cpu_baseline(mesh, bvh_host, mom_host, q, order, beta, budget_s=12.0) -> dict:
    """The oracle's port of the reference Taylor traversal on all host threads, bounded sample."""
    import oracle

    threads = oracle.max_threads()
    chunk = 20_000
    done = 0
    t0 = time.perf_counter()
    while time.perf_counter() - t0 < budget_s and done < q[0].size:
        sl = slice(done, min(done + chunk, q[0].size))
        oracle.taylor(order, bvh_host["nodes"], mom_host, bvh_host["triangles"], bvh_host["root_reference"],
                      q[0][sl], q[1][sl], q[2][sl], beta=beta, threads=threads)
        done = sl.stop
    dt = time.perf_counter() - t0
    return {"value": done / dt, "unit": "queries/s", "cores": threads, "kind": "port",
            "sample": f"{done} of the {q[0].size} queries (order {order}, beta {beta}) in {dt:.1f} s"}


def run_reference_arm(args) -> None:
    """CPU implementation of the path, same metric and config, bounded samples per step."""
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    import torch

    import oracle
    import smallgwn_b200 as g
    from smallgwn_b200 import api

    mesh, q = make_workload(0, args.queries)
    # The BVH and moments the CPU traverses are the same ones the GPU path uses.
    geo = g.gwn_geometry_object()
    assert g.gwn_upload_geometry(geo, mesh["x"], mesh["y"], mesh["z"], mesh["i0"], mesh["i1"], mesh["i2"]).is_ok()
    bvh = g.gwn_bvh4_object()
    assert g.gwn_build_bvh(geo, bvh, g.gwn_bvh_build_options(method=0, hploc_search_radius=8)).is_ok()
    mom = g.gwn_bvh4_moment_object(args.order)
    assert g.gwn_refit_bvh_moment(args.order, bvh, mom).is_ok()
    bh = api.bvh_host_arrays(bvh)
    mh = api.moment_host_array(mom)
    torch.cuda.synchronize()
    threads = oracle.max_threads()
    sample = 40_000
    rng = np.random.default_rng(0)

    def step():
        idx = rng.integers(0, q[0].size, sample)
        t0 = time.perf_counter()
        oracle.taylor(args.order, bh["nodes"], mh, bh["triangles"], bh["root_reference"], q[0][idx], q[1][idx],
                      q[2][idx], beta=args.beta, threads=threads)
        return time.perf_counter() - t0

    for _ in range(args.warmup):
        step()
    total = sum(step() for _ in range(args.steps))
    value = sample * args.steps / total
    line = {
        "metric": METRIC, "value": value, "unit": "queries/s", "n_gpus": args.gpus, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": total / args.steps * 1e3, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic", "impl": "reference",
        "config": config_dict(args, mesh),
        "cpu_baseline": {"value": value, "unit": "queries/s", "cores": threads, "kind": "port",
                         "sample": f"{sample} random queries of the workload per step, Taylor order {args.order}, "
                                   f"beta {args.beta}, {threads} host threads"},
        "e2e": {"value": value, "unit": "queries/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def config_dict(args, mesh) -> dict:
    return {"workload": "displaced UV sphere 1024x512 (1,046,528 tris), 10M mixed queries per GPU",
            "triangles": int(mesh["i0"].size), "queries_per_gpu": int(args.queries), "builder": "hploc r=8",
            "width": 4, "taylor_order": int(args.order), "accuracy_scale": float(args.beta),
            "near_field": "compensated fp32 (fp64 on flagged triangles)", "query_order": "morton-sorted in batch",
            "l2": "flushed (256 MiB write) between timed steps", "parallelism": f"replicas x{args.gpus}"}


def main() -> None:
    args = parse()
    if args.profile is not None:
        run_profile(args)
        return
    if args.impl == "reference":
        run_reference_arm(args)
        return
    import torch

    import smallgwn_b200 as g
    from smallgwn_b200 import api

    rank, world, dist = dist_setup(args.gpus)
    dev = torch.cuda.current_device()
    stream = torch.cuda.current_stream()
    mesh, q = make_workload(rank, args.queries)
    n = q[0].size

    geo = g.gwn_geometry_object()
    st = g.gwn_upload_geometry(geo, mesh["x"], mesh["y"], mesh["z"], mesh["i0"], mesh["i1"], mesh["i2"], stream)
    assert st.is_ok(), st.message
    bvh = g.gwn_bvh4_object()
    t0 = time.perf_counter()
    st = g.gwn_build_bvh(geo, bvh, g.gwn_bvh_build_options(method=0, hploc_search_radius=8), stream)
    assert st.is_ok(), st.message
    torch.cuda.synchronize()
    build_ms = (time.perf_counter() - t0) * 1e3
    mom = g.gwn_bvh4_moment_object(args.order)
    assert g.gwn_refit_bvh_moment(args.order, bvh, mom, stream).is_ok()

    dq = [torch.from_numpy(v).to("cuda") for v in q]
    out = torch.empty(n, dtype=torch.float32, device="cuda")
    flush = torch.empty(256 << 20, dtype=torch.uint8, device="cuda")

    def batch(qs, o, sort=True, precision=g.near_precision.compensated, per_thread=False):
        st = g.gwn_compute_winding_number_taylor_batch(args.order, bvh, mom, *qs, o, accuracy_scale=args.beta,
                                                       stream=stream, sort_queries=sort, precision=precision,
                                                       per_thread=per_thread)
        assert st.is_ok(), st.message

    def plain_batch(qs, o):
        # the plain per-call FP32 form: one independent traversal per thread in input order, FP32
        # near field -- the structure of smallgwn's own batch kernel
        batch(qs, o, sort=False, precision=g.near_precision.plain, per_thread=True)

    for _ in range(args.warmup):
        batch(dq, out)
    torch.cuda.synchronize()

    # ---- timed region: K steps, L2 flushed between steps, CUDA events on the launching stream ----
    events = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
    if dist is not None:
        dist.barrier()
    torch.cuda.synchronize()
    with ClockSampler(dev) as clocks:
        for e0, e1 in events:
            flush.fill_(1)
            e0.record(stream)
            batch(dq, out)
            e1.record(stream)
        torch.cuda.synchronize()
    if dist is not None:
        dist.barrier()
    torch.cuda.synchronize()
    total_ms = sum(a.elapsed_time(b) for a, b in events)
    t = torch.tensor([total_ms], dtype=torch.float64, device="cuda")
    if dist is not None:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    total_ms = float(t.item())
    value = world * n * args.steps / (total_ms / 1e3)

    # ---- end to end through the public API with host buffers (pinned), same step definition ----
    hq = [torch.from_numpy(v).pin_memory() for v in q]
    hout = torch.empty(n, dtype=torch.float32).pin_memory()
    e2e_q = [torch.empty(n, dtype=torch.float32, device="cuda") for _ in range(3)]
    e2e_steps = max(3, min(args.steps, 10))

    def e2e_step():
        for d, h in zip(e2e_q, hq):
            d.copy_(h, non_blocking=True)
        batch(e2e_q, out)
        hout.copy_(out, non_blocking=True)

    e2e_step()
    torch.cuda.synchronize()
    e2e_events = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(e2e_steps)]
    if dist is not None:
        dist.barrier()
    for e0, e1 in e2e_events:
        flush.fill_(1)
        e0.record(stream)
        e2e_step()
        e1.record(stream)
    torch.cuda.synchronize()
    e2e_ms = sum(a.elapsed_time(b) for a, b in e2e_events)
    t = torch.tensor([e2e_ms], dtype=torch.float64, device="cuda")
    if dist is not None:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    e2e_value = world * n * e2e_steps / (float(t.item()) / 1e3)

    # ---- plain per-call FP32 form (same queries and accuracy scale; not part of `value`) ----
    plain_events = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(3)]
    plain_batch(dq, out)
    for e0, e1 in plain_events:
        flush.fill_(1)
        e0.record(stream)
        plain_batch(dq, out)
        e1.record(stream)
    torch.cuda.synchronize()
    plain_ms = sum(a.elapsed_time(b) for a, b in plain_events) / len(plain_events)

    # ---- dominant kernel alone: traversal over pre-ordered queries (one launch) ----
    order = torch.empty(n, dtype=torch.int32, device="cuda")
    assert api.query_order(bvh, *dq, order, stream).is_ok()
    idx = order.long()
    sq = [d[idx].contiguous() for d in dq]
    batch(sq, out, sort=False)
    kev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(3)]
    for e0, e1 in kev:
        flush.fill_(1)
        e0.record(stream)
        batch(sq, out, sort=False)
        e1.record(stream)
    torch.cuda.synchronize()
    kernel_ms = sum(a.elapsed_time(b) for a, b in kev) / len(kev)
    stats = [torch.empty(n, dtype=torch.int32, device="cuda") for _ in range(3)]
    assert api.taylor_traversal_stats(bvh, mom, *dq, *stats, accuracy_scale=args.beta, stream=stream).is_ok()
    torch.cuda.synchronize()
    nodes_entered = float(stats[0].double().sum().item())
    near_tris = float(stats[2].double().sum().item())
    alg_bytes = n * 16 + nodes_entered * (128 + MOMENT_BYTES[args.order]) + near_tris * 36
    pk = peaks()
    achieved = alg_bytes / (kernel_ms / 1e3) / 1e9
    traffic = profiled_traffic(args.order, args.beta, n)

    # ---- accuracy against FP64 on a 100k subset (untimed) ----
    sub = slice(0, min(ERROR_SUBSET, n))
    ref64 = torch.empty(sub.stop, dtype=torch.float64, device="cuda")
    assert api.exact_winding_fp64(geo, *[d[sub] for d in dq], ref64, stream).is_ok()
    batch(dq, out)
    torch.cuda.synchronize()
    err = (out[sub].double() - ref64).abs().cpu().numpy()
    plain_out = torch.empty_like(out)
    plain_batch(dq, plain_out)
    torch.cuda.synchronize()
    perr = (plain_out[sub].double() - ref64).abs().cpu().numpy()

    cpu = None
    if rank == 0 and not args.no_cpu_baseline:
        cpu = cpu_baseline(mesh, api.bvh_host_arrays(bvh), api.moment_host_array(mom), q, args.order, args.beta)

    if rank == 0:
        cfg = config_dict(args, mesh)
        cfg.update({"max_err_vs_fp64": float(err.max()), "p99_err_vs_fp64": float(np.quantile(err, 0.99)),
                    "error_subset": int(sub.stop),
                    "plain_form_queries_per_s": world * n / (plain_ms / 1e3),
                    "plain_form_max_err_vs_fp64": float(perr.max()),
                    "chosen_over_plain": (value / world) / (n / (plain_ms / 1e3)),
                    "build_ms_hploc": build_ms, "bvh_nodes": int(bvh.accessor().node_count),
                    "fp64_fallbacks_per_batch": api.fp64_fallback_count(bvh, stream)})
        launches_per_step = 7  # query codes, sort histogram, 4 digit passes, traversal
        line = {
            "metric": METRIC, "value": value, "unit": "queries/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": total_ms / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic", "config": cfg,
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": pk["hbm_gbs"], "unit": "GB/s",
                         "frac": achieved / pk["hbm_gbs"], "peak_source": pk["source"],
                         "traffic": traffic,
                         "kernel": "k_taylor_warp (traversal, compensated, pre-ordered queries)",
                         "kernel_ms": kernel_ms,
                         "algorithmic_bytes": alg_bytes,
                         "bytes_model": "16 B/query + (128 B node + moment node) per node entered + 36 B per exact triangle"},
            "cpu_baseline": cpu,
            "e2e": {"value": e2e_value, "unit": "queries/s", "h2d_bytes_per_step": 12 * n, "d2h_bytes_per_step": 4 * n},
            "gpu_launches": launches_per_step * args.steps,
            "clocks": clocks.summary(),
        }
        print(json.dumps(line), flush=True)
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
