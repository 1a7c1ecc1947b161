"""smallgwn's benchmark harness over this library: the same stages, the same timing rule and the
same CSV, so that a row measured here lines up with the row smallgwn's own harness writes for the
same model.

Restated from smallgwn's tests (none of that code is used):
  - stages, their order, units and throughput denominators: tests/benchmark_main.cu:576-866
    (bvh_build_<builder>, refit_bvh, refit_moment_o{0,1,2}, build_boundary_chain,
    build_bvh_moment_o{0,1,2}, query_taylor_o{0,1,2}, query_exact, query_antipodal_crossings,
    query_antipodal_boundary, query_antipodal_gradient, query_antipodal, query_ray_first_hit,
    dynamic_refit_query_o2), each stage's set-up call run before its timed calls;
  - timing: warm-up calls, then each measured call bracketed by CUDA events on the stage's stream
    (and a stream synchronization per call when `stream_sync_per_iter`), mean and linearly
    interpolated p50 / p95 of the per-call milliseconds (tests/benchmark_utils.cuh:64-134);
  - queries and rays: the seeded mixes of tests/benchmark_utils.cuh:136-370
    (`meshes.reference_mixed_queries`, `meshes.reference_mixed_rays`), and the dynamic stage's
    positions z + 0.001 * ((i mod 17) - 8) (tests/benchmark_main.cu:454-461);
  - defaults: 1M queries, 5 warm-up and 20 measured calls, accuracy scale 2, stack capacity 96,
    a synchronization per call, seed 0xB3A9E5D4, H-PLOC (tests/benchmark_main.cu:31-37);
  - CSV: the header and row layout of tests/benchmark_csv.cuh:48-74.

`query_antipodal_crossings` and `query_antipodal_boundary` time the two halves of smallgwn's
antipodal query, which smallgwn's harness launches through its own detail functors; this library
evaluates both halves in one kernel, so those rows are written with success = 0 and the reason,
and `query_antipodal` times the whole query. The Taylor stages take the library's timed walk choice
(the warm-up's first two calls time the warp-cooperative and the per-thread walk, the measured calls
take the faster); `--traversal warp|thread` forces one walk (the same results). Every stage runs
inside an NVTX range of its name (the library's own calls add ranges of theirs inside it).

Usage: python -m smallgwn_b200.stages [--model mesh.ply | --sphere] [--queries N] [--csv PATH] ...
"""
from __future__ import annotations

import argparse
import csv
import datetime
import io
import math
from dataclasses import dataclass, field
from pathlib import Path

import numpy as np

CSV_HEADER = ("timestamp,gpu_name,cuda_runtime_version,model_path,vertex_count,triangle_count,"
              "boundary_edge_count,query_count,stage,warmup_iters,measure_iters,latency_mean_ms,"
              "latency_p50_ms,latency_p95_ms,throughput_per_s,unit,builder,accuracy_scale,stack_capacity,"
              "stream_sync_per_iter,seed,success,error_message")

STAGES = ("bvh_build_{builder}", "refit_bvh", "refit_moment_o0", "refit_moment_o1", "refit_moment_o2",
          "build_boundary_chain", "build_bvh_moment_o0", "build_bvh_moment_o1", "build_bvh_moment_o2",
          "query_taylor_o0", "query_taylor_o1", "query_taylor_o2", "query_exact", "query_antipodal_crossings",
          "query_antipodal_boundary", "query_antipodal_gradient", "query_antipodal", "query_ray_first_hit",
          "dynamic_refit_query_o2")

FUSED_ANTIPODAL = "evaluated inside query_antipodal's single kernel in this library (no separate entry point)"


@dataclass
class options:
    """Mirror of smallgwn's benchmark_cli_options (tests/benchmark_main.cu:52-66)."""
    query_count: int = 1_000_000
    warmup_iters: int = 5
    measure_iters: int = 20
    accuracy_scale: float = 2.0
    stack_capacity: int = 96
    stream_sync_per_iter: bool = True
    seed: int = 0xB3A9E5D4
    builder: str = "hploc"
    skip_exact: bool = False
    winding_query_only: bool = False
    # Taylor stages: the walk that the timed calls of the warm-up pick ("timed"), or a forced
    # "warp" / "thread" walk (identical results)
    traversal: str = "timed"
    only: tuple = ()         # run just these stages (empty: all)
    # Not smallgwn's: time the calls as its kernels are timed beside them -- a 256 MiB write that
    # flushes the L2 before each measured call, the events read after the last call (no
    # synchronization between calls), so the host's enqueueing overlaps the flush.
    flush_l2: bool = False


@dataclass
class stage_result:
    """Mirror of smallgwn's gwn_benchmark_stage_result."""
    stage: str
    unit: str
    warmup_iters: int
    measure_iters: int
    vertex_count: int
    triangle_count: int
    query_count: int
    success: bool = False
    error_message: str = ""
    latency_mean_ms: float = 0.0
    latency_p50_ms: float = 0.0
    latency_p95_ms: float = 0.0
    throughput_per_s: float = 0.0
    samples_ms: list = field(default_factory=list)


def percentile_ms(samples, q: float) -> float:
    """Linear interpolation between the order statistics around q (n - 1) (smallgwn's percentile_ms)."""
    if len(samples) == 0:
        return 0.0
    s = sorted(float(v) for v in samples)
    pos = min(max(q, 0.0), 1.0) * (len(s) - 1)
    lo = int(math.floor(pos))
    hi = min(len(s) - 1, lo + 1)
    t = pos - lo
    return s[lo] * (1.0 - t) + s[hi] * t


def summarize(samples) -> tuple[float, float, float]:
    """(mean, p50, p95) of per-call milliseconds."""
    if len(samples) == 0:
        return 0.0, 0.0, 0.0
    return float(np.mean(np.asarray(samples, dtype=np.float64))), percentile_ms(samples, 0.5), percentile_ms(samples, 0.95)


def measure_stage_latency_ms(warmup_iters: int, measure_iters: int, stream, sync_per_iter: bool, fn,
                             flush=None) -> list:
    """Per-call milliseconds of `fn` (a callable returning a gwn_status) after `warmup_iters` untimed
    calls, CUDA events around each call on `stream` (smallgwn's gwn_measure_stage_latency_ms).
    With `flush` (a device buffer larger than the L2), the buffer is written before each measured
    call, outside its events, and the events are read after the last call. Raises RuntimeError with
    the status message when a call fails."""
    import torch

    if warmup_iters < 0 or measure_iters <= 0:
        raise ValueError("Benchmark warmup/iteration counts are invalid.")

    def call():
        st = fn()
        if not st.is_ok():
            raise RuntimeError(st.message)

    for _ in range(warmup_iters):
        call()
        if sync_per_iter:
            stream.synchronize()
    if flush is not None:
        stream.synchronize()
        ev = []
        for i in range(measure_iters):
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            with torch.cuda.stream(stream):
                flush.fill_(i & 0xFF)
            e0.record(stream)
            call()
            e1.record(stream)
            ev.append((e0, e1))
        stream.synchronize()
        return [a.elapsed_time(b) for a, b in ev]
    out = []
    for _ in range(measure_iters):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        call()
        e1.record(stream)
        e1.synchronize()
        out.append(e0.elapsed_time(e1))
        if sync_per_iter:
            stream.synchronize()
    return out


def run_stage(name: str, unit: str, denominator: int, opts: options, vertex_count: int, triangle_count: int,
              stream, setup, fn, flush=None) -> stage_result:
    """One stage: `setup` once (untimed), then the timed calls of `fn`; failures become the row's
    error message, as in smallgwn's run_stage (tests/benchmark_main.cu:286-330)."""
    import torch

    r = stage_result(name, unit, opts.warmup_iters, opts.measure_iters, vertex_count, triangle_count,
                     opts.query_count)
    with torch.cuda.nvtx.range(name):
        try:
            st = setup()
            if not st.is_ok():
                r.error_message = st.message
                return r
            r.samples_ms = measure_stage_latency_ms(opts.warmup_iters, opts.measure_iters, stream,
                                                    opts.stream_sync_per_iter, fn, flush)
        except RuntimeError as e:
            r.error_message = str(e)
            return r
    r.success = True
    r.latency_mean_ms, r.latency_p50_ms, r.latency_p95_ms = summarize(r.samples_ms)
    if r.latency_mean_ms > 0.0:
        r.throughput_per_s = denominator / (r.latency_mean_ms / 1e3)
    return r


def _unavailable(name: str, unit: str, opts: options, vertex_count: int, triangle_count: int, why: str):
    return stage_result(name, unit, opts.warmup_iters, opts.measure_iters, vertex_count, triangle_count,
                        opts.query_count, success=False, error_message=why)


def run_model(mesh: dict, opts: options, stream=None) -> tuple[list, dict]:
    """Every stage of smallgwn's harness on one mesh (SoA dict), in its order; returns the stage
    results and the per-model CSV context (boundary edge count)."""
    import torch

    from . import api, meshes

    stream = stream if stream is not None else torch.cuda.current_stream()
    s = stream.cuda_stream
    nv, nt, nq = int(mesh["x"].size), int(mesh["i0"].size), int(opts.query_count)
    method = {"hploc": api.gwn_bvh_build_method.k_hploc, "lbvh": api.gwn_bvh_build_method.k_lbvh}[opts.builder]
    geo = api.gwn_geometry_object()
    st = api.gwn_upload_geometry(geo, mesh["x"], mesh["y"], mesh["z"], mesh["i0"], mesh["i1"], mesh["i2"], s)
    if not st.is_ok():
        raise RuntimeError(st.message)
    bvh = api.gwn_bvh4_object()
    mom = {o: api.gwn_bvh4_moment_object(o) for o in (0, 1, 2)}
    chain = api.gwn_boundary_chain_object()
    st = api.gwn_build_boundary_chain(geo, chain, s)
    context = {"boundary_edge_count": chain.edge_count() if st.is_ok() else 0}

    dynamic = [mesh["x"].astype(np.float32), mesh["y"].astype(np.float32), mesh["z"].astype(np.float32).copy()]
    dynamic[2] += np.float32(0.001) * ((np.arange(nv) % 17) - 8).astype(np.float32)
    dev = lambda a: torch.from_numpy(np.ascontiguousarray(a)).to("cuda")  # noqa: E731
    q = [dev(v) for v in meshes.reference_mixed_queries(mesh, nq, opts.seed)]
    rays = [dev(v) for v in meshes.reference_mixed_rays(mesh, nq, opts.seed)]
    out = torch.empty(nq, dtype=torch.float32, device="cuda")
    grad = [torch.empty(nq, dtype=torch.float32, device="cuda") for _ in range(3)]
    hits = torch.empty((nq, 8), dtype=torch.int32, device="cuda")
    cfg = api.gwn_query_batch_config(stack_capacity=opts.stack_capacity)
    ok = api.gwn_status()
    flush = torch.empty(256 << 20, dtype=torch.uint8, device="cuda") if opts.flush_l2 else None

    def build():
        return api.gwn_build_bvh(geo, bvh, api.gwn_bvh_build_options(method=method), s)

    def build_moment(o):
        def f():
            r = build()
            return r if not r.is_ok() else api.gwn_refit_bvh_moment(o, bvh, mom[o], s)
        return f

    def taylor(o):
        return lambda: api.gwn_compute_winding_number_taylor_batch(o, bvh, mom[o], *q, out, opts.accuracy_scale, s,
                                                                   config=cfg, traversal=opts.traversal)

    def setup_boundary():
        return api.gwn_build_boundary_chain(geo, chain, s)

    def setup_bvh_and_boundary():
        r = build()
        return r if not r.is_ok() else setup_boundary()

    def setup_rays():
        r = build()
        if not r.is_ok():
            return r
        r = api.gwn_compute_ray_first_hit_batch(bvh, *rays, hits, stream=s, config=cfg)
        if not r.is_ok():
            return r
        stream.synchronize()
        ratio = float((api.ray_hit_records(hits)["status"] == api.gwn_ray_first_hit_status.k_hit).mean())
        context["ray_mix_hit_ratio"] = ratio
        if not (0.05 < ratio < 0.95):
            return api.gwn_status(api.gwn_error.invalid_argument, "Ray benchmark mix hit ratio is outside (0.05, 0.95).")
        return ok

    def dynamic_frame():
        r = api.gwn_update_geometry(geo, *dynamic, s)
        if r.is_ok():
            r = api.gwn_refit_bvh(geo, bvh, s)
        if r.is_ok():
            r = api.gwn_refit_bvh_moment(2, bvh, mom[2], s)
        return r if not r.is_ok() else taylor(2)()

    def stage(name, unit, denom, setup, fn):
        if opts.only and name not in opts.only:
            return None
        return run_stage(name, unit, denom, opts, nv, nt, stream, setup, fn, flush)

    query_o1 = lambda: stage("query_taylor_o1", "queries/s", nq, build_moment(1), taylor(1))  # noqa: E731
    query_antipodal = lambda: stage(  # noqa: E731
        "query_antipodal", "queries/s", nq, setup_bvh_and_boundary,
        lambda: api.gwn_compute_winding_number_antipodal_batch(geo, bvh, chain, *q, out, stream=s, config=cfg))
    if opts.winding_query_only:
        return [r for r in (query_o1(), query_antipodal()) if r is not None], context

    res = [stage(f"bvh_build_{opts.builder}", "triangles/s", nt, lambda: ok, build),
           stage("refit_bvh", "triangles/s", nt, build, lambda: api.gwn_refit_bvh(geo, bvh, s))]
    for o in (0, 1, 2):
        res.append(stage(f"refit_moment_o{o}", "triangles/s", nt, build,
                         lambda o=o: api.gwn_refit_bvh_moment(o, bvh, mom[o], s)))
    res.append(stage("build_boundary_chain", "triangles/s", nt, lambda: ok, setup_boundary))
    for o in (0, 1, 2):
        res.append(stage(f"build_bvh_moment_o{o}", "triangles/s", nt, lambda: ok, build_moment(o)))
    res.append(stage("query_taylor_o0", "queries/s", nq, build_moment(0), taylor(0)))
    res.append(query_o1())
    res.append(stage("query_taylor_o2", "queries/s", nq, build_moment(2), taylor(2)))
    if not opts.skip_exact:
        res.append(stage("query_exact", "queries/s", nq, build,
                         lambda: api.gwn_compute_winding_number_exact_batch(bvh, *q, out, s, config=cfg)))
    for name in ("query_antipodal_crossings", "query_antipodal_boundary"):
        if not opts.only or name in opts.only:
            res.append(_unavailable(name, "queries/s", opts, nv, nt, FUSED_ANTIPODAL))
    res.append(stage("query_antipodal_gradient", "queries/s", nq, setup_boundary,
                     lambda: api.gwn_compute_winding_gradient_antipodal_batch(geo, chain, *q, *grad, stream=s,
                                                                              config=cfg)))
    res.append(query_antipodal())
    res.append(stage("query_ray_first_hit", "rays/s", nq, setup_rays,
                     lambda: api.gwn_compute_ray_first_hit_batch(bvh, *rays, hits, stream=s, config=cfg)))
    res.append(stage("dynamic_refit_query_o2", "queries/s", nq, build, dynamic_frame))
    return [r for r in res if r is not None], context


def csv_rows(results, context: dict, model_path: str, opts: options, gpu_name: str, cuda_runtime: int,
             timestamp: str) -> str:
    """CSV text of the results with smallgwn's header and column order (tests/benchmark_csv.cuh:48-74)."""
    buf = io.StringIO()
    w = csv.writer(buf, lineterminator="\n")
    buf.write(CSV_HEADER + "\n")
    for r in results:
        w.writerow([timestamp, gpu_name, cuda_runtime, model_path, r.vertex_count, r.triangle_count,
                    context.get("boundary_edge_count", 0), r.query_count, r.stage, r.warmup_iters, r.measure_iters,
                    f"{r.latency_mean_ms:.6f}", f"{r.latency_p50_ms:.6f}", f"{r.latency_p95_ms:.6f}",
                    f"{r.throughput_per_s:.6f}", r.unit, opts.builder, opts.accuracy_scale, opts.stack_capacity,
                    1 if opts.stream_sync_per_iter else 0, opts.seed, 1 if r.success else 0, r.error_message])
    return buf.getvalue()


def main(argv=None) -> int:
    import torch

    from . import _lib, api, meshes

    ap = argparse.ArgumentParser(description=__doc__.split("\n\n")[0])
    src = ap.add_mutually_exclusive_group()
    src.add_argument("--model", type=Path, help="PLY mesh (smallgwn's --model)")
    src.add_argument("--sphere", action="store_true", help="the displaced 1024 x 512 UV sphere (default)")
    d = options()
    ap.add_argument("--queries", type=int, default=d.query_count)
    ap.add_argument("--warmup", type=int, default=d.warmup_iters)
    ap.add_argument("--iters", type=int, default=d.measure_iters)
    ap.add_argument("--accuracy-scale", type=float, default=d.accuracy_scale)
    ap.add_argument("--stack-capacity", type=int, default=d.stack_capacity)
    ap.add_argument("--no-stream-sync", action="store_true")
    ap.add_argument("--seed", type=lambda v: int(v, 0), default=d.seed)
    ap.add_argument("--builder", choices=["hploc", "lbvh"], default=d.builder)
    ap.add_argument("--skip-exact", action="store_true")
    ap.add_argument("--winding-query-only", action="store_true")
    ap.add_argument("--traversal", choices=["timed", "warp", "thread"], default=d.traversal,
                    help="Taylor stages: the faster walk from timed warm-up calls, the warp-cooperative walk "
                         "or one walk per thread")
    ap.add_argument("--csv", type=Path, default=Path("smallgwn_bench.csv"))
    a = ap.parse_args(argv)
    opts = options(a.queries, a.warmup, a.iters, a.accuracy_scale, a.stack_capacity, not a.no_stream_sync, a.seed,
                   a.builder, a.skip_exact, a.winding_query_only, a.traversal)
    if a.model is not None:
        mesh, model = api.read_ply(a.model), str(a.model)
    else:
        mesh, model = meshes.sphere_mesh(), "synthetic:displaced_uv_sphere_1024x512_seed2"
    results, context = run_model(mesh, opts)
    for r in results:
        line = (f"  {r.stage:<26s} mean={r.latency_mean_ms:9.3f} ms p50={r.latency_p50_ms:9.3f} ms "
                f"p95={r.latency_p95_ms:9.3f} ms thr={r.throughput_per_s:.2e} {r.unit}") if r.success else \
            f"  {r.stage:<26s} FAILED: {r.error_message}"
        print(line, flush=True)
    stamp = datetime.datetime.now(datetime.timezone.utc).strftime("%Y-%m-%dT%H:%M:%SZ")
    a.csv.write_text(csv_rows(results, context, model, opts, torch.cuda.get_device_name(),
                              _lib.load().gwnb_cuda_runtime_version(), stamp))
    return 0 if all(r.success or r.error_message == FUSED_ANTIPODAL for r in results) else 1


if __name__ == "__main__":
    raise SystemExit(main())
