#!/usr/bin/env python
"""Benchmark of the LBVH microbench (1,048,576 triangles, 4,194,304 rays, seed 7).

One step = build the triangle LBVH, trace 4,194,304 closest-hit rays, refit after
vertex jitter, build the LBVH over 1,048,576 query boxes and run the cross overlap
query.  Metric: Mrays/s of the whole step (rays / step time); the per-phase times,
LBVH Mtri/s and traversal Mrays/s are reported beside it.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl lux|reference]

N > 1 runs under torchrun: every rank runs an independent replica (the build is a
global sort, so ranks share nothing) and value = all ranks' rays / max rank time.
--impl reference times the reference's own CPU code (oracle/_ref) on bounded samples.
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

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

from lux_b200 import workloads as W  # noqa: E402

N_TRIS = 1 << 20
N_RAYS = 1 << 22
N_QUERIES = 1 << 20
SEED = 7
WORKLOAD = ("LBVH microbench: 1,048,576 soup triangles (lognormal edges, median 2e-3), "
            "4,194,304 uniform rays, refit after N(0,1e-4) jitter, 1,048,576 query boxes "
            "(half extent 1e-3), seed 7")
METRIC = "Mrays/s"
# Algorithmic bytes (per unit) used for the roofline: build 120 B/tri, refit 104 B/tri,
# traversal 32 B ray + 8 B hit + 32 B per box test + 36 B per triangle test.
BUILD_BYTES_PER_TRI = 120
TRACE_DRAM_BYTES_PER_RAY = (0.7169208e9 + 0.0557215e9) / 1048576
REFIT_BYTES_PER_TRI = 104


def measured_peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(path):
        with open(path) as f:
            p = json.load(f)
        return float(p["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi clocks/throttle sampling during the timed region."""

    QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int):
        self.device = device
        self.proc = None
        self.path = None

    def start(self):
        fd, self.path = tempfile.mkstemp(suffix=".csv")
        os.close(fd)
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.device), f"--query-gpu={self.QUERY}",
                 "--format=csv,noheader,nounits", "-lms", "100"],
                stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except (FileNotFoundError, OSError):
            self.proc = None
        time.sleep(0.15)

    def stop(self) -> dict:
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        time.sleep(0.15)
        self.proc.terminate()
        self.proc.wait()
        sm, smax, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        with open(self.path) as f:
            for line in f:
                parts = [p.strip() for p in line.split(",")]
                if len(parts) < 9:
                    continue
                try:
                    sm.append(float(parts[1]))
                    smax.append(float(parts[2]))
                except ValueError:
                    continue
                for name, flag in zip(names, parts[5:9]):
                    if flag.lower() == "active":
                        reasons.add(name)
        os.unlink(self.path)
        return {"sm_mhz": statistics.median(sm) if sm else None,
                "sm_max_mhz": max(smax) if smax else None,
                "reasons": sorted(reasons), "samples": len(sm)}


# ------------------------------------------------------------------ reference CPU arm

def reference_step_estimate(data: dict, ray_sample: int, threads: int) -> dict:
    """Times the reference's own host code (oracle/_ref) on bounded samples of the step.

    Build: build_cpu_lbvh_tree over all 1,048,576 triangles (the reference builder is
    single threaded).  Trace: intersect_cpu_bvh_tree on `ray_sample` rays over all host
    threads, scaled to 4,194,304.  Refit: the reference refit re-runs its whole layout
    (bvh/gpu_bvh.cu:597-613); on the host that is a rebuild, timed as one.  Query build
    + overlap: a second build over the query boxes plus the oracle port's overlap
    traversal over a sample of queries, scaled.
    """
    from oracle.bindings import Oracle, Ref

    ref = Ref()
    tris = data["triangles"]
    rays = data["rays"][:ray_sample]
    t0 = time.perf_counter()
    tree = ref.tree_create(tris)
    t_build = time.perf_counter() - t0
    t0 = time.perf_counter()
    ref.tree_trace(tree, rays, threads=threads)
    t_trace = (time.perf_counter() - t0) * (N_RAYS / len(rays))
    ref.tree_destroy(tree)
    t0 = time.perf_counter()
    ref.tree_destroy(ref.tree_create(data["refit_triangles"]))
    t_refit = time.perf_counter() - t0
    t0 = time.perf_counter()
    ref.tree_destroy(ref.tree_create(data["queries"], kind=1))
    t_qbuild = time.perf_counter() - t0
    ora = Oracle()
    tree = ora.build(ora.triangle_bounds(data["refit_triangles"]))
    qs = data["queries"][: N_QUERIES // 16]
    t0 = time.perf_counter()
    ora.overlap(tree, qs, self_pairs=False, max_pairs=1 << 22)
    t_overlap = (time.perf_counter() - t0) * 16
    total = t_build + t_trace + t_refit + t_qbuild + t_overlap
    return {"step_s": total, "build_s": t_build, "trace_s": t_trace, "refit_s": t_refit,
            "query_build_s": t_qbuild, "overlap_s": t_overlap}


def run_reference(args) -> None:
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    from oracle.bindings import Ref

    if not Ref.available():
        print(json.dumps({"impl": "reference",
                          "unavailable": "oracle/_ref/libluxref.so was not built "
                                         "(reference sources absent when built)"}))
        return
    threads = os.cpu_count() or 1
    data = W.lbvh_microbench(N_TRIS, N_RAYS, N_QUERIES, SEED)
    sample = 16384
    for _ in range(args.warmup):
        reference_step_estimate(data, 2048, threads)
    steps = [reference_step_estimate(data, sample, threads) for _ in range(args.steps)]
    step_s = statistics.median(s["step_s"] for s in steps)
    value = N_RAYS / step_s / 1e6
    line = {
        "impl": "reference",
        "metric": METRIC, "value": value, "unit": "Mrays/s",
        "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": step_s * 1e3,
        "ms_per_step_kind": "extrapolated from bounded samples of the step (see sample)",
        "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": lbvh_config(args.gpus),
        "cpu_baseline": {
            "value": value, "unit": "Mrays/s", "cores": threads, "kind": "reference",
            "sample": (f"reference host code: full 1,048,576-triangle builds (1 thread), "
                       f"{sample} of 4,194,304 rays traced on {threads} threads and scaled, "
                       f"overlap on 1/16 of the queries scaled"),
        },
        "e2e": {"value": value, "unit": "Mrays/s", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
        "phases_ms": {k: statistics.median(s[k] for s in steps) * 1e3
                      for k in ["build_s", "trace_s", "refit_s", "query_build_s", "overlap_s"]},
    }
    print(json.dumps(line))


# ------------------------------------------------------------------ GPU arm

def lbvh_config(world: int) -> dict:
    """The LBVH microbench's config dict, identical in both arms."""
    return {"workload": WORKLOAD, "l2": "flushed between timed steps (256 MiB write)",
            "parallelism": f"replicas x{world}" if world > 1 else "single GPU"}


def max_over_ranks(value: float, dist, device) -> float:
    """The largest per-rank value: a multi-GPU step lasts as long as its slowest rank.
    Works with any process group (NCCL on GPUs; the CPU tests use gloo)."""
    if dist is None:
        return value
    import torch
    t = torch.tensor([value], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def whole_job_rate(units_per_rank: int, world: int, step_ms: float) -> float:
    """Whole-job throughput in millions of units per second: every rank processes the
    same units per step (replicas), timed by the slowest rank."""
    return world * units_per_rank / (step_ms * 1e-3) / 1e6


def run_lux(args) -> None:
    import torch

    import lux_b200

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime

        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))

    dev = torch.device("cuda", local)
    # A dedicated stream for everything (the legacy default stream has handle 0, which
    # the C ABI reads as "use the context's own stream").
    torch.cuda.set_stream(torch.cuda.Stream(dev))
    data = W.lbvh_microbench(N_TRIS, N_RAYS, N_QUERIES, SEED)
    d_tris = torch.from_numpy(data["triangles"]).to(dev)
    d_rays = torch.from_numpy(data["rays"]).to(dev)
    d_refit = torch.from_numpy(data["refit_triangles"]).to(dev)
    d_queries = torch.from_numpy(data["queries"]).to(dev)
    hit_id = torch.empty(N_RAYS, dtype=torch.int32, device=dev)
    hit_t = torch.empty(N_RAYS, dtype=torch.float32, device=dev)
    max_pairs = 1 << 21
    pairs = torch.empty((max_pairs, 2), dtype=torch.int32, device=dev)
    found = torch.zeros(1, dtype=torch.int64, device=dev)
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=dev)

    stream = torch.cuda.current_stream(dev)
    assert stream.cuda_stream != 0
    ctx = lux_b200.Context(local, stream.cuda_stream)
    bvh = ctx.build_lbvh(d_tris)
    qbvh = ctx.build_lbvh(d_queries, kind=lux_b200.PRIM_AABBS)
    ctx.set_option(lux_b200.OPT_TRACE_VARIANT, args.trace_variant)
    ctx.set_option(lux_b200.OPT_TRACE_BUDGET, args.trace_budget)
    lib = ctx._lib
    found_ptr = found.data_ptr()

    phases = ["build", "trace", "refit", "query_build", "overlap"]

    def step(ev=None):
        if ev:
            ev[0].record(stream)
        bvh.rebuild(d_tris)
        if ev:
            ev[1].record(stream)
        bvh.trace_closest(d_rays, hit_id, hit_t)
        if ev:
            ev[2].record(stream)
        bvh.refit(d_refit)
        if ev:
            ev[3].record(stream)
        qbvh.rebuild(d_queries)
        if ev:
            ev[4].record(stream)
        status = lib.lux_overlap_cross(ctx.handle, bvh.handle, qbvh.handle, pairs.data_ptr(),
                                       max_pairs, found_ptr)
        if status:
            lux_b200._check(status)
        if ev:
            ev[5].record(stream)

    for _ in range(max(args.warmup, 1)):
        step()
        flush.zero_()
    torch.cuda.synchronize()

    evs = [[torch.cuda.Event(enable_timing=True) for _ in range(6)] for _ in range(args.steps)]
    clocks = ClockSampler(local)
    launches0 = ctx.launch_count()
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    clocks.start()
    wall0 = time.perf_counter()
    for k in range(args.steps):
        flush.zero_()          # L2 flush between timed steps (outside the step events)
        step(evs[k])
    torch.cuda.synchronize()
    wall = time.perf_counter() - wall0
    clock_info = clocks.stop()
    if dist:
        dist.barrier()
    launches = ctx.launch_count() - launches0
    ctx.synchronize()

    per_phase = {p: [] for p in phases}
    totals = []
    for e in evs:
        for i, p in enumerate(phases):
            per_phase[p].append(e[i].elapsed_time(e[i + 1]))
        totals.append(e[0].elapsed_time(e[5]))
    step_ms = float(np.sum(totals)) / args.steps
    step_ms = max_over_ranks(step_ms, dist, dev)
    value = whole_job_rate(N_RAYS, world, step_ms)
    phase_ms = {p: float(np.mean(v)) for p, v in per_phase.items()}

    # Roofline of the dominant kernel (the traversal: one launch per trace phase).
    # DRAM traffic per ray of k_trace_wide_persistent from one ncu capture of this
    # generator at 1,048,576 triangles and 1,048,576 rays (0.717 GB read + 0.056 GB
    # written, 737 B per ray), scaled by the ray count.
    box_tests, tri_tests = bvh.trace_stats(d_rays)
    trace_bytes = N_RAYS * (32 + 8) + 32 * box_tests + 36 * tri_tests
    peak, peak_kind = measured_peaks()
    dominant = max(phase_ms, key=phase_ms.get)
    if dominant == "trace":
        achieved = trace_bytes / (phase_ms["trace"] * 1e-3) / 1e9
        alg = trace_bytes
    elif dominant == "build":
        alg = BUILD_BYTES_PER_TRI * N_TRIS
        achieved = alg / (phase_ms["build"] * 1e-3) / 1e9
    else:
        alg = trace_bytes
        achieved = trace_bytes / (phase_ms["trace"] * 1e-3) / 1e9
        dominant = "trace"

    trace_traffic = TRACE_DRAM_BYTES_PER_RAY * N_RAYS if dominant == "trace" else None
    found_count = int(found.item())
    hits = int((hit_id >= 0).sum().item())

    e2e = None
    cpu_baseline = None
    if rank == 0 and not args.skip_e2e:
        e2e = measure_e2e(ctx, data, args, dev, contexts=3)
    if rank == 0 and world == 1 and not args.skip_cpu_baseline:
        cpu_baseline = measure_cpu_baseline(data)
    reference_gpu = None
    if rank == 0 and world == 1 and not args.skip_reference_gpu:
        reference_gpu = measure_reference_gpu(data)

    line = {
        "metric": METRIC, "value": value, "unit": "Mrays/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": step_ms,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f32", "data": "synthetic",
        "config": lbvh_config(world),
        "phases_ms": phase_ms,
        "lbvh_mtri_s": N_TRIS / (phase_ms["build"] * 1e-3) / 1e6,
        "trace_mrays_s": N_RAYS / (phase_ms["trace"] * 1e-3) / 1e6,
        "refit_mtri_s": N_TRIS / (phase_ms["refit"] * 1e-3) / 1e6,
        "hits": hits, "overlap_pairs": found_count,
        "roofline": {"bound": "hbm",
                     "kernel": "k_trace_wide_persistent" if dominant == "trace" else dominant,
                     "achieved": achieved, "peak": peak, "peak_kind": peak_kind,
                     "unit": "GB/s", "frac": achieved / peak, "traffic": trace_traffic,
                     "traffic_source": "ncu dram__bytes_read+write of k_trace_wide_persistent "
                                       "at 1,048,576 rays, scaled by rays",
                     "algorithmic_bytes_per_launch": alg,
                     "box_tests_per_ray": box_tests / N_RAYS,
                     "tri_tests_per_ray": tri_tests / N_RAYS},
        "clocks": clock_info,
        "gpu_launches": launches,
        "wall_s_timed_region": wall,
        "e2e": e2e,
        "cpu_baseline": cpu_baseline,
        "reference_gpu": reference_gpu,
    }
    if rank == 0 and world == 1 and not args.skip_render:
        # The path-tracer half (configs 1, 3, 4 and 5), each with its own timing, after
        # the LBVH microbench's timed steps.
        bvh.close()
        qbvh.close()
        line["render_configs"] = render_suite(args)
    if rank == 0:
        print(json.dumps(line))
    if dist:
        dist.barrier()
        dist.destroy_process_group()


def measure_e2e(ctx, data, args, dev, contexts=2, steps=None) -> dict:
    """The same step through the C ABI with pinned host buffers: copies are timed.
    contexts: contexts (each on its own host thread) taking the steps in turn; steps:
    timed steps in all (default: a multiple of contexts near 10)."""
    import torch

    import lux_b200

    def pinned(a):
        t = torch.from_numpy(a).pin_memory()
        return t

    h_tris = pinned(data["triangles"])
    h_rays = pinned(data["rays"])
    h_refit = pinned(data["refit_triangles"])
    h_queries = pinned(data["queries"])
    h_id = torch.empty(N_RAYS, dtype=torch.int32).pin_memory()
    h_t = torch.empty(N_RAYS, dtype=torch.float32).pin_memory()
    max_pairs = 1 << 21
    h_pairs = torch.empty((max_pairs, 2), dtype=torch.int32).pin_memory()
    found = np.zeros(1, np.int64)
    lib = ctx._lib

    # Two contexts (each its own stream, BVHs and output buffers) so that one step's
    # copies overlap the other's kernels, as a caller with a stream of steps would run
    # them; every step still copies its inputs in and its results out.
    import threading

    device = dev.index or 0 if hasattr(dev, "index") else int(dev)
    ctxs = [ctx] + [lux_b200.Context(device) for _ in range(contexts - 1)]
    outs = [(h_id, h_t, h_pairs, found)] + [
        (torch.empty(N_RAYS, dtype=torch.int32).pin_memory(),
         torch.empty(N_RAYS, dtype=torch.float32).pin_memory(),
         torch.empty((max_pairs, 2), dtype=torch.int32).pin_memory(), np.zeros(1, np.int64))
        for _ in range(contexts - 1)]
    trees = [(c.build_lbvh(h_tris), c.build_lbvh(h_queries, kind=lux_b200.PRIM_AABBS))
             for c in ctxs]

    def step(k):
        bvh, qbvh = trees[k]
        o_id, o_t, o_pairs, o_found = outs[k]
        bvh.rebuild(h_tris)
        bvh.trace_closest(h_rays, o_id, o_t)
        bvh.refit(h_refit)
        qbvh.rebuild(h_queries)
        lux_b200._check(lib.lux_overlap_cross(ctxs[k].handle, bvh.handle, qbvh.handle,
                                              o_pairs.data_ptr(), max_pairs,
                                              o_found.ctypes.data))

    def run(k, n):
        for _ in range(n):
            step(k)

    for _ in range(max(args.warmup, 1)):
        for k in range(contexts):
            step(k)
    if steps is None:
        steps = max(4, min(args.steps, 10) // 2 * 2)
    steps = max(contexts, steps // contexts * contexts)
    # One context alone: each step's copies and kernels in sequence.
    t0 = time.perf_counter()
    run(0, steps)
    ctx.synchronize()
    serial = (time.perf_counter() - t0) / steps
    # All contexts, steps taken in turn.
    workers = [threading.Thread(target=run, args=(k, steps // contexts)) for k in range(contexts)]
    t0 = time.perf_counter()
    for w in workers:
        w.start()
    for w in workers:
        w.join()
    for c in ctxs:
        c.synchronize()
    dt = (time.perf_counter() - t0) / steps
    h2d = sum(d.nbytes for d in (data["triangles"], data["rays"], data["refit_triangles"],
                                  data["queries"]))
    d2h = N_RAYS * 8 + min(int(found[0]), max_pairs) * 8 + 8
    for bvh, qbvh in trees:
        bvh.close()
        qbvh.close()
    for c in ctxs[1:]:
        c.close()
    return {"value": N_RAYS / dt / 1e6, "unit": "Mrays/s", "h2d_bytes_per_step": h2d,
            "d2h_bytes_per_step": d2h, "ms_per_step": dt * 1e3, "steps": steps,
            "host_buffers": "pinned",
            "pipelining": f"{contexts} contexts on {contexts} host threads, steps taken in turn",
            "one_context_ms_per_step": serial * 1e3}


def measure_reference_gpu(data) -> dict | None:
    """The same step on the reference's own GPU code (build_gpu_lbvh,
    intersect_gpu_bvh_stackless, refit_gpu_lbvh, query_aabb_overlaps_cross) compiled for
    sm_100a, on the same B200 and inputs: medians of 3 runs after one untimed run.  Its
    API takes and returns host vectors, so its step includes its copies; the kernel-only
    trace time is reported beside it."""
    try:
        from oracle.bindings import RefGpu
    except Exception:
        return None
    if not RefGpu.available():
        return None
    try:
        ms, found = RefGpu().microbench(data["triangles"], data["rays"], data["refit_triangles"],
                                        data["queries"], max_pairs=1 << 21, reps=3)
    except Exception as e:  # the reference threw: report it, keep this build's line
        return {"unavailable": str(e)}
    step = ms["build"] + ms["trace_api"] + ms["refit"] + ms["query_build"] + ms["overlap"]
    return {"kind": "reference GPU code (bvh/gpu_bvh.cu, bvh/bvh_overlap.cu) for sm_100a",
            "step_ms": step, "step_mrays_s": N_RAYS / (step * 1e-3) / 1e6,
            "trace_kernel_mrays_s": N_RAYS / (ms["trace_kernel"] * 1e-3) / 1e6,
            "lbvh_mtri_s": N_TRIS / (ms["build"] * 1e-3) / 1e6,
            "phases_ms": ms, "overlap_pairs": found,
            "timing": "host clock around each API call (copies included); trace kernel by "
                      "CUDA events with L2 flushed"}


def measure_cpu_baseline(data) -> dict | None:
    try:
        from oracle.bindings import Ref
    except Exception:
        return None
    if not Ref.available():
        return None
    threads = os.cpu_count() or 1
    est = reference_step_estimate(data, 16384, threads)
    return {"value": N_RAYS / est["step_s"] / 1e6, "unit": "Mrays/s", "cores": threads,
            "kind": "reference",
            "sample": ("reference host code: full 1,048,576-triangle builds (1 thread), 16384 "
                       f"of 4,194,304 rays on {threads} threads scaled, overlap on 1/16 of "
                       "the queries (oracle port) scaled"),
            "phases_ms": {k: v * 1e3 for k, v in est.items()}}


# ------------------------------------------------------------------ render configurations

def _render_setup(local=0):
    import torch

    import lux_b200

    torch.cuda.set_device(local)
    torch.cuda.set_stream(torch.cuda.Stream(torch.device("cuda", local)))
    stream = torch.cuda.current_stream()
    return torch, lux_b200.Context(local, stream.cuda_stream), stream


RENDER_CONFIGS = {
    # name: (width, height, spp, depth, seed, metric, workload)
    "cornell": (256, 256, 64, 4, 1, "Mrays/s (Cornell 256^2, 64 spp, depth 4)",
                "Cornell box 256x256, 64 spp, max depth 4, power light sampler, seed 1"),
    "heavy": (1024, 1024, 256, 8, 1, "Mrays/s (heavy render 1024^2, 256 spp, depth 8)",
              "Cornell box + displaced icosphere (327,680 tris, GGX 0.3) + glass icosphere "
              "(5,120 tris, IOR 1.5), 1024x1024, 256 spp, max depth 8, power light sampler, "
              "seed 1"),
}

# Render roofline, algorithmic bytes: per traced ray (camera, extension or shadow segment)
# the ray (32 B) and its hit (8 B), 32 B per node box and 36 B per triangle the reference's
# visit order tests; per bounce the minimal path state read and written once (throughput
# 12, radiance 12, pixel 4, depth/flags 4, eta 4, previous pdf and position 16, RNG 16 =
# 68 B, twice); per path its 12-byte film contribution.
RAY_BYTES = 40
PATH_STATE_BYTES_PER_BOUNCE = 2 * 68
FILM_BYTES_PER_PATH = 12
# The Cornell render's kernels run from L1 (a 71-node BLAS): its bound is instruction
# issue, measured by ncu as the issue-active fraction of the dominant bounce kernel
# (profiles/render_kernels_cornell_c1.md).
CORNELL_ISSUE_ACTIVE = None


def render_roofline(stats: dict, paths: int, seconds: float, scale: float = 1.0,
                    kernel: str = "all bounce kernels of the render") -> dict:
    """HBM roofline of a render from its traversal statistics (lux_render_traversal_stats):
    algorithmic bytes / device time.  scale: timed rays / counted rays, when the counts
    come from a sample of the timed work."""
    rays = stats["rays"] + stats["shadow_segments"]
    alg = (RAY_BYTES * rays + 32 * stats["box_tests"] + 36 * stats["tri_tests"]
           + PATH_STATE_BYTES_PER_BOUNCE * stats["rays"] + FILM_BYTES_PER_PATH * paths) * scale
    peak, peak_kind = measured_peaks()
    achieved = alg / seconds / 1e9
    return {"bound": "hbm", "kernel": kernel, "achieved": achieved, "peak": peak,
            "peak_kind": peak_kind, "unit": "GB/s", "frac": achieved / peak, "traffic": None,
            "algorithmic_bytes_per_step": alg,
            "algorithmic_bytes_per_ray": alg / (rays * scale) if rays else None,
            "box_tests_per_ray": stats["box_tests"] / rays if rays else None,
            "tri_tests_per_ray": stats["tri_tests"] / rays if rays else None,
            "instance_visits_per_ray": stats["instance_visits"] / rays if rays else None,
            "counts": "lux_render_traversal_stats: the reference's visit order, shadow "
                      "segments walked to their closest hit"}


def reference_gpu_render(builder, req, ours_ms, ours_rays, batch=0) -> dict | None:
    """The reference's own GPU wavefront tracer (oracle/_ref/libluxrefpt.so:
    PreparedScene::prepare_gpu + WavefrontPathTracer::render, its stock 65,536-path
    batches) on the same scene and request: one untimed render, then the median of three
    by CUDA events.  Its rays are counted as this build's for the same request (the same
    random streams; the reference counts none)."""
    try:
        from oracle.bindings import RefPt
    except Exception:
        return None
    if not RefPt.available():
        return None
    try:
        ref = RefPt()
        handle = ref.scene(builder)
        try:
            ref.render(handle, req, batch)
            runs = [ref.render(handle, req, batch) for _ in range(3)]
        finally:
            ref.destroy(handle)
    except Exception as e:  # the reference threw: report it, keep this build's line
        return {"unavailable": str(e)}
    ms = statistics.median(r[1] for r in runs)
    host_ms = statistics.median(r[2] for r in runs)
    return {"kind": "reference GPU wavefront tracer (integrator/wavefront_*.cu) for sm_100a",
            "request": f"{req.width}x{req.height}, {req.spp} spp, depth {req.max_depth}",
            "ms": ms, "host_ms": host_ms, "mrays_s": ours_rays / (ms * 1e-3) / 1e6,
            "this_build_ms": ours_ms, "this_build_mrays_s": ours_rays / (ours_ms * 1e-3) / 1e6,
            "speedup": ms / ours_ms,
            "timing": "CUDA events around WavefrontPathTracer::render (its film copied to the "
                      "host inside); rays counted by this build for the same request"}


def render_line(args, name: str, steps: int, warmup: int, nested: bool = False) -> dict:
    """Config 1 (Cornell) or config 3 (heavy render): one lux_render per step.  Under
    torchrun (N > 1) the frame's samples are split across the ranks and their films are
    summed with one NCCL reduce (lux_b200.distributed): strong scaling of one frame."""
    world = 1 if nested else int(os.environ.get("WORLD_SIZE", "1"))
    rank = 0 if nested else int(os.environ.get("RANK", "0"))
    local = 0 if nested else int(os.environ.get("LOCAL_RANK", "0"))
    torch, ctx, stream = _render_setup(local)
    dist = None
    if world > 1:
        import datetime

        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    from lux_b200 import distributed as D
    from lux_b200 import scene as S
    from lux_b200 import scenes as SC

    W, H, spp, depth, seed, metric, workload = RENDER_CONFIGS[name]
    reduced = bool(args.render_size or args.render_spp) and not nested
    if reduced:  # reduced profiling case of the same scene
        W = H = args.render_size or W
        spp = args.render_spp or spp
        workload = f"{workload} (reduced profiling case: {W}x{H}, {spp} spp)"
    builder = S.make_cornell_scene(W, H) if name == "cornell" else SC.heavy_render_scene(W, H)
    sc = S.Scene(ctx, builder)
    req = S.request(W, H, spp, depth, seed)
    # The autotuner (lux_autotune_render) picks the traversal variant, step budget and
    # batch on a probe of this scene (the frame itself when it is small), before timing.
    from lux_b200 import autotune
    probe = req if W * H * spp <= (1 << 23) else S.request(min(W, 512), min(H, 512),
                                                            min(spp, 16), depth, seed)
    if args.no_autotune and not nested:  # profiling: the variant given, other defaults
        import lux_b200
        ctx.set_option(lux_b200.OPT_TRACE_VARIANT, args.trace_variant)
        tune = autotune.TuneResult(args.trace_variant, ctx.get_option(lux_b200.OPT_PATH_BUDGET),
                                   ctx.get_option(lux_b200.OPT_RENDER_BATCH), 0.0, 0.0, 0)
    else:
        tune = autotune.autotune_render(ctx, sc, probe)
    film = torch.zeros((H, W, 3), dtype=torch.float32, device=f"cuda:{local}")

    def step(target):
        if world == 1:
            S.render(ctx, sc, req, target)
        else:
            D.render_sharded(lambda q, f: S.render(ctx, sc, q, f), req, target)

    for _ in range(max(warmup, 1)):
        step(film)
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    launches0 = ctx.launch_count()
    clocks = ClockSampler(local)
    clocks.start()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(steps):
        step(film)
    e1.record(stream)
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    clock_info = clocks.stop()
    launches = ctx.launch_count() - launches0
    ms = e0.elapsed_time(e1) / steps
    rays = list(S.ray_counts(ctx))
    if dist:  # the whole frame's rays, the slowest rank's time
        t = torch.tensor(rays, dtype=torch.float64, device=film.device)
        dist.all_reduce(t)
        rays = [int(v) for v in t.tolist()]
        ms = max_over_ranks(ms, dist, film.device)
    total_rays = sum(rays)
    value = total_rays / (ms * 1e-3) / 1e6
    # e2e: the frame's film on the host (device -> host copy timed; rank 0 receives it).
    host_film = np.zeros((H, W, 3), np.float32)
    e2e_steps = max(1, min(steps, 10 if name == "cornell" else 2))
    if dist:
        dist.barrier()
    t0 = time.perf_counter()
    for _ in range(e2e_steps):
        if world == 1:
            S.render(ctx, sc, req, host_film)
        else:
            step(film)
            if rank == 0:
                host_film[...] = film.cpu().numpy()
    torch.cuda.synchronize()
    e2e_ms = (time.perf_counter() - t0) / e2e_steps * 1e3
    if dist:
        e2e_ms = max_over_ranks(e2e_ms, dist, film.device)
        step(film)  # the timed film itself for the image check below (rank 0 holds it)
        torch.cuda.synchronize()
    cpu = None
    if rank == 0 and world == 1 and not args.skip_cpu_baseline:
        from oracle.bindings import Ref
        if Ref.available():
            threads = os.cpu_count() or 1
            rows = 32 if name == "cornell" else 2
            ref = Ref()
            handle = ref.desc_scene(builder)
            # The reference CPU path on one thread as well (the shipped CPU renderer is
            # single-threaded), on a smaller band of rows.
            rows1 = 8 if name == "cornell" else 1
            try:
                t0 = time.perf_counter()
                ref.desc_render(handle, req, rows=(H // 2, H // 2 + rows), threads=threads)
                cpu_s = (time.perf_counter() - t0) * H / rows
                t0 = time.perf_counter()
                ref.desc_render(handle, req, rows=(H // 2, H // 2 + rows1), threads=1)
                cpu1_s = (time.perf_counter() - t0) * H / rows1
            finally:
                ref.desc_scene_destroy(handle)
            cpu = {"value": total_rays / cpu_s / 1e6, "unit": "Mrays/s", "cores": threads,
                   "kind": "reference",
                   "sample": f"reference trace_path on {rows} of {H} rows ({threads} threads), "
                             "scaled to the frame; ray count of the same config; host BVH "
                             "build excluded",
                   "single_thread": {"value": total_rays / cpu1_s / 1e6, "unit": "Mrays/s",
                                     "cores": 1,
                                     "sample": f"{rows1} of {H} rows on one thread, scaled"}}
    # Traversal statistics for the roofline: the Cornell frame itself; the heavy frame at
    # 16 spp, scaled to the timed rays.
    roofline = None
    if rank == 0 and world == 1:
        stats_req = req if name == "cornell" or reduced else S.request(W, H, 16, depth, seed)
        st = S.traversal_stats(ctx, sc, stats_req)
        scale = total_rays / (st["rays"] + st["shadow_segments"])
        roofline = render_roofline(st, W * H * spp, ms * 1e-3 / max(world, 1), scale)
        roofline["counted_on"] = f"{stats_req.width}x{stats_req.height}, {stats_req.spp} spp"
        if name == "cornell":
            roofline["note"] = ("the scene (36 triangles, 71 BVH nodes) is L1-resident: the "
                                "render is bound by instruction issue, not HBM")
            roofline["issue_active_frac_ncu"] = CORNELL_ISSUE_ACTIVE
    # Image error against the FP64 high-spp oracle (tests/golden/make_fp64.py): relative
    # RMSE and measured / noise-predicted MSE (1 for an unbiased renderer).
    fp64 = None
    fixture = os.path.join(ROOT, "tests", "golden", f"{name}_fp64.npz")
    if rank == 0 and os.path.exists(fixture) and not reduced:
        g = np.load(fixture)
        x0, y0, x1, y1 = (int(v) for v in g["rect"]) if "rect" in g else (0, 0, W, H)
        img = film.double().cpu().numpy()[y0:y1, x0:x1] / spp
        ref_img = g["mean"].astype(np.float64)
        var = g["var"].astype(np.float64)
        mse = float(np.mean((img - ref_img) ** 2))
        oracle_noise = float(np.mean(var / int(g["spp"])))
        rms = float(np.sqrt(np.mean(ref_img ** 2)))
        fp64 = {"relative_rmse": float(np.sqrt(max(mse - oracle_noise, 0.0))) / rms,
                "relative_rmse_raw": float(np.sqrt(mse)) / rms,
                "mse_over_noise": mse / (float(np.mean(var / spp)) + oracle_noise),
                "oracle_spp": int(g["spp"]),
                "pixels": "all" if "rect" not in g else f"crop x{x0}..{x1} y{y0}..{y1}"}
    # The reference's own GPU wavefront tracer on the same scene (Cornell: the frame;
    # heavy: the frame at 8 spp, this build timed on the same request).
    reference_gpu = None
    if rank == 0 and world == 1 and not args.skip_reference_gpu:
        if name == "cornell" or reduced:
            rreq, r_ms, r_rays = req, ms, total_rays
        else:
            rreq = S.request(W, H, 8, depth, seed)
            S.render(ctx, sc, rreq, film)
            torch.cuda.synchronize()
            times = []
            for _ in range(3):
                a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                a.record(stream)
                S.render(ctx, sc, rreq, film)
                b.record(stream)
                torch.cuda.synchronize()
                times.append(a.elapsed_time(b))
            r_ms, r_rays = statistics.median(times), sum(S.ray_counts(ctx))
        reference_gpu = reference_gpu_render(builder, rreq, r_ms, r_rays)
    line = {"metric": metric, "value": value, "unit": "Mrays/s",
            "n_gpus": world, "steps": steps, "warmup": warmup, "ms_per_step": ms,
            "higher_is_better": True, "scaling": "weak" if world == 1 else "strong",
            "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {"workload": workload,
                       "l2": "scene L2/L1 resident" if name == "cornell" else
                             "path state 4M paths x 192 B > L2",
                       "parallelism": "single GPU" if world == 1 else
                                      f"samples split over {world} ranks, films summed by "
                                      "one NCCL reduce",
                       "autotuned": {"trace_variant": tune.trace_variant,
                                     "path_budget": tune.budget,
                                     "render_batch": tune.render_batch,
                                     "refill_blocks_per_sm": tune.refill_blocks,
                                     "probe": f"{probe.width}x{probe.height}, {probe.spp} spp"}},
            "rays": {"camera_extension": rays[0], "shadow_segments": rays[1]},
            "clocks": clock_info, "gpu_launches": launches,
            "e2e": {"value": total_rays / (e2e_ms * 1e-3) / 1e6, "unit": "Mrays/s",
                    "h2d_bytes_per_step": 0, "d2h_bytes_per_step": W * H * 12,
                    "ms_per_step": e2e_ms, "steps": e2e_steps},
            "roofline": roofline, "cpu_baseline": cpu, "reference_gpu": reference_gpu,
            "image_error_vs_fp64_oracle": fp64}
    if dist:
        dist.barrier()
        dist.destroy_process_group()
    ctx.close()
    return line


def run_render(args, name: str) -> None:
    line = render_line(args, name, args.steps, args.warmup)
    if int(os.environ.get("RANK", "0")) == 0:
        print(json.dumps(line))


def batched_line(args, nested: bool = False) -> dict:
    """Config 4: 64 requests over 4 resident scenes, server vs the per-request path."""
    torch, ctx, stream = _render_setup()
    from lux_b200 import scene as S
    from lux_b200 import scenes as SC
    from lux_b200 import server as SV

    builders = SC.resident_scenes(512, 512)
    scenes = [S.Scene(ctx, b) for b in builders]
    reqs = SC.batched_requests(args.requests, seed=11)
    films_plain = [torch.zeros((r["height"], r["width"], 3), device="cuda") for r in reqs]
    films_batch = [torch.zeros((r["height"], r["width"], 3), device="cuda") for r in reqs]
    rr = [S.request(r["width"], r["height"], r["spp"], r["max_depth"], r["seed"]) for r in reqs]
    # Autotuned tunables (lux_autotune_render) on a probe of the mixed workload's heaviest
    # resident scene, used by both the plain path and the server.
    from lux_b200 import autotune
    tune = autotune.autotune_render(ctx, scenes[1], S.request(512, 512, 16, 8, 3))
    path_budget = tune.budget
    S.render(ctx, scenes[0], S.request(64, 64, 4, 4, 1))
    torch.cuda.synchronize()

    def plain_pass(batch, subset):
        # Plain per-request path: lux_render one request after the other.
        ctx.set_option(3, batch)
        rays = 0
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for k in subset:
            S.render(ctx, scenes[reqs[k]["scene"]], rr[k], films_plain[k])
            rays += sum(S.ray_counts(ctx))
        e1.record(stream)
        torch.cuda.synchronize()
        return rays, e0.elapsed_time(e1) * 1e-3

    everything = list(range(len(reqs)))
    # The reference scheduler's 65,536-path batches (RenderSettings::batch_size,
    # integrator/render_context.h:18) on this build's kernels: every 8th request when
    # nested in the default run (the whole mix takes about two minutes at that batch).
    ref_subset = everything[::8] if nested else everything
    ref_rays, ref_s = ((0, float("nan")) if args.skip_reference_batch
                       else plain_pass(65536, ref_subset))
    plain_batch = max(tune.render_batch, 1 << 22)
    sub_rays, sub_s = plain_pass(plain_batch, ref_subset)
    plain_rays, plain_s = plain_pass(plain_batch, everything)
    # Batched: one server, all requests submitted at once.
    clocks = ClockSampler(0)
    with SV.Server(scenes, pool_paths=args.batch_pool, path_budget=path_budget) as srv:
        warm, _ = srv.submit(0, S.request(64, 64, 4, 4, 1))
        srv.wait(warm)
        base = srv.stats()
        clocks.start()
        ids = [srv.submit(r["scene"], q, f)[0] for r, q, f in zip(reqs, rr, films_batch)]
        srv.wait_all()
        clock_info = clocks.stop()
        stats = srv.stats()
        t_sub = min(srv.times(i)[0] for i in ids)
        t_done = max(srv.times(i)[2] for i in ids)
    batch_s = (t_done - t_sub) * 1e-9
    batch_rays = (stats["rays"] - base["rays"]) + (stats["shadow_rays"] - base["shadow_rays"])
    rel = max(float(((a - b).abs() / (1 + b.abs())).max()) for a, b in zip(films_batch, films_plain))
    value = batch_rays / batch_s / 1e6
    # The reference's own GPU wavefront tracer, request by request, on every 16th request
    # (nested) and this build's plain path on the same requests.
    reference_gpu = None
    if not args.skip_reference_gpu:
        # At most about a minute of the reference's renders: requests are taken in this
        # order until the budget is spent, and both sides are compared on those done.
        ref_gpu_order = everything[::16] if nested else everything[::4]
        ref_gpu_subset = []
        try:
            from oracle.bindings import RefPt
            if RefPt.available():
                ref = RefPt()
                handles = {}
                ms = 0.0
                try:
                    for k in ref_gpu_order:
                        if ms > 60e3:
                            break
                        si = reqs[k]["scene"]
                        if si not in handles:
                            handles[si] = ref.scene(builders[si])
                            ref.render(handles[si], S.request(64, 64, 2, 4, 1))
                        ms += ref.render(handles[si], rr[k])[1]
                        ref_gpu_subset.append(k)
                finally:
                    for h in handles.values():
                        ref.destroy(h)
                g_rays, g_s = plain_pass(plain_batch, ref_gpu_subset)
                reference_gpu = {
                    "kind": "reference GPU wavefront tracer (integrator/wavefront_*.cu) for "
                            "sm_100a, one WavefrontPathTracer::render per request",
                    "requests": ref_gpu_subset, "seconds": ms * 1e-3,
                    "mrays_s": g_rays / (ms * 1e-3) / 1e6,
                    "this_build_plain_mrays_s": g_rays / g_s / 1e6,
                    "server_speedup_vs_reference_gpu": value / (g_rays / (ms * 1e-3) / 1e6),
                    "timing": "CUDA events per render; rays counted by this build"}
        except Exception as e:
            reference_gpu = {"unavailable": str(e)}
    # Roofline of the server's work: traversal statistics of every 8th request, scaled to
    # the served rays.
    st_tot = {"rays": 0, "shadow_segments": 0, "box_tests": 0, "tri_tests": 0,
              "instance_visits": 0}
    st_paths = 0
    for k in everything[::8]:
        st = S.traversal_stats(ctx, scenes[reqs[k]["scene"]], rr[k])
        for key in st_tot:
            st_tot[key] += st[key]
        st_paths += reqs[k]["width"] * reqs[k]["height"] * reqs[k]["spp"]
    paths = sum(r["width"] * r["height"] * r["spp"] for r in reqs)
    scale = batch_rays / (st_tot["rays"] + st_tot["shadow_segments"])
    roofline = render_roofline(st_tot, 0, batch_s, scale, kernel="the server's bounce kernels")
    roofline["algorithmic_bytes_per_step"] += FILM_BYTES_PER_PATH * paths
    roofline["achieved"] = roofline["algorithmic_bytes_per_step"] / batch_s / 1e9
    roofline["frac"] = roofline["achieved"] / roofline["peak"]
    roofline["counted_on"] = "every 8th request of the mix, scaled to the served rays"
    return {"metric": "Mrays/s (batched: 64 mixed requests over 4 resident scenes)",
            "value": value, "unit": "Mrays/s", "n_gpus": 1, "steps": 1, "warmup": 1,
            "ms_per_step": batch_s * 1e3, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {"workload": f"{args.requests} requests: resolution log-uniform 128^2..1024^2,"
                                   " spp log-uniform 16..256, depth uniform 4..12, seed 11; scenes:"
                                   " Cornell, displaced icosphere + glass (332,836 tris),"
                                   " 2,097,152-tri soup, 16x16 icosphere grid",
                       "pool_paths": args.batch_pool,
                       "autotuned": {"trace_variant": tune.trace_variant, "path_budget": tune.budget,
                                     "render_batch": tune.render_batch}},
            "clocks": clock_info,
            "e2e": {"value": value, "unit": "Mrays/s",
                    "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": sum(r["width"] * r["height"] * 12 for r in reqs),
                    "note": "films are device tensors; request latency runs from submission "
                            "to the completed film"},
            "plain_per_request": {"value": plain_rays / plain_s / 1e6, "unit": "Mrays/s",
                                  "seconds": plain_s, "rays": plain_rays,
                                  "batch_paths": plain_batch,
                                  "what": "this build's lux_render, one request after the "
                                          "other, at its own batch size"},
            "plain_per_request_reference_batch": {
                "value": ref_rays / ref_s / 1e6 if ref_rays else None, "unit": "Mrays/s",
                "seconds": ref_s, "batch_paths": 65536, "requests": ref_subset,
                "this_build_batch_on_same_requests_mrays_s": sub_rays / sub_s / 1e6,
                "what": "this build's lux_render at the reference scheduler's 65,536-path "
                        "batches (integrator/render_context.h:18)"},
            "speedup_vs_plain": (batch_rays / batch_s) / (plain_rays / plain_s),
            "speedup_vs_plain_reference_batch": ((batch_rays / batch_s) / (ref_rays / ref_s)
                                                 if ref_rays else None),
            "reference_gpu": reference_gpu, "roofline": roofline,
            "rays": batch_rays, "iterations": stats["iterations"] - base["iterations"],
            "max_rel_film_difference_vs_plain": rel}


def run_batched(args) -> None:
    print(json.dumps(batched_line(args)))


def _poisson_arrivals(rate: float, count: int, seed: int) -> np.ndarray:
    u = W.splitmix_uniform(seed, 31, count)
    return np.cumsum(-np.log(1.0 - u) / rate)


def _displaced(base: np.ndarray, frame: int) -> np.ndarray:
    """Sinusoidal vertex displacement of the animated icosphere at a frame."""
    v = base.copy()
    phase = 0.35 * frame
    v[:, 1] += 0.02 * np.sin(6.0 * v[:, 0] + phase)
    return v


def serving_line(args, rates: list[float]) -> dict:
    """Config 5: Poisson arrivals over the resident scenes; the displaced icosphere is
    refit every frame; p50/p99 latency and Mrays/s, against a FIFO one-request-at-a-time
    server built from the per-request path's measured service times."""
    import threading

    torch, ctx, stream = _render_setup()
    from lux_b200 import scene as S
    from lux_b200 import scenes as SC
    from lux_b200 import server as SV

    builders = SC.resident_scenes(512, 512)
    scenes = [S.Scene(ctx, b) for b in builders]
    anim_scene, anim_mesh = 1, 1
    base = builders[anim_scene].meshes[anim_mesh].vertices.copy()
    frame_s = 1.0 / args.refit_hz if args.refit_hz > 0 else None
    results = []
    clocks = ClockSampler(0)
    clocks.start()
    for ri, rate in enumerate(rates):
        reqs = SC.batched_requests(args.requests, seed=100 + ri)
        if args.request_scale != 1.0:
            for r in reqs:
                side = max(16, int(r["width"] * args.request_scale))
                r["width"] = r["height"] = side
                r["spp"] = max(1, int(r["spp"] * args.request_scale))
        arrivals = _poisson_arrivals(rate, len(reqs), seed=200 + ri)
        rr = [S.request(r["width"], r["height"], r["spp"], r["max_depth"], r["seed"])
              for r in reqs]
        films = [torch.zeros((r["height"], r["width"], 3), device="cuda") for r in reqs]
        # Per-request service times (plain path), for the FIFO comparison; the plain
        # runtime is first sized for the largest request of the mix (no allocation is
        # timed).
        largest = max(range(len(reqs)), key=lambda k: reqs[k]["width"] ** 2 * reqs[k]["spp"])
        for sc_i in range(len(scenes)):
            S.render(ctx, scenes[sc_i], rr[largest], films[largest])
        torch.cuda.synchronize()
        service, host_service, plain_rays = [], [], 0
        for r, q, f in zip(reqs, rr, films):
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            h0 = time.perf_counter()
            e0.record(stream)
            S.render(ctx, scenes[r["scene"]], q, f)
            e1.record(stream)
            torch.cuda.synchronize()
            host_service.append(time.perf_counter() - h0)
            service.append(e0.elapsed_time(e1) * 1e-3)
            plain_rays += sum(S.ray_counts(ctx))
        free_at, fifo_lat = 0.0, []
        for a, sv in zip(arrivals, service):
            start = max(a, free_at)
            free_at = start + sv
            fifo_lat.append(free_at - a)
        with SV.Server(scenes, pool_paths=args.pool,
                       memory_budget_bytes=int(args.budget_gb * 1e9)) as srv:
            warm, _ = srv.submit(0, S.request(32, 32, 2, 2, 1))
            srv.wait(warm)
            base_stats = srv.stats()
            ids = [None] * len(reqs)
            stop = threading.Event()

            def animate():
                frame = 0
                while frame_s is not None and not stop.wait(frame_s):
                    frame += 1
                    srv.update_mesh(anim_scene, anim_mesh, _displaced(base, frame))

            anim = threading.Thread(target=animate)
            anim.start()
            t0 = time.perf_counter()
            for k, (r, q, f) in enumerate(zip(reqs, rr, films)):
                delay = arrivals[k] - (time.perf_counter() - t0)
                if delay > 0:
                    time.sleep(delay)
                ids[k] = srv.submit(r["scene"], q, f)[0]
            try:
                srv.wait_all(timeout_s=600)
            finally:
                stop.set()
                anim.join()
            stats = srv.stats()
            lat = [(srv.times(i)[2] - srv.times(i)[0]) * 1e-9 for i in ids]
            span = (max(srv.times(i)[2] for i in ids) - min(srv.times(i)[0] for i in ids)) * 1e-9
        rays = (stats["rays"] - base_stats["rays"]) + (stats["shadow_rays"] - base_stats["shadow_rays"])
        results.append({"rate_req_s": rate, "requests": len(reqs),
                        "p50_ms": float(np.percentile(lat, 50) * 1e3),
                        "p99_ms": float(np.percentile(lat, 99) * 1e3),
                        "mrays_s": rays / span / 1e6, "span_s": span, "refits": stats["refits"],
                        "fifo_plain_p50_ms": float(np.percentile(fifo_lat, 50) * 1e3),
                        "fifo_plain_p99_ms": float(np.percentile(fifo_lat, 99) * 1e3),
                        "fifo_plain_mrays_s": plain_rays / max(free_at, 1e-9) / 1e6,
                        "plain_service_ms": {"p50": float(np.percentile(service, 50) * 1e3),
                                             "max": float(np.max(service) * 1e3),
                                             "argmax": int(np.argmax(service)),
                                             "argmax_host_ms": float(host_service[int(np.argmax(service))] * 1e3),
                                             "argmax_request": reqs[int(np.argmax(service))]}})
    clock_info = clocks.stop()
    best = max(results, key=lambda r: r["mrays_s"])
    return {"metric": "p50/p99 render-request latency and Mrays/s (served)",
            "value": best["mrays_s"], "unit": "Mrays/s", "n_gpus": 1, "steps": len(rates),
            "warmup": 1, "ms_per_step": float(np.mean([r["span_s"] for r in results]) * 1e3),
            "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {"workload": "Poisson arrivals over the 4 resident scenes; requests from the "
                                   "batched distribution scaled by %g; displaced icosphere refit "
                                   "every 1/%g s" % (args.request_scale, args.refit_hz),
                       "pool_paths": args.pool, "memory_budget_gb": args.budget_gb},
            "clocks": clock_info,
            "e2e": {"value": best["mrays_s"], "unit": "Mrays/s", "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0,
                    "note": "latency is submission to completed film, arrivals in real time"},
            "p50_ms": {str(r["rate_req_s"]): r["p50_ms"] for r in results},
            "p99_ms": {str(r["rate_req_s"]): r["p99_ms"] for r in results},
            "sweep": results}


def run_serving(args) -> None:
    print(json.dumps(serving_line(args, [float(r) for r in args.rates.split(",")])))


def render_suite(args) -> dict:
    """The render configurations nested in the default line: config 1 (Cornell, 20 timed
    frames), config 3 (heavy, 3 frames), config 4 (batched mix) and a three-rate sweep of
    config 5 (serving), each with its own clocks, e2e, roofline and baselines."""
    out = {}
    t0 = time.perf_counter()
    for name, steps, warmup in (("cornell", 20, 3), ("heavy", 3, 1)):
        s = time.perf_counter()
        out[name] = render_line(args, name, steps, warmup, nested=True)
        out[name]["leg_wall_s"] = time.perf_counter() - s
    s = time.perf_counter()
    out["batched"] = batched_line(args, nested=True)
    out["batched"]["leg_wall_s"] = time.perf_counter() - s
    s = time.perf_counter()
    out["serving"] = serving_line(args, [10.0, 100.0, 500.0])
    out["serving"]["leg_wall_s"] = time.perf_counter() - s
    out["wall_s"] = time.perf_counter() - t0
    return out


def main():
    global N_TRIS, N_RAYS, N_QUERIES, WORKLOAD
    ap = argparse.ArgumentParser()
    ap.add_argument("--config", default="lbvh", choices=["lbvh", "cornell", "heavy", "batched", "serving"],
                    help="lbvh: the LBVH microbench (default); cornell: config 1; heavy: config 3; "
                         "batched: config 4; serving: config 5")
    ap.add_argument("--rates", default="10,50,100,200,500")
    ap.add_argument("--render-size", type=int, default=0,
                    help="cornell/heavy: film side override (profiling cases only)")
    ap.add_argument("--render-spp", type=int, default=0,
                    help="cornell/heavy: samples per pixel override (profiling cases only)")
    ap.add_argument("--refit-hz", type=float, default=30.0,
                    help="serving: displaced-icosphere refits per second (0: none)")
    ap.add_argument("--budget-gb", type=float, default=120.0,
                    help="serving: device-memory admission budget for queues and films")
    ap.add_argument("--request-scale", type=float, default=0.25,
                    help="serving: scale of request resolution and spp")
    ap.add_argument("--requests", type=int, default=64)
    ap.add_argument("--skip-reference-batch", action="store_true",
                    help="batched: skip the plain pass at the reference's 65,536-path batch")
    ap.add_argument("--pool", type=int, default=1 << 22,
                    help="paths in flight of the serving configuration's server")
    ap.add_argument("--batch-pool", type=int, default=1 << 23,
                    help="paths in flight of the batched configuration's server (4M: 964, "
                         "8M: 993, 16M: 997 Mrays/s on one B200)")
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=50)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="lux", choices=["lux", "reference"])
    ap.add_argument("--skip-e2e", action="store_true")
    ap.add_argument("--skip-render", action="store_true",
                    help="lbvh: leave out the nested render configurations (1, 3, 4, 5)")
    ap.add_argument("--skip-cpu-baseline", action="store_true")
    ap.add_argument("--skip-reference-gpu", action="store_true",
                    help="lbvh: skip timing the reference's own GPU LBVH code")
    ap.add_argument("--tris", type=int, default=N_TRIS,
                    help="smaller cases for profiling captures only")
    ap.add_argument("--rays", type=int, default=N_RAYS)
    ap.add_argument("--queries", type=int, default=N_QUERIES)
    ap.add_argument("--trace-variant", type=int, default=0,
                    help="0 auto, 1 one thread per ray, 2 persistent (tunable)")
    ap.add_argument("--trace-budget", type=int, default=16)
    ap.add_argument("--no-autotune", action="store_true",
                    help="cornell/heavy: skip the autotuner and render with --trace-variant "
                         "(profiling captures, so the first launches are the render's)")
    args = ap.parse_args()
    if (args.tris, args.rays, args.queries) != (N_TRIS, N_RAYS, N_QUERIES):
        N_TRIS, N_RAYS, N_QUERIES = args.tris, args.rays, args.queries
        WORKLOAD = (f"LBVH microbench generator at reduced size (profiling case): {N_TRIS} "
                    f"triangles, {N_RAYS} rays, {N_QUERIES} query boxes, seed 7")
    if args.config in ("cornell", "heavy") and args.impl == "lux":
        run_render(args, args.config)
    elif args.config == "batched":
        run_batched(args)
    elif args.config == "serving":
        run_serving(args)
    elif args.impl == "reference":
        run_reference(args)
    else:
        run_lux(args)


if __name__ == "__main__":
    main()
