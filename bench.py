"""Benchmark of the packed strand generator on B200.

Workload (per GPU): the single large description -- displaced sphere with
200,000 triangles, 4,096 guides of 32 CVs, 8-guide stencils, 1,000,000
strands x 32 points, taper 0.02 -> 0.002, noise 0.2 at frequency 12 --
written as float4(position, radius) plus point counts, roots and root UVs,
the outputs of the reference's generate_packed_cpu (asset.cpp:412-449).

A step is one generation of that workload with inputs resident in HBM.
The L2 is flushed (a 256 MiB write) between timed steps.  With N GPUs each
rank generates its own 1,000,000-strand range of an N x 1,000,000-strand
description (weak scaling; strands are independent, so there is no
collective on the data path).

    python bench.py [--gpus N --steps K --warmup W] [--impl reference]
"""
from __future__ import annotations

import argparse
import json
import os
import re
import statistics
import subprocess
import sys
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

STRANDS_PER_GPU = 1_000_000
FALLBACK_HBM_GBS = 6650.0
# strand_keys, exclusive_scan, scatter_order (the strand order), guide_offsets,
# strand_roots, generate
# Launches per step of the large workload: strand keys, bin scan, scatter,
# guide offsets, then the lane-walk generator (tile lanes 1) or strand roots
# plus the lane-group generator.
def kernels_per_step(tile) -> int:
    return 5 if tile[0] == 1 else 6


def parse_args():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=50)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", choices=["nxg", "reference"], default="nxg")
    ap.add_argument("--workload", choices=["large", "batched", "motion", "classic", "batched_classic",
                                           "asset_build", "classic_fx", "curve_cache", "payload"],
                    default="large",
                    help="large: the single large description (headline); batched: nine descriptions in one "
                         "persistent launch vs. one launch per description; motion: five shutter samples of the "
                         "large description in one graph")
    ap.add_argument("--strands", type=int, default=STRANDS_PER_GPU, help="strands per GPU")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--cpu-seconds", type=float, default=12.0, help="CPU-baseline budget")
    ap.add_argument("--tile", type=str, default=None,
                    help="lanes,cvs_per_lane,block_size of the generate kernel (default: autotuned in warm-up)")
    ap.add_argument("--noise-amplitude", type=float, default=None,
                    help="override the workload's noise magnitude (0 = the noise-free path)")
    ap.add_argument("--no-autotune", action="store_true",
                    help="batched workloads: keep the library's default tiles instead of timing tiles in warm-up")
    return ap.parse_args()


def measured_peak():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(path) as fh:
            return float(json.load(fh)["hbm_gbs"]), "measured"
    except (OSError, ValueError, KeyError):
        return FALLBACK_HBM_GBS, "fallback"


def profile_traffic_per_point(walk: bool = True):
    """DRAM bytes per generated point of the generate kernel (the lane-walk
    kernel, or the lane-group kernel), from the ncu summary committed under
    profiles/ (None until one exists)."""
    name = "generate_walk_kernel_large_sphere.md" if walk else "generate_kernel_large_sphere.md"
    path = os.path.join(ROOT, "profiles", name)
    try:
        with open(path) as fh:
            m = re.search(r"traffic_bytes_per_point:\s*([0-9.eE+-]+)", fh.read())
            return float(m.group(1)) if m else None
    except OSError:
        return None


def profile_instructions_per_strand(walk: bool, noise: bool):
    """Warp instructions per generated strand of the generate kernel, from the
    ncu summary committed under profiles/ (None until one exists)."""
    if not walk:
        return None, None
    name = "generate_walk_kernel_large_sphere.md" if noise else "generate_walk_kernel_plain_large_sphere.md"
    try:
        with open(os.path.join(ROOT, "profiles", name)) as fh:
            m = re.search(r"warp_instructions_per_strand:\s*([0-9.eE+-]+)", fh.read())
            return (float(m.group(1)), "profiles/" + name) if m else (None, None)
    except OSError:
        return None, None


def issue_ceiling(walk: bool, noise: bool, strands: int, alg_bytes: int, peak: float, sm_mhz):
    """The HBM fraction the generate kernel would reach if every SM issued one
    warp instruction per scheduler per cycle: instructions per strand (ncu) x
    strands / (148 SMs x 4 schedulers x clock)."""
    per, source = profile_instructions_per_strand(walk, noise)
    if per is None:
        return None
    mhz = sm_mhz or 1965.0
    ms = per * strands / (148 * 4 * mhz * 1e6) * 1e3
    return {"warp_instructions_per_strand": per, "ms_at_full_issue": ms,
            "frac_at_full_issue": alg_bytes / (ms / 1e3) / 1e9 / peak, "sm_mhz": mhz, "source": source}


def limiter(frac: float, issue) -> str:
    if frac >= 0.6:
        return "hbm"
    if issue is not None and issue["frac_at_full_issue"] < 1.0:
        return "instruction issue and latency (frac_at_full_issue < 1)"
    return "latency"


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.gpu = gpu_index
        self.proc = None

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.gpu), "--query-gpu=" + self.FIELDS, "--format=csv,noheader,nounits",
                 "-lms", "50"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except OSError:
            self.proc = None

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            out, _ = self.proc.communicate(timeout=10)
        except subprocess.TimeoutExpired:
            self.proc.kill()
            out, _ = self.proc.communicate()
        sm, mx, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in out.strip().splitlines():
            parts = [p.strip() for p in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                mx.append(float(parts[2]))
            except ValueError:
                continue
            for name, flag in zip(names, parts[5:9]):
                if flag.lower() == "active":
                    reasons.add(name)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": sorted(reasons), "samples": len(sm)}


def workload(strands_total: int):
    from nanoxgen_b200 import fixtures
    w = fixtures.large_sphere(strands=strands_total)
    return w


def cpu_model() -> str:
    try:
        with open("/proc/cpuinfo") as fh:
            for line in fh:
                if line.startswith("model name"):
                    return line.split(":", 1)[1].strip()
    except OSError:
        pass
    return "unknown"


def _percentile(values, q: float) -> float:
    v = sorted(values)
    return v[min(len(v) - 1, int(round(q * (len(v) - 1))))]


def _reference_runner(blob):
    """run(n, workers, want_output) -> (seconds, outputs) over the first n
    strands: the reference's generate_packed_cpu (oracle/_ref) where it is
    built, else the oracle's C restatement; plus the kind and the
    validation-only timer (the reference hashes the asset inside every call)."""
    from oracle.checker import Oracle, Reference, reference_available
    if reference_available():
        ref = Reference()
        handle = ref.handle(blob)

        def run(params, n, workers, want_output=False):
            t0 = time.perf_counter()
            out = ref.generate(handle, params.copy(strand_count=n), 1.0, workers=workers, want_output=want_output)
            return time.perf_counter() - t0, out

        def validate():
            t0 = time.perf_counter()
            ref.validate_asset(blob)
            return time.perf_counter() - t0
        return run, validate, "reference"
    orc = Oracle()

    def run(params, n, workers, want_output=False):
        t0 = time.perf_counter()
        out = orc.generate(blob, params.copy(strand_count=n), 1.0, count=n, threads=workers)
        return time.perf_counter() - t0, out

    def validate():
        t0 = time.perf_counter()
        orc.validate_asset(blob)
        return time.perf_counter() - t0
    return run, validate, "port"


def cpu_baseline(blob, params, seconds: float, diag: float, gpu_points=None, gpu_triangles=None):
    """The reference's generate_packed_cpu (oracle/_ref) on all host cores over
    a bounded prefix sample of the workload's strands: one warm-up, then
    median and p90 of 7 calls (the reference's tools/benchmark.cpp:62-80
    pattern), one single-thread sample, the per-call asset validation timed
    on its own; and, when the GPU's output is given, the largest distance
    between the GPU's points and the reference's over the first strands."""
    import numpy as np
    cores = os.cpu_count() or 1
    run, validate, kind = _reference_runner(blob)
    P = int(params.cvs_per_strand)
    probe = 20_000
    per_strand = run(params, probe, cores)[0] / probe
    reps = 7
    n = int(min(params.strand_count, max(probe, seconds / (reps + 1) / max(per_strand, 1e-9))))
    run(params, n, cores)
    times = [run(params, n, cores)[0] for _ in range(reps)]
    med, p90 = statistics.median(times), _percentile(times, 0.9)
    val = statistics.median([validate() for _ in range(3)])
    n1 = max(2_000, n // cores)
    single = statistics.median([run(params, n1, 1)[0] for _ in range(3)])
    out = {"value": n * P / med, "unit": "points/s", "cores": cores, "kind": kind, "cpu_model": cpu_model(),
           "sample": "first %d strands x %d CVs of the workload; median of %d calls after one warm-up "
                     "(%.3f s; p90 %.3f s), including the per-call asset validation" % (n, P, reps, med, p90),
           "median_s": med, "p90_s": p90,
           "value_p90": n * P / p90,
           "value_without_validation": n * P / max(med - val, 1e-9), "validation_s": val,
           "single_thread": {"value": n1 * P / single, "strands": n1, "median_s": single, "calls": 3}}
    if gpu_points is not None:
        m = min(n, 20_000)
        _, ref_out = run(params, m, cores, want_output=True)
        rpts, rroots = ref_out[0], ref_out[1]
        d = gpu_points[:m * P, :3].astype(np.float64) - rpts[:m * P, :3].astype(np.float64)
        err = float(np.sqrt((d * d).sum(-1)).max())
        rerr = float(np.abs(gpu_points[:m * P, 3].astype(np.float64) - rpts[:m * P, 3]).max())
        out["parity"] = {"strands_checked": m, "max_error_rel_diag": err / diag,
                         "max_radius_error_rel_diag": rerr / diag, "tolerance_rel_diag": 1e-5,
                         "root_triangles_equal": bool(gpu_triangles is not None and
                                                      np.array_equal(gpu_triangles[:m], rroots["triangle_index"]))}
    return out


def run_reference_arm(args):
    """The reference's own generate_packed_cpu on the host cores, on the asset
    its own build_asset makes from the workload (nothing of this library is
    loaded on this arm)."""
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    from oracle.checker import Reference, reference_available
    w = workload(args.strands)
    if not reference_available():
        print(json.dumps({"impl": "reference", "unavailable": "the reference library oracle/_ref/libnxg_ref.so is "
                          "not built and the reference sources are absent"}), flush=True)
        return
    blob = Reference().build_asset(w.build_input)
    if w.stencil_slots != 8:
        raise SystemExit("the headline workload uses 8-guide stencils")
    cores = os.cpu_count() or 1
    P = int(w.params.cvs_per_strand)
    run, validate, kind = _reference_runner(blob)
    per = run(w.params, 20_000, cores)[0] / 20_000
    budget = 90.0 / max(1, args.steps + args.warmup)
    n = int(min(w.params.strand_count, max(20_000, min(2.0, budget) / max(per, 1e-9))))
    for _ in range(args.warmup):
        run(w.params, n, cores)
    times = [run(w.params, n, cores)[0] for _ in range(args.steps)]
    total = sum(times)
    value = args.steps * n * P / total
    line = {"metric": "points/sec", "value": value, "unit": "points/s", "n_gpus": args.gpus, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": 1e3 * total / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "impl": "reference",
            "config": {"workload": w.name, "strands_per_step": n, "cvs_per_strand": P,
                       "note": "generate_packed_cpu on the host cores over a prefix sample of the workload; "
                               "asset made by the reference's build_asset"},
            "cpu_baseline": {"value": value, "unit": "points/s", "cores": cores, "kind": kind,
                             "cpu_model": cpu_model(),
                             "sample": "first %d strands x %d CVs per step (median %.3f s, p90 %.3f s)"
                                       % (n, P, statistics.median(times), _percentile(times, 0.9))},
            "e2e": {"value": value, "unit": "points/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def run_gpu_arm(args):
    import torch

    from nanoxgen_b200.asset import build_asset
    from nanoxgen_b200.generator import (DeviceAsset, HostPipeline, allocate_outputs, autotune,
                                         generate_packed_ordered, prepare_strand_order, set_tile)

    from nanoxgen_b200 import distributed

    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    device = torch.device("cuda", local)
    rank, world = distributed.init("nccl", device)

    def barrier():
        distributed.barrier()

    def max_over_ranks(x: float) -> float:
        return distributed.max_over_ranks(x, device)

    S = args.strands
    first, _ = distributed.shard(S, rank)
    w = workload(S * world)
    if args.noise_amplitude is not None:
        w.params = w.params.copy(noise_amplitude=args.noise_amplitude)
    params = w.params
    P = int(params.cvs_per_strand)
    asset = build_asset(w.build_input, w.stencil_slots)
    dasset = DeviceAsset(asset, device)
    points, roots, uvs, counts = allocate_outputs(S, P, device)
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=device)
    stream = torch.cuda.current_stream(device)

    def step(ev=None):
        ws = prepare_strand_order(dasset, params, first, S, stream=stream)
        if ev is not None:
            ev.record(stream)
        generate_packed_ordered(dasset, params, points, roots, uvs, counts, 1.0, None, first, S, ws, stream=stream)

    noise = params.noise_amplitude != 0.0 and params.noise_mask != 0.0
    if args.tile:
        lanes, ppt, block = (int(x) for x in args.tile.split(","))
        set_tile(P, noise, lanes, ppt, block)
        tile = (lanes, ppt, block)
    else:
        tile, _ = autotune(dasset, params, points, first_strand=first, count=S, repeats=2)
    for _ in range(args.warmup):
        flush.fill_(1)
        step()
    torch.cuda.synchronize(device)

    sampler = ClockSampler(local)
    sampler.start()
    barrier()
    torch.cuda.synchronize(device)
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True),
           torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
    for k in range(args.steps):
        flush.fill_(k & 0xFF)
        ev[k][0].record(stream)
        step(ev[k][1])
        ev[k][2].record(stream)
    torch.cuda.synchronize(device)
    barrier()
    step_ms = [a.elapsed_time(c) for a, b, c in ev]
    kern_ms = [b.elapsed_time(c) for a, b, c in ev]
    total_ms = max_over_ranks(sum(step_ms))
    kernel_ms = max_over_ranks(statistics.mean(kern_ms))

    e2e = None
    if not args.no_e2e:
        pipe = HostPipeline(asset, params, 1.0, chunks=8, device=device, first_strand=first, count=S)
        for _ in range(max(1, min(args.warmup, 3))):
            pipe.run()
        torch.cuda.synchronize(device)
        barrier()
        torch.cuda.synchronize(device)
        e_start, e_stop = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e_start.record(pipe.compute)
        for _ in range(args.steps):
            pipe.run()
        pipe.compute.wait_stream(pipe.copy)
        e_stop.record(pipe.compute)
        torch.cuda.synchronize(device)
        barrier()
        e2e_ms = max_over_ranks(e_start.elapsed_time(e_stop))
        pts = pipe.host_points.numpy()
        assert pts.shape[0] == S * P and float(abs(pts[:, 3]).max()) > 0.0
        e2e = {"value": world * S * P * args.steps / (e2e_ms / 1e3), "unit": "points/s",
               "h2d_bytes_per_step": pipe.h2d_bytes, "d2h_bytes_per_step": pipe.d2h_bytes,
               "ms_per_step": e2e_ms / args.steps,
               "path": "HostPipeline: pinned asset upload, nxg_generate_packed_range in 8 ranges, "
                       "overlapped D2H of points/roots/root_uvs/point_counts to pinned host arrays"}
    clocks = sampler.stop()

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        m = min(S, 20_000)
        gpu_pts = points[:m * P].cpu().numpy()
        gpu_tris = roots.view(-1, 12)[:m, 8].cpu().numpy().view("uint32")
        cpu = cpu_baseline(asset.buffer, params.copy(strand_count=S), args.cpu_seconds, asset.bbox_diagonal(),
                           gpu_pts, gpu_tris)

    distributed.finalize()
    if rank != 0:
        return

    ms_per_step = total_ms / args.steps
    points_total = world * S * P
    out_bytes = S * P * 16 + S * (48 + 8 + 4)
    alg_bytes = out_bytes + asset.nbytes
    peak, peak_kind = measured_peak()
    achieved = alg_bytes / (kernel_ms / 1e3) / 1e9
    tpp = profile_traffic_per_point(tile[0] == 1)
    issue = issue_ceiling(tile[0] == 1, noise, S, alg_bytes, peak, clocks.get("sm_mhz"))
    if tile[0] != 1:
        kernel_name = "generate_kernel<%d,%d,%s>" % (tile[0], tile[1], "noise" if noise else "plain")
    elif noise and tile[2] <= 64:
        kernel_name = "generate_pipe_kernel"
    else:
        kernel_name = "generate_walk_kernel<%s>" % ("noise" if noise else "plain")
    line = {
        "metric": "points/sec", "value": points_total / (ms_per_step / 1e3), "unit": "points/s",
        "n_gpus": world, "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_per_step,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic",
        "config": {"workload": w.name, "triangles": int(asset.header.triangle_count),
                   "guides": int(asset.header.guide_count), "stencil_slots": w.stencil_slots,
                   "strands_per_gpu": S, "cvs_per_strand": P, "noise_amplitude": params.noise_amplitude,
                   "noise_frequency": params.noise_frequency, "outputs": "points,roots,root_uvs,point_counts",
                   "l2": "flushed between timed steps (256 MiB write); outputs 572 MB > L2",
                   "parallelism": "strand ranges per GPU (no collective)"},
        "hbm_gbs": world * alg_bytes / (ms_per_step / 1e3) / 1e9,
        "tile": {"lanes_per_strand": tile[0], "cvs_per_lane": tile[1], "block_size": tile[2],
                 "chosen_by": "--tile" if args.tile else "nxg_autotune_packed in warm-up"},
        "roofline": {"bound": "hbm", "kernel": kernel_name,
                     "achieved": achieved,
                     "peak": peak, "unit": "GB/s", "frac": achieved / peak, "peak_source": peak_kind,
                     "traffic": (tpp * S * P) if tpp else None,
                     "algorithmic_bytes": alg_bytes, "kernel_ms": kernel_ms,
                     "limiter": limiter(achieved / peak, issue),
                     "issue_ceiling": issue,
                     "note": "algorithmic bytes = 16 B/point + 60 B/strand (roots, root UVs, counts) + asset; "
                             "'bound' names the roofline the fraction is taken against, 'limiter' what the "
                             "profile shows limiting the kernel"},
        "clocks": clocks, "gpu_launches": kernels_per_step(tile) * args.steps,
    }
    parity_ok = True
    if cpu and "parity" in cpu:
        par = cpu["parity"]
        line["max_error_rel_diag"] = par["max_error_rel_diag"]
        parity_ok = (par["max_error_rel_diag"] <= par["tolerance_rel_diag"] and
                     par["max_radius_error_rel_diag"] <= par["tolerance_rel_diag"] and par["root_triangles_equal"])
        line["parity_ok"] = parity_ok
    if e2e:
        line["e2e"] = e2e
    if cpu:
        line["cpu_baseline"] = cpu
    print(json.dumps(line), flush=True)
    if not parity_ok:  # a fast wrong answer is not a result
        raise SystemExit("the generated points differ from the reference's beyond the tolerance")


def _graph_time(device, fn, steps: int, warmup: int, flush) -> list:
    """Capture `fn` in a CUDA graph and time `steps` replays with events,
    flushing L2 between replays; returns per-replay milliseconds."""
    import torch
    s = torch.cuda.Stream(device)
    s.wait_stream(torch.cuda.current_stream(device))
    with torch.cuda.stream(s):
        fn(s)  # untimed eager run (also allocates cached workspaces)
    torch.cuda.synchronize(device)
    g = torch.cuda.CUDAGraph()
    with torch.cuda.graph(g, stream=s):
        fn(s)
    for _ in range(warmup):
        flush.fill_(1)
        g.replay()
    torch.cuda.synchronize(device)
    out = []
    for k in range(steps):
        flush.fill_(k & 0xFF)
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record()
        g.replay()
        b.record()
        torch.cuda.synchronize(device)
        out.append(a.elapsed_time(b))
    del g
    return out


def run_batched(args):
    """Nine descriptions on one 500,000-triangle mesh (log-uniform strand
    counts, 8..64 CVs, stencils of 4 or 8, noise on two in three) in one
    persistent launch, graph-captured, tiles autotuned per (CVs, noise);
    compared with the plain path (one nxg_generate_packed per description,
    in one graph)."""
    import torch

    from nanoxgen_b200 import fixtures
    from nanoxgen_b200.asset import build_asset
    from nanoxgen_b200.generator import BatchRunner, DeviceAsset, autotune, generate_packed
    device = torch.device("cuda", 0)
    torch.cuda.set_device(device)
    batch = fixtures.batched_descriptions()
    assets = [build_asset(w.build_input, w.stencil_slots) for w in batch.workloads]
    dassets = [DeviceAsset(a, device) for a in assets]
    runner = BatchRunner(dassets, [w.params for w in batch.workloads])
    tuned = {}
    for w, d, o in zip(batch.workloads, dassets, runner.outputs):
        key = (int(w.params.cvs_per_strand), w.params.noise_amplitude != 0.0)
        if key not in tuned:
            tuned[key] = "default" if args.no_autotune else autotune(d, w.params, o[0], repeats=2)[0]
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=device)
    sampler = ClockSampler(0)
    sampler.start()
    batched_ms = _graph_time(device, lambda s: runner.run(stream=s), args.steps, args.warmup, flush)

    def plain(s):
        for w, d, o in zip(batch.workloads, dassets, runner.outputs):
            generate_packed(d, w.params, points=o[0], roots=o[1], root_uvs=o[2], point_counts=o[3], stream=s)
    plain_ms = _graph_time(device, plain, args.steps, args.warmup, flush)
    clocks = sampler.stop()
    ms = statistics.mean(batched_ms)
    pms = statistics.mean(plain_ms)
    points = batch.points
    line = {"metric": "points/sec", "value": points / (ms / 1e3), "unit": "points/s", "n_gpus": 1,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {"workload": batch.name, "descriptions": [w.name for w in batch.workloads],
                       "strands": batch.strands, "points": points,
                       "tiles": {"%d%s" % (k[0], "n" if k[1] else ""): v for k, v in tuned.items()},
                       "l2": "flushed between timed replays (256 MiB write)"},
            "plain_path": {"ms_per_step": pms, "value": points / (pms / 1e3),
                           "how": "one nxg_generate_packed per description, all in one CUDA graph"},
            "batched_speedup_vs_plain": pms / ms, "clocks": clocks, "gpu_launches": 7 * args.steps}
    print(json.dumps(line), flush=True)


def run_motion(args):
    """Five shutter samples of the single large description (per-vertex
    sinusoidal displacement, amplitude 0.03) written to five float4 buffers by
    one nxg_generate_motion_packed call, replayed as one CUDA graph."""
    import numpy as np
    import torch

    from nanoxgen_b200 import fixtures
    from nanoxgen_b200.asset import build_asset
    from nanoxgen_b200.generator import (DeformedGeometry, DeviceAsset, allocate_outputs, autotune,
                                         generate_motion_packed)
    device = torch.device("cuda", 0)
    torch.cuda.set_device(device)
    w = workload(args.strands)
    asset = build_asset(w.build_input, w.stencil_slots)
    d = DeviceAsset(asset, device)
    frames = fixtures.motion_frames(w.build_input, 5)
    dev = lambda a: torch.from_numpy(np.ascontiguousarray(a)).to(device)
    geoms = [DeformedGeometry(dev(p), dev(n), dev(g)) for p, n, g in zip(frames.positions, frames.normals,
                                                                            frames.guide_cvs)]
    S, P = int(w.params.strand_count), int(w.params.cvs_per_strand)
    outputs = [allocate_outputs(S, P, device) for _ in geoms]
    tile = autotune(d, w.params, outputs[0][0], repeats=2)[0]
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=device)
    sampler = ClockSampler(0)
    sampler.start()
    times = _graph_time(device, lambda s: generate_motion_packed(d, w.params, geoms, frames.times,
                                                                 outputs=outputs, stream=s),
                        args.steps, args.warmup, flush)
    clocks = sampler.stop()
    ms = statistics.mean(times)
    points = 5 * S * P
    alg = 5 * (S * P * 16 + S * 60) + asset.nbytes + sum(g.positions.numel() * 8 + g.guide_cvs.numel() * 4
                                                         for g in geoms)
    peak, kind = measured_peak()
    line = {"metric": "points/sec", "value": points / (ms / 1e3), "unit": "points/s", "n_gpus": 1,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {"workload": w.name + "/5-motion-samples", "samples": 5, "strands": S, "cvs_per_strand": P,
                       "tile": tile, "l2": "flushed between timed replays (256 MiB write)"},
            "hbm_gbs": alg / (ms / 1e3) / 1e9, "hbm_frac": alg / (ms / 1e3) / 1e9 / peak, "peak_source": kind,
            "clocks": clocks, "gpu_launches": (4 + 3 * 5) * args.steps}
    print(json.dumps(line), flush=True)


def _train_surrogate(dasset, asset, params, plan, samples: int, epochs: int):
    """A surrogate trained on `samples` roots of `params` (training seed) with
    targets from the exact runtime; returns (model, seconds)."""
    import torch

    from nanoxgen_b200.classic import check_status, root_scalars
    from nanoxgen_b200.surrogate import Surrogate, asset_input_normalisation
    tp = params.copy(strand_count=samples, seed=int(params.seed) + 7919)
    off, sc = asset_input_normalisation(asset)
    t0 = time.perf_counter()
    model = Surrogate(dasset.device, off, sc, seed=3)
    feats = Surrogate.features(dasset, tp)
    targets, status = root_scalars(dasset, tp, plan)
    torch.cuda.synchronize()
    check_status(status)
    targets = targets[:samples].contiguous()
    model.fit_outputs(targets)
    result = model.train(feats, targets, epochs=epochs, batch=16384, learning_rate=3e-3, lr_decay=0.85)
    torch.cuda.synchronize()
    return model, time.perf_counter() - t0, result


def _relative_errors(got, exact):
    import numpy as np
    g = got.cpu().numpy().astype(np.float64)
    e = exact.cpu().numpy().astype(np.float64)
    rel = np.abs(g - e) / np.abs(e)
    return {"length_max": float(rel[:, 0].max()), "length_p99": float(np.percentile(rel[:, 0], 99)),
            "length_mean": float(rel[:, 0].mean()), "width_max": float(rel[:, 1].max()),
            "width_p99": float(np.percentile(rel[:, 1], 99))}


def run_classic(args):
    """Learned-expression workload: 4,000,000 strands x 24 points on the
    200,000-triangle sphere with Classic length / width expressions.  The
    exact runtime (nxg_classic_root_scalars) and the tensor-core surrogate
    (trained here on 1M exact samples, judged per 128-root batch at 1e-3
    relative error, adaptive) feed nxg_generate_packed_classic; each path is
    one CUDA graph replay per step."""
    import numpy as np
    import torch

    from nanoxgen_b200 import fixtures
    from nanoxgen_b200.asset import build_asset
    from nanoxgen_b200.classic import Expression, ScalarPlan, generate_packed_classic, root_scalars
    from nanoxgen_b200.generator import DeviceAsset, allocate_outputs
    device = torch.device("cuda", 0)
    torch.cuda.set_device(device)
    strands = args.strands if args.strands != STRANDS_PER_GPU else 4_000_000
    w = fixtures.classic_sphere(strands=strands)
    asset = build_asset(w.build_input, w.stencil_slots)
    d = DeviceAsset(asset, device)
    params = w.params
    S, P = int(params.strand_count), int(params.cvs_per_strand)
    plan = ScalarPlan(Expression.classic(fixtures.CLASSIC_LENGTH, "length"),
                      Expression.classic(fixtures.CLASSIC_WIDTH, "width"))
    model, train_s, result = _train_surrogate(d, asset, params, plan, 1_000_000, 8)
    out = allocate_outputs(S, P, device)
    scal = torch.empty((S, 2), dtype=torch.float32, device=device)
    status2 = torch.zeros(2, dtype=torch.int32, device=device)
    status4 = torch.zeros(4, dtype=torch.int32, device=device)
    tol = 1e-3

    def exact_scalars(s):
        root_scalars(d, params, plan, out=scal, status=status2, stream=s)

    def surrogate_scalars(mode):
        return lambda s: model.root_scalars(d, params, plan, length_tolerance=tol, width_tolerance=tol,
                                            checks_per_batch=4, mode=mode, out=scal, status=status4, stream=s)

    def gen(s):
        generate_packed_classic(d, params, scal, points=out[0], roots=out[1], root_uvs=out[2],
                                point_counts=out[3], stream=s)

    # accuracy of the network alone and of the judged output, against the exact runtime
    exact_scalars(None)
    exact = scal.clone()
    surrogate_scalars(2)(None)
    network = scal.clone()
    surrogate_scalars(3)(None)  # the first adaptive launch checks every batch and sets the model's trust
    status4.zero_()
    surrogate_scalars(3)(None)
    torch.cuda.synchronize()
    judged = scal.clone()
    tiles = (S + 127) // 128
    adaptive_status = status4.cpu().tolist()
    status4.zero_()
    surrogate_scalars(0)(None)
    torch.cuda.synchronize()
    checked_status = status4.cpu().tolist()
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=device)
    sampler = ClockSampler(0)
    sampler.start()
    t = {}
    t["scalars_exact"] = _graph_time(device, exact_scalars, args.steps, args.warmup, flush)
    t["scalars_network_only"] = _graph_time(device, surrogate_scalars(2), args.steps, args.warmup, flush)
    t["scalars_judged_adaptive"] = _graph_time(device, surrogate_scalars(3), args.steps, args.warmup, flush)
    t["scalars_judged_every_batch"] = _graph_time(device, surrogate_scalars(0), args.steps, args.warmup, flush)
    t["exact_path"] = _graph_time(device, lambda s: (exact_scalars(s), gen(s)), args.steps, args.warmup, flush)
    t["surrogate_path"] = _graph_time(device, lambda s: (surrogate_scalars(3)(s), gen(s)), args.steps,
                                      args.warmup, flush)
    clocks = sampler.stop()
    ms = {k: statistics.mean(v) for k, v in t.items()}
    points = S * P
    line = {"metric": "points/sec", "value": points / (ms["surrogate_path"] / 1e3), "unit": "points/s",
            "n_gpus": 1, "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms["surrogate_path"],
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32 (network bf16)",
            "data": "synthetic",
            "config": {"workload": w.name, "strands": S, "cvs_per_strand": P, "length": fixtures.CLASSIC_LENGTH,
                       "width": fixtures.CLASSIC_WIDTH, "tolerance": tol, "checks_per_batch": 4,
                       "l2": "flushed between timed replays (256 MiB write)"},
            "exact_path": {"ms_per_step": ms["exact_path"], "value": points / (ms["exact_path"] / 1e3)},
            "scalar_stage_ms": {k[len("scalars_"):]: v for k, v in ms.items() if k.startswith("scalars_")},
            "surrogate": {"training_s": train_s, "training_samples": 1_000_000, "epochs": 8,
                          "epoch_losses": [float(x) for x in result.epoch_losses],
                          "network_only_error": _relative_errors(network, exact),
                          "judged_error": _relative_errors(judged, exact),
                          "batches": tiles,
                          "adaptive_steady_state": {"checked": adaptive_status[3],
                                                    "rerun_exactly": adaptive_status[2],
                                                    "served_by_exact_kernel": tiles - adaptive_status[3]},
                          "every_batch": {"checked": checked_status[3], "rerun_exactly": checked_status[2]}},
            "clocks": clocks, "gpu_launches": 7 * args.steps}
    print(json.dumps(line), flush=True)


def run_batched_classic(args):
    """The nine-description workload with Classic length / width expressions:
    the plain path (per description: exact scalars + generate_packed_classic)
    against the batched form (per description surrogate scalars, adaptive,
    judged at 1e-3, then one batched generate launch with the scalars fused),
    each one CUDA graph; also batched with exact scalars."""
    import torch

    from nanoxgen_b200 import fixtures
    from nanoxgen_b200.asset import build_asset
    from nanoxgen_b200.classic import Expression, ScalarPlan, generate_packed_classic, root_scalars
    from nanoxgen_b200.generator import BatchRunner, DeviceAsset, autotune
    device = torch.device("cuda", 0)
    torch.cuda.set_device(device)
    batch = fixtures.batched_descriptions()
    assets = [build_asset(w.build_input, w.stencil_slots) for w in batch.workloads]
    dassets = [DeviceAsset(a, device) for a in assets]
    params = [w.params for w in batch.workloads]
    plan = ScalarPlan(Expression.classic(fixtures.CLASSIC_LENGTH, "length"),
                      Expression.classic(fixtures.CLASSIC_WIDTH, "width"))
    runner = BatchRunner(dassets, params)
    for w, d, o in zip(batch.workloads, dassets, runner.outputs):
        autotune(d, w.params, o[0], repeats=2)
    # One network for every description: they share the mesh and the expressions.
    model, train_s, _ = _train_surrogate(dassets[0], assets[0], params[0].copy(noise_amplitude=0.0), plan,
                                         1_000_000, 8)
    scal = [torch.empty((int(p.strand_count), 2), dtype=torch.float32, device=device) for p in params]
    st2 = [torch.zeros(2, dtype=torch.int32, device=device) for _ in params]
    st4 = [torch.zeros(4, dtype=torch.int32, device=device) for _ in params]

    def exact(s):
        for d, p, t, st in zip(dassets, params, scal, st2):
            root_scalars(d, p, plan, out=t, status=st, stream=s)

    def surrogate(s):
        for d, p, t, st in zip(dassets, params, scal, st4):
            model.root_scalars(d, p, plan, length_tolerance=1e-3, width_tolerance=1e-3, checks_per_batch=4,
                               mode=3, out=t, status=st, stream=s)

    def plain(s):
        exact(s)
        for d, p, t, o in zip(dassets, params, scal, runner.outputs):
            generate_packed_classic(d, p, t, points=o[0], roots=o[1], root_uvs=o[2], point_counts=o[3], stream=s)

    flush = torch.empty(256 << 20, dtype=torch.uint8, device=device)
    sampler = ClockSampler(0)
    sampler.start()
    t_batched = _graph_time(device, lambda s: (surrogate(s), runner.run(stream=s, scalars=scal)), args.steps,
                            args.warmup, flush)
    t_batched_exact = _graph_time(device, lambda s: (exact(s), runner.run(stream=s, scalars=scal)), args.steps,
                                  args.warmup, flush)
    t_plain = _graph_time(device, plain, args.steps, args.warmup, flush)
    clocks = sampler.stop()
    # the judged scalars against the exact runtime, per strand
    exact(None)
    ref = [t.clone() for t in scal]
    for st in st4:
        st.zero_()
    surrogate(None)
    torch.cuda.synchronize()
    worst = max(_relative_errors(t, r)["length_max"] for t, r in zip(scal, ref))
    fallback = [s.cpu().tolist() for s in st4]
    ms, pms, ems = statistics.mean(t_batched), statistics.mean(t_plain), statistics.mean(t_batched_exact)
    points = batch.points
    line = {"metric": "points/sec", "value": points / (ms / 1e3), "unit": "points/s", "n_gpus": 1,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32 (network bf16)", "data": "synthetic",
            "config": {"workload": batch.name + "/classic-length-width", "strands": batch.strands, "points": points,
                       "tolerance": 1e-3, "checks_per_batch": 4, "judge": "adaptive",
                       "l2": "flushed between timed replays (256 MiB write)"},
            "plain_path": {"ms_per_step": pms, "value": points / (pms / 1e3),
                           "how": "per description nxg_classic_root_scalars + nxg_generate_packed_classic, one graph"},
            "batched_exact": {"ms_per_step": ems, "value": points / (ems / 1e3)},
            "speedup_vs_plain": pms / ms, "max_relative_length_error": worst,
            "surrogate": {"training_s": train_s, "status_per_description": fallback},
            "clocks": clocks, "gpu_launches": (len(params) + 6) * args.steps}
    print(json.dumps(line), flush=True)


def _fx_workload():
    """The Classic FX workload's plan: the cfg5 length and width expressions,
    a NoiseFX pass, a ClumpingFX pass with guide noise, a CutFX pass on a
    share of cLength and a taper."""
    from nanoxgen_b200 import fixtures
    primitive = {"length": fixtures.CLASSIC_LENGTH.replace("*clamp(1-$v,0.2,1)", ""),
                 "width": fixtures.CLASSIC_WIDTH, "taper": "0.6", "taperStart": "0.3"}
    effects = [("noise", dict(mask="1", magnitude="0.03", magnitudeScale="1", frequency="8", correlation="30",
                              preserveLength="40")),
               ("clump", dict(mask="1", clump="0.6", clumpScale="0.1", noise="0.02", noiseScale="1",
                              noiseFrequency="6", noiseCorrelation="40")),
               ("cut", {"amount": "$cLength*0.1"})]
    return primitive, effects


def _fx_clump_guides(w, P, roots, device):
    """ClumpingFX guides of the FX workload: the description's own guides
    resampled linearly to P CVs, their root normals and uvs, tangents normal x
    z (y near the poles), seeded SeExpr prefixes; each strand takes the guide
    whose root is nearest to its root (found on the device)."""
    import numpy as np
    import torch
    gs = w.build_input.guides
    counts = gs.cv_counts.astype(np.int64)
    starts = np.concatenate([[0], np.cumsum(counts)[:-1]])
    u = np.linspace(0.0, 1.0, P)
    axes = np.empty((counts.size, P, 3), np.float32)
    for g in range(counts.size):
        c = gs.cvs[starts[g]:starts[g] + counts[g]].astype(np.float64)
        x = np.linspace(0.0, 1.0, counts[g])
        axes[g] = np.stack([np.interp(u, x, c[:, k]) for k in range(3)], 1)
    n = gs.root_normals.astype(np.float64)
    ref = np.where(np.abs(n[:, 2:3]) < 0.999, [[0.0, 0.0, 1.0]], [[0.0, 1.0, 0.0]])
    t = np.cross(n, ref)
    t /= np.maximum(np.linalg.norm(t, axis=1, keepdims=True), 1e-30)
    guide_roots = torch.from_numpy(axes[:, 0, :]).to(device)
    strand_roots = torch.from_numpy(roots["position"].astype(np.float32)).to(device)
    nearest = torch.cat([torch.cdist(strand_roots[i:i + 65536], guide_roots).argmin(1)
                         for i in range(0, strand_roots.shape[0], 65536)])
    return dict(axes=axes, normals=gs.root_normals.astype(np.float32), tangents=t.astype(np.float32),
                uvs=gs.root_uvs.astype(np.float32),
                prefixes=np.random.default_rng(77).integers(0, 2**32, counts.size, dtype=np.uint32),
                strand_guides=nearest.cpu().numpy().astype(np.uint32))


def run_classic_fx(args):
    """Classic FX passes over a generated frame: the large description's mesh
    (200,000 triangles, 4,096 guides), 1,000,000 strands x 24 CVs generated
    without generator noise, then nxg_classic_fx_apply with the plan of
    _fx_workload (NoiseFX, ClumpingFX toward the description's guides,
    CutFX, taper).  A step is generation plus the FX pass (the pass works in
    place, so each step regenerates its input); the FX kernel is also timed
    alone.  The CPU baseline is the reference's
    apply_xgen_classic_float_runtime_plan_cpu on a prefix sample."""
    import numpy as np
    import torch

    from nanoxgen_b200 import fixtures
    from nanoxgen_b200.asset import build_asset
    from nanoxgen_b200.classic import ClumpGuides, FxPlan, classic_fx_apply
    from nanoxgen_b200.generator import DeviceAsset, allocate_outputs, generate_packed, get_tile
    device = torch.device("cuda", 0)
    torch.cuda.set_device(device)
    S = args.strands
    w = fixtures.large_sphere(strands=S, cvs=24)
    params = w.params.copy(noise_amplitude=0.0)
    P = int(params.cvs_per_strand)
    asset = build_asset(w.build_input, w.stencil_slots)
    d = DeviceAsset(asset, device)
    primitive, effects = _fx_workload()
    plan = FxPlan(primitive, effects, 3, "description")
    plan.upload(device)
    points, roots, uvs, counts = allocate_outputs(S, P, device)
    out = generate_packed(d, params, points=points, roots=roots, root_uvs=uvs, point_counts=counts)
    torch.cuda.synchronize()
    # One surface tangent per strand: the root normal crossed with the z axis
    # (y near the poles), the NoiseFX frame's own fallback direction.
    rn = out.roots_numpy()["normal"].astype(np.float64)
    axis = np.where(np.abs(rn[:, 2:3]) < 0.999, [[0.0, 0.0, 1.0]], [[0.0, 1.0, 0.0]])
    tan = np.cross(rn, axis)
    tan /= np.maximum(np.linalg.norm(tan, axis=1, keepdims=True), 1e-30)
    tangents = torch.from_numpy(tan.astype(np.float32)).to(device)
    cg = _fx_clump_guides(w, P, out.roots_numpy(), device)
    guides = [ClumpGuides(cg["axes"], cg["normals"], cg["tangents"], cg["uvs"], cg["prefixes"], cg["strand_guides"],
                          device=device)]
    status = torch.zeros(2, dtype=torch.int32, device=device)
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=device)
    stream = torch.cuda.current_stream(device)
    diag = asset.bbox_diagonal()

    def step(ev=None):
        generate_packed(d, params, points=points, roots=roots, root_uvs=uvs, point_counts=counts, stream=stream)
        if ev is not None:
            ev.record(stream)
        classic_fx_apply(plan, out, tangents, status=status, stream=stream, clumps=guides)

    for _ in range(args.warmup):
        flush.fill_(1)
        step()
    torch.cuda.synchronize()
    sampler = ClockSampler(0)
    sampler.start()
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True),
           torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
    for k in range(args.steps):
        flush.fill_(k & 0xFF)
        ev[k][0].record(stream)
        step(ev[k][1])
        ev[k][2].record(stream)
    torch.cuda.synchronize()
    clocks = sampler.stop()
    step_ms = statistics.mean(a.elapsed_time(c) for a, b, c in ev)
    fx_ms = statistics.mean(b.elapsed_time(c) for a, b, c in ev)
    st = status.cpu().tolist()
    kept = int((counts.cpu() != 0).sum())
    line = {"metric": "points/sec", "value": S * P / (step_ms / 1e3), "unit": "points/s", "n_gpus": 1,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": step_ms, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {"workload": "classic-fx/displaced-sphere-200k-tris/%d-strands-x%d" % (S, P),
                       "plan": {"primitive": primitive, "effects": [[k, v] for k, v in effects]},
                       "l2": "flushed between timed steps (256 MiB write)"},
            "fx_pass": {"ms": fx_ms, "points_per_s": S * P / (fx_ms / 1e3), "strands_kept": kept,
                        "status": st},
            "clocks": clocks, "gpu_launches": (kernels_per_step(get_tile(P, False)) + 2) * args.steps}
    if not args.no_cpu_baseline:
        from oracle.checker import Reference, reference_available
        if reference_available():
            # The reference's runtime on the same input curves: this library's
            # generated frame (first n strands) before the FX pass.
            n = min(S, 20_000)
            generate_packed(d, params, points=points, roots=roots, root_uvs=uvs, point_counts=counts)
            torch.cuda.synchronize()
            in_pts = points[:n * P].cpu().numpy().copy()
            in_roots = out.roots_numpy()[:n].copy()
            in_uvs = uvs[:n].cpu().numpy().copy()
            in_counts = counts[:n].cpu().numpy().view(np.uint32).copy()
            classic_fx_apply(plan, out, tangents, status=status, clumps=guides)
            torch.cuda.synchronize()
            ref = Reference()
            rplan = ref.classic_plan_fx(primitive, effects, 3, "description")
            freqs = rplan.info()["pref_noise"]
            inputs = (np.stack([ref.classic_noise(in_roots["position"], f) for f in freqs], 1)
                      if len(freqs) else None)
            cores = os.cpu_count() or 1
            sample_guides = [dict(cg, strand_guides=cg["strand_guides"][:n])]
            apply = lambda: ref.classic_apply_fx(rplan, in_pts, in_counts, in_roots, in_uvs, P, 1.0, inputs,
                                                 tan[:n].astype(np.float32), workers=cores, clumps=sample_guides)
            got = apply()
            times = []
            for _ in range(7):
                t0 = time.perf_counter()
                apply()
                times.append(time.perf_counter() - t0)
            med, p90 = statistics.median(times), _percentile(times, 0.9)
            t0 = time.perf_counter()
            ref.classic_apply_fx(rplan, in_pts, in_counts, in_roots, in_uvs, P, 1.0, inputs,
                                 tan[:n].astype(np.float32), workers=1, clumps=sample_guides)
            single = time.perf_counter() - t0
            mine_pts = points[:n * P].cpu().numpy()
            keep = counts[:n].cpu().numpy() != 0
            same = bool(keep.sum() == got[1].size)
            parity = {"strands_checked": n, "same_survivors": same, "tolerance_rel_diag": 1e-5}
            if same:
                sel = np.repeat(keep, P)
                dd = mine_pts[sel, :3].astype(np.float64) - got[0][:, :3]
                parity["max_error_rel_diag"] = float(np.sqrt((dd * dd).sum(-1)).max(initial=0.0)) / diag
                parity["max_radius_error_rel_diag"] = float(
                    np.abs(mine_pts[sel, 3].astype(np.float64) - got[0][:, 3]).max(initial=0.0)) / diag
            line["cpu_baseline"] = {"value": n * P / med, "unit": "points/s", "cores": cores, "kind": "reference",
                                    "cpu_model": cpu_model(), "median_s": med, "p90_s": p90,
                                    "value_p90": n * P / p90,
                                    "single_thread": {"value": n * P / single, "strands": n, "seconds": single},
                                    "sample": "the reference's apply_xgen_classic_float_runtime_plan_cpu on the "
                                              "first %d strands x %d CVs of the generated frame (median of 7 "
                                              "calls after one warm-up)" % (n, P),
                                    "parity": parity}
    print(json.dumps(line), flush=True)


def run_curve_cache(args):
    """Curve-cache (.nxc) ingest on the device: a cache of the large
    description's generated frame (1,000,000 strands x 32 CVs of float4,
    point counts, root uvs as patch uvs, triangles as face ids; 530 MB),
    uploaded once; a step is one nxg_curve_cache_validate_device pass over
    the device copy (every element check of validate_curve_cache, the
    point-count sum and the bit checksum), timed with CUDA events; the blob
    exceeds L2, which is also flushed between steps.  `e2e` adds the upload
    of the blob from pinned host memory and the read-back of the result.
    The CPU baseline is the reference's validate_curve_cache on the same
    blob (serial: its content hash is a dependent chain over 64-bit words),
    with this library's host hash of the same bytes beside it."""
    import ctypes

    import numpy as np
    import torch

    from nanoxgen_b200.asset import build_asset
    from nanoxgen_b200.curve_cache import (DeviceCurveCache, build_curve_cache, content_hash, header,
                                           point_checksum)
    from nanoxgen_b200.generator import DeviceAsset, generate_packed
    device = torch.device("cuda", 0)
    torch.cuda.set_device(device)
    w = workload(args.strands)
    asset = build_asset(w.build_input, w.stencil_slots)
    out = generate_packed(DeviceAsset(asset, device), w.params)
    torch.cuda.synchronize()
    S, P = int(w.params.strand_count), int(w.params.cvs_per_strand)
    roots = out.roots_numpy()
    blob = build_curve_cache(np.full(S, P, np.uint32), out.points.cpu().numpy(),
                             patch_uvs=out.root_uvs.cpu().numpy(), face_ids=roots["triangle_index"])
    del out
    h = header(blob)
    cache = DeviceCurveCache(blob, device)
    pinned = torch.empty(blob.size, dtype=torch.uint8, pin_memory=True)
    pinned.numpy()[:] = blob
    result_host = torch.empty(cache.result.numel(), dtype=torch.uint8, pin_memory=True)
    stream = torch.cuda.current_stream(device)
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=device)
    algorithmic = 4 * S + 16 * h.point_count + 8 * S  # counts, points, patch uvs
    for _ in range(args.warmup):
        flush.fill_(1)
        cache.validate(stream)
    torch.cuda.synchronize()
    sampler = ClockSampler(0)
    sampler.start()
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
    for k in range(args.steps):
        flush.fill_(k & 0xFF)
        ev[k][0].record(stream)
        cache.validate(stream)
        ev[k][1].record(stream)
    torch.cuda.synchronize()
    clocks = sampler.stop()
    ms = statistics.mean(a.elapsed_time(b) for a, b in ev)
    message, point_sum, checksum = cache.outcome()
    host_checksum = point_checksum(blob)
    if message or point_sum != h.point_count or checksum != host_checksum:
        raise SystemExit("device check disagrees with the host: %r %d %d" % (message, point_sum, checksum))
    # e2e: upload + check + result read-back per step
    e2e = []
    for k in range(max(3, args.steps // 2)):
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(stream)
        cache.blob.copy_(pinned, non_blocking=True)
        cache.validate(stream)
        result_host.copy_(cache.result, non_blocking=True)
        b.record(stream)
        b.synchronize()
        e2e.append(a.elapsed_time(b))
    e2e_ms = statistics.median(e2e)
    peak, peak_kind = measured_peak()
    achieved = algorithmic / (ms / 1e3) / 1e9
    line = {"metric": "points/sec", "value": h.point_count / (ms / 1e3), "unit": "points/s", "n_gpus": 1,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "u32/f32", "data": "synthetic",
            "config": {"workload": "curve-cache/displaced-sphere-200k-tris/%d-strands-x%d" % (S, P),
                       "blob_bytes": int(blob.size), "sections": "point counts, points, patch uvs, face ids",
                       "l2": "blob larger than L2; flushed between steps (256 MiB write)",
                       "reference_doc": "the reference's own GPU traversal of 47.4 M cached points: 1.24 ms "
                                        "(docs/xgen-research.md:266-268, other hardware)"},
            "roofline": {"bound": "hbm", "kernel": "check_kernel", "achieved": achieved, "peak": peak,
                         "unit": "GB/s", "frac": achieved / peak, "peak_source": peak_kind,
                         "traffic": None, "algorithmic_bytes": algorithmic},
            "device_check": {"message": message, "point_sum": point_sum, "checksum": "%016x" % checksum},
            "e2e": {"value": h.point_count / (e2e_ms / 1e3), "unit": "points/s",
                    "h2d_bytes_per_step": int(blob.size), "d2h_bytes_per_step": int(cache.result.numel())},
            "clocks": clocks, "gpu_launches": 3 * args.steps}
    if not args.no_cpu_baseline:
        from oracle.checker import Reference, reference_available
        t0 = time.perf_counter()
        ours = content_hash(blob[128:])
        hash_s = time.perf_counter() - t0
        base = {"cores": 1, "cpu_model": cpu_model(), "host_content_hash_s": hash_s,
                "host_content_hash_matches": ours == h.content_hash}
        if reference_available():
            ref = Reference()
            times = []
            for _ in range(3):
                t0 = time.perf_counter()
                msg = ref.curve_cache_validate(blob)
                times.append(time.perf_counter() - t0)
            med = statistics.median(times)
            base.update({"value": h.point_count / med, "unit": "points/s", "kind": "reference",
                         "median_s": med, "message": msg,
                         "sample": "the reference's validate_curve_cache on the whole %d-byte blob "
                                   "(median of 3 calls)" % blob.size})
        line["cpu_baseline"] = base
    print(json.dumps(line), flush=True)


def run_payload(args):
    """Renderer payload batches: the large description's generated frame
    (1,000,000 strands x 32 CVs) as the base curve set (positions, widths =
    2 x radius, root uvs) with one motion sample (the positions moved by
    0.01), cut into 65,536-strand batches through an affine transform -- one
    nxg_build_curve_batches per step over resident inputs, timed with CUDA
    events (inputs and outputs exceed L2; L2 is also flushed between steps).
    The CPU baseline is the reference's build_curve_batches on a 100,000-strand
    prefix of the same set (single-threaded, as the reference is)."""
    import numpy as np
    import torch

    from nanoxgen_b200.asset import build_asset
    from nanoxgen_b200.generator import DeviceAsset, generate_packed
    from nanoxgen_b200.payload import Curves, build_curve_batches
    device = torch.device("cuda", 0)
    torch.cuda.set_device(device)
    w = workload(args.strands)
    out = generate_packed(DeviceAsset(build_asset(w.build_input, w.stencil_slots), device), w.params)
    torch.cuda.synchronize()
    S, P = int(w.params.strand_count), int(w.params.cvs_per_strand)
    xyz = out.points[:, :3].contiguous()
    widths = (2.0 * out.points[:, 3]).contiguous()
    uvs = out.root_uvs.contiguous()
    moved = (xyz + 0.01).contiguous()
    del out
    transform = (0.98, -0.17, 0.0, 0.5, 0.17, 0.98, 0.0, -0.25, 0.0, 0.0, 1.0, 2.0)
    base = Curves(points=xyz, strand_count=S, fixed_cvs_per_strand=P, widths=widths, root_uvs=uvs)
    sample = Curves(points=moved, strand_count=S, fixed_cvs_per_strand=P, constant_width=0.0)
    kw = dict(max_strands_per_batch=65536, transform=transform)
    stream = torch.cuda.current_stream(device)
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=device)
    result = None
    for _ in range(args.warmup):
        flush.fill_(1)
        result = build_curve_batches(base, [(0.5, sample)], **kw)
    torch.cuda.synchronize()
    sampler = ClockSampler(0)
    sampler.start()
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
    for k in range(args.steps):
        flush.fill_(k & 0xFF)
        ev[k][0].record(stream)
        result = build_curve_batches(base, [(0.5, sample)], **kw)
        ev[k][1].record(stream)
    torch.cuda.synchronize()
    clocks = sampler.stop()
    ms = statistics.mean(a.elapsed_time(b) for a, b in ev)
    points = S * P
    # reads: base xyz + widths, sample xyz, root uvs; writes: float4 points,
    # motion xyz, counts, root uvs
    algorithmic = points * (12 + 4 + 12) + S * 8 + points * (16 + 12) + S * (4 + 8)
    peak, peak_kind = measured_peak()
    achieved = algorithmic / (ms / 1e3) / 1e9
    line = {"metric": "points/sec", "value": points / (ms / 1e3), "unit": "points/s", "n_gpus": 1,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {"workload": "payload/displaced-sphere-200k-tris/%d-strands-x%d/1-motion-sample" % (S, P),
                       "batches": int(result.batch_first_point.numel() - 1), "max_strands_per_batch": 65536,
                       "transform": transform, "l2": "inputs and outputs larger than L2; flushed between steps"},
            "roofline": {"bound": "hbm", "kernel": "batches_kernel", "achieved": achieved, "peak": peak,
                         "unit": "GB/s", "frac": achieved / peak, "peak_source": peak_kind, "traffic": None,
                         "algorithmic_bytes": algorithmic},
            "clocks": clocks, "gpu_launches": args.steps}
    if not args.no_cpu_baseline:
        from oracle.checker import Reference, reference_available
        if reference_available():
            n = 100_000
            host = lambda t: t[:n * P].cpu().numpy()
            rbase = dict(points=host(xyz), strands=n, fixed=P, widths=host(widths), root_uvs=uvs[:n].cpu().numpy())
            rsample = dict(points=host(moved), strands=n, fixed=P)
            ref = Reference()
            times = []
            for _ in range(3):
                t0 = time.perf_counter()
                theirs = ref.build_curve_batches(rbase, [(0.5, rsample)], per_batch=65536, transform=transform)
                times.append(time.perf_counter() - t0)
            med = statistics.median(times)
            mine = result.points[:n * P].cpu().numpy()
            same = bool(np.array_equal(mine.view(np.uint32), theirs["points"].view(np.uint32)))
            line["cpu_baseline"] = {"value": n * P / med, "unit": "points/s", "cores": 1, "kind": "reference",
                                    "cpu_model": cpu_model(), "median_s": med,
                                    "sample": "the reference's build_curve_batches on the first %d strands "
                                              "(median of 3 calls, including the test shim's copy of its batches "
                                              "into flat arrays)" % n,
                                    "parity": {"strands_checked": n, "points_bit_identical": same}}
    print(json.dumps(line), flush=True)


def run_asset_build(args):
    """The asset build of the large description's mesh (200,000 triangles,
    4,096 guides): the per-triangle stencil search (stencil.cu) timed alone
    on resident device inputs (`value`, candidates/s), the whole
    nxg_build_asset_device call from host arrays (`e2e`), and the host
    builders beside it (this library's threaded nxg_build_asset, and the
    reference's own single-threaded build_asset when its library is built)."""
    import numpy as np
    import torch

    from nanoxgen_b200.asset import build_asset, build_asset_device
    from nanoxgen_b200.generator import build_stencils
    device = torch.device("cuda", 0)
    torch.cuda.set_device(device)
    src = workload(args.strands).build_input
    host = build_asset(src, 8)
    guides = host.guides()
    dev = lambda a: torch.from_numpy(np.ascontiguousarray(a)).to(device)
    positions = dev(np.asarray(src.positions, np.float32))
    triangles = dev(np.asarray(src.triangles, np.uint32).view(np.int32))
    roots = dev(guides["root_position"].astype(np.float32))
    normals = dev(guides["root_normal"].astype(np.float32))
    out = torch.empty((triangles.shape[0], 8), dtype=torch.int32, device=device)
    tris, count = int(triangles.shape[0]), int(roots.shape[0])
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=device)
    sampler = ClockSampler(0)
    sampler.start()
    times = _graph_time(device, lambda s: build_stencils(positions, triangles, roots, normals, 8, out=out, stream=s),
                        args.steps, args.warmup, flush)
    clocks = sampler.stop()
    same_rows = bool(np.array_equal(out.cpu().numpy().view(np.uint32), host.stencil().reshape(tris, 8)))
    ms = statistics.mean(times)
    build_asset_device(src, 8)  # warm
    e2e = []
    for _ in range(max(3, min(args.steps, 10))):
        t0 = time.perf_counter()
        blob = build_asset_device(src, 8)
        e2e.append((time.perf_counter() - t0) * 1e3)
    same_blob = bool(np.array_equal(blob.buffer, host.buffer))
    t0 = time.perf_counter()
    build_asset(src, 8)
    host_ms = (time.perf_counter() - t0) * 1e3
    port = {"value": host_ms, "unit": "ms per build", "cores": os.cpu_count(),
            "sample": "this library's nxg_build_asset (host threads), one full build"}
    cpu = None
    if not args.no_cpu_baseline:
        sys.path.insert(0, os.path.join(os.path.dirname(os.path.abspath(__file__)), "oracle"))
        import checker
        if checker.reference_available():
            r = checker.Reference()
            runs, ref_blob = [], None
            for _ in range(3):
                t0 = time.perf_counter()
                ref_blob = r.build_asset(src)
                runs.append((time.perf_counter() - t0) * 1e3)
            cpu = {"value": statistics.median(runs), "unit": "ms per build", "cores": 1, "kind": "reference",
                   "cpu_model": cpu_model(), "runs_ms": runs,
                   "sample": "the reference's build_asset (single-threaded), three full builds, median",
                   "same_bytes": bool(np.array_equal(ref_blob, host.buffer))}
    em = statistics.mean(e2e)
    line = {"metric": "stencil candidates/sec", "value": tris * count / (ms / 1e3), "unit": "candidates/s",
            "n_gpus": 1, "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32 (IEEE-rounded, uncontracted)", "data": "synthetic",
            "config": {"workload": "asset-build/displaced-sphere-%dk-tris/%d-guides" % (tris // 1000, count),
                       "triangles": tris, "guides": count, "stencil_slots": 8,
                       "l2": "flushed between timed replays (256 MiB write)"},
            "rows_equal_host_build": same_rows,
            "e2e": {"value": em, "unit": "ms per nxg_build_asset_device call",
                    "h2d_bytes_per_step": int(positions.numel() * 4 + triangles.numel() * 4 + 2 * roots.numel() * 4),
                    "d2h_bytes_per_step": int(out.numel() * 4), "blob_equal_host_build": same_blob},
            "cpu_baseline": cpu, "host_port_build": port, "clocks": clocks, "gpu_launches": args.steps}
    print(json.dumps(line), flush=True)


def main():
    args = parse_args()
    if args.impl == "reference":
        run_reference_arm(args)
    elif args.workload == "classic":
        run_classic(args)
    elif args.workload == "batched_classic":
        run_batched_classic(args)
    elif args.workload == "batched":
        run_batched(args)
    elif args.workload == "motion":
        run_motion(args)
    elif args.workload == "asset_build":
        run_asset_build(args)
    elif args.workload == "classic_fx":
        run_classic_fx(args)
    elif args.workload == "curve_cache":
        run_curve_cache(args)
    elif args.workload == "payload":
        run_payload(args)
    else:
        run_gpu_arm(args)


if __name__ == "__main__":
    main()
