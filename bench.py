#!/usr/bin/env python
"""Benchmark of the periodic Delaunay hot path: full triangulation + one test-and-repair step.

Workload (default "build_repair_4m"): N = 4,194,304 i.i.d. uniform points in a periodic
square of side L = 2048 (unit density), float64 coordinates, cell size 1.0.  One step is
  globalDelaunayTriangulation(P0) -> testAndRepairDelaunayTriangulation(P1)
with P1 = P0 displaced by N(0, 0.02^2) per axis and wrapped (displacement precomputed, as in
an MD code that hands the new positions over).  Predicates: float32 filter -> float64 ->
exact (the "fp64_plain" key repeats the measurement with float64 predicates).
Metric: Mpoints/s = N / step time (each point goes through one build and one repair).

  python bench.py [--gpus N --steps K --warmup W] [--impl reference]

Under torchrun each rank runs an independent replica (no data-path collective: the sets
are independent); value = all ranks' points / max-over-ranks device time.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

import numpy as np  # noqa: E402

from gpudelaunaytriangulation_b200 import workloads as W  # noqa: E402
from gpudelaunaytriangulation_b200.replicas import ReplicaGroup, replica_seed  # noqa: E402

METRIC = "Mpoints/s full build + repair on 1 B200, FP32-filter vs FP64 plain, 0 mismatches"
UNIT = "Mpoints/s"

WORKLOADS = {
    # name: (n, L, sigma, cell size, maxNeighs)
    "build_repair_4m": (4_194_304, 2048.0, 0.02, 1.0, 16),
    "build_repair_1m": (1_000_000, 1000.0, 0.02, 1.0, 16),
}

# Algorithmic (compulsory) DRAM bytes per point of the one-ring kernel k_build: own position
# (16 B) + own index (4 B) + cell start (4 B) + ring written (6 neighbours x 4 B on average,
# exactly 6 on the torus) + ring length (4 B).  Candidate re-reads served on chip are not
# counted.
BUILD_BYTES_PER_POINT = 16 + 4 + 4 + 24 + 4
# DRAM bytes per point that ncu measured for k_build (dram__bytes_read.sum +
# dram__bytes_write.sum of one launch / points) on a 1,048,576-point capture of the same
# kernel (the --profile build case below); traffic scales with the number of points at fixed
# density, so the 4M launch is reported as this figure times its points.
BUILD_DRAM_BYTES_PER_POINT_NCU = 87.3
FALLBACK_HBM_GBS = 6650.0


def measured_peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(path) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return FALLBACK_HBM_GBS, "fallback"


class ClockSampler:
    """nvidia-smi samples during the timed region (SM clock, throttle reasons)."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.gpu = gpu_index
        self.proc = None
        self.lines: list[str] = []
        self.thread = None

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.gpu}", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "200"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except Exception:
            self.proc = None
            return
        self.thread = threading.Thread(target=self._read, daemon=True)
        self.thread.start()

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        if self.thread:
            self.thread.join(timeout=2)
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            parts = [p.strip() for p in ln.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                smax = float(parts[2])
            except ValueError:
                continue
            for nm, v in zip(names, parts[5:9]):
                if v.lower() == "active":
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": smax,
                "reasons": sorted(reasons), "samples": len(sm)}


def dist_setup():
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return world, rank, local


def cpu_model():
    try:
        with open("/proc/cpuinfo") as f:
            for ln in f:
                if ln.startswith("model name"):
                    return ln.split(":", 1)[1].strip()
    except Exception:
        pass
    return "unknown"


class _StdoutToStderr:
    """The reference library prints progress with printf; keep fd 1 for the JSON line."""

    def __enter__(self):
        sys.stdout.flush()
        self.saved = os.dup(1)
        os.dup2(2, 1)
        return self

    def __exit__(self, *exc):
        sys.stdout.flush()
        os.dup2(self.saved, 1)
        os.close(self.saved)
        return False


def reference_cpu_run(n, L, sigma, cell, maxn, steps, warmup, seed, threads=None, budget_s=None):
    with _StdoutToStderr():
        return _reference_cpu_run(n, L, sigma, cell, maxn, steps, warmup, seed, threads, budget_s)


def _reference_cpu_run(n, L, sigma, cell, maxn, steps, warmup, seed, threads=None, budget_s=None):
    """The reference's own host path (oracle/_ref: DelaunayGPU class, GPUcompute=false,
    OpenMP over all host threads), build + test-and-repair per step.  Falls back to the C
    restatement (oracle/liboracle.so) when the reference library is absent."""
    from oracle import oracle as O

    threads = threads or O.default_threads()
    p0 = W.uniform_points(n, L, seed)
    p1 = W.displace(p0, sigma, L, L, seed + 1)
    kind = "reference"
    cls = None
    try:
        if O.ref_lib() is None:
            raise RuntimeError("oracle/_ref not built")
        cls = O.ReferenceClass(n, max(maxn, 24), cell, L, L, threads)
    except Exception:
        kind = "port"
    times = []
    total = warmup + steps
    t_start = time.perf_counter()
    for it in range(total):
        t0 = time.perf_counter()
        if cls is not None:
            cls.global_triangulation(p0, fetch=False)
            cls.test_and_repair(p1, fetch=False)
        else:
            t = O.restated_global(p0, L, L, cell, 32, threads)
            O.restated_test_and_repair(p1, L, L, t, cell, threads)
        dt = time.perf_counter() - t0
        if it >= warmup:
            times.append(dt)
        if budget_s is not None and time.perf_counter() - t_start > budget_s and len(times) >= 1:
            break
    if cls is not None:
        cls.close()
    return {"seconds": times, "kind": kind, "threads": threads}


def reference_gpu_run(n, L, sigma, cell, p0, p1, steps, warmup, ours=None):
    """The reference's own CUDA kernels (its DelaunayGPU class with GPUcompute=true and safety
    mode, compiled for sm_100a into oracle/_ref) on the same workload: per step a global
    triangulation of p0 and a test-and-repair with p1, each timed with CUDA events on the
    legacy default stream it launches on.  maxNeighs 24: its seed pass has no row-capacity
    check, and its largest seed polygon on this workload (measured on the host first, below)
    must stay well inside the rows.  ours: (tri, nn) of this library for p0 and for p1, to
    count the rings that differ."""
    from oracle import oracle as O

    with _StdoutToStderr():
        seed_max = max(O.reference_seed_max(p0, L, L, cell, 64), O.reference_seed_max(p1, L, L, cell, 64))
        if not (0 < seed_max <= 12):
            return {"unavailable": f"seed polygons of {seed_max} entries: too close to the 24-entry rows"}
        R = O.ReferenceGPU(p0, p1, L, L, 24, cell)
        diff = {}
        for it in range(warmup):
            R.build()
            if not R.triangles_ok():
                R.close()
                return {"unavailable": "its build is not a 2N-triangle torus triangulation; repair not run"}
            if it == 0 and ours is not None:
                diff["build"] = _rings_differing(R.fetch(32), *ours[0])
            R.repair()
            if it == 0 and ours is not None:
                diff["repair"] = _rings_differing(R.fetch(32), *ours[1])
        b_ms, r_ms = [], []
        for _ in range(steps):
            b_ms.append(R.build())
            r_ms.append(R.repair())   # refuses (raises) unless the build has exactly 2N triangles
        R.close()
    step = float(np.mean(b_ms) + np.mean(r_ms))
    return {"value": n / step / 1e3, "unit": UNIT, "ms_per_step": step, "build_ms": float(np.mean(b_ms)),
            "repair_ms": float(np.mean(r_ms)), "steps": steps, "max_neighs": 24, "seed_polygon_max": seed_max,
            "rings_differing_from_ours": diff,
            "path": "reference DelaunayGPU class, GPUcompute=true, safety mode, its CUDA kernels for sm_100a"}


def _rings_differing(ref, tri, nn):
    from oracle import oracle as O

    if not np.array_equal(ref.nn, nn):
        return int((ref.nn != nn).sum())
    w = min(ref.tri.shape[1], tri.shape[1])
    return int((O.canonical(ref.tri, ref.nn)[:, :w] != O.canonical(tri, nn)[:, :w]).any(axis=1).sum())


def run_reference(args):
    world, rank, local = dist_setup()
    if rank != 0:
        return 0
    n, L, sigma, cell, maxn = WORKLOADS[args.workload]
    if args.n:
        n, L = args.n, float(np.sqrt(args.n))
    r = reference_cpu_run(n, L, sigma, cell, maxn, args.steps, args.warmup, seed=2026)
    secs = r["seconds"]
    mean = sum(secs) / len(secs)
    value = n / mean / 1e6
    out = {
        "impl": "reference",
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus, "steps": len(secs),
        "warmup": args.warmup, "ms_per_step": mean * 1e3, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded uniform periodic points)",
        "config": {"workload": args.workload, "n_points": n, "box": L, "sigma": sigma, "cell_size": cell,
                   "path": "reference DelaunayGPU host path (GPUcompute=false, OpenMP)"},
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": r["threads"], "kind": r["kind"],
                         "sample": f"full workload: build + one repair of {n} points per step",
                         "cpu": cpu_model()},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(out))
    return 0


# compulsory bytes per point of one repair step (bin 16+8, ring + lengths 28, positions 16,
# cell-order index 4, CSR 8 at one cell per point) plus 48 B per rebuilt point
REPAIR_BYTES_PER_POINT = 80
REPAIR_BYTES_PER_REBUILT = 48


def ensemble_md_measure(dev, num_sets=256, lo=1000, hi=65536, sigma=0.01, steps=100, graph_steps=10, rounds=4,
                        seed=7):
    """Batched ensemble: num_sets independent periodic sets (sizes log-uniform in [lo, hi],
    unit density) triangulated by one launch sequence, then `steps` MD steps (device
    displacement sigma + test-and-repair with `rounds` rounds) replayed from a CUDA graph of
    `graph_steps` steps."""
    import torch

    from gpudelaunaytriangulation_b200.delaunay import DelaunayBatch

    pts, sizes, boxes = W.ensemble(num_sets, lo, hi, seed=seed)
    n = len(pts)
    b = DelaunayBatch(sizes, boxes, 16, 1.0)
    b.setTiming(True)
    P = torch.from_numpy(pts).to(dev)
    P0 = P.clone()
    tri = torch.zeros(16 * n, dtype=torch.int32, device=dev)
    nn = torch.zeros(n, dtype=torch.int32, device=dev)
    tune = b.autotune(P, tri, nn)   # cell size (relative to each set's spacing) and kernel shape
    for _ in range(3):
        P.copy_(P0)
        b.globalDelaunayTriangulation(P, tri, nn)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    b.globalDelaunayTriangulation(P, tri, nn)
    e1.record()
    torch.cuda.synchronize()
    build_ms = e0.elapsed_time(e1)
    stream = torch.cuda.Stream(device=dev)
    stream.wait_stream(torch.cuda.current_stream())
    with torch.cuda.stream(stream):
        g = b.mdGraph(P, tri, nn, sigma, seed=seed + 1, steps=graph_steps, rounds=rounds, stream=stream)
        g.launch(stream)   # warm-up replay
        b.clearFlags(stream)
        stream.synchronize()
        f0, f1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        f0.record(stream)
        for _ in range(steps // graph_steps):
            g.launch(stream)
        f1.record(stream)
        stream.synchronize()
    md_ms = f0.elapsed_time(f1) / ((steps // graph_steps) * graph_steps)
    st = b.stats()
    g.close()
    # one more MD step outside the graph for the repaired fraction
    with torch.cuda.stream(stream):
        b.mdStep(P, tri, nn, sigma, seed=seed + 2, rounds=rounds, stream=stream)
        stream.synchronize()
    rep = b.stats()
    f = rep["repaired"] / n
    peak, kind = measured_peaks()
    step_bytes = n * (REPAIR_BYTES_PER_POINT + REPAIR_BYTES_PER_REBUILT * f)
    achieved = step_bytes / (md_ms / 1e3) / 1e9
    b.close()
    return {"sets": num_sets, "points": n, "steps": (steps // graph_steps) * graph_steps, "sigma": sigma,
            "graph_steps": graph_steps, "rounds": rounds,
            "build_ms": build_ms, "build_mpts": n / (build_ms / 1e3) / 1e6,
            "md_ms_per_step": md_ms, "md_mpts": n / (md_ms / 1e3) / 1e6,
            "repaired_fraction": f, "sticky_flags": st["sticky_flags"], "tuning": tune,
            "repair_roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                                "frac": achieved / peak, "bytes_per_point": REPAIR_BYTES_PER_POINT
                                + REPAIR_BYTES_PER_REBUILT * f, "peak_source": f"{kind} hbm_gbs"}}


def _timed_call(fn, stream=None):
    import torch

    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    fn()
    e1.record(stream)
    torch.cuda.synchronize()
    return e0.elapsed_time(e1)


def configs_measure(dev):
    """The other workload families, each measured once (not the headline): 1M points with 20
    float64 repair steps; 1M-site jittered triangular lattice and 1M-point 64-cluster Gaussian
    mixture (float32 filter, autotuned settings, check mode for mismatches); 1M points in a
    general (60-degree) periodic box."""
    import torch

    from gpudelaunaytriangulation_b200.delaunay import DelaunayGPU

    out = {}
    # 1,000,000 uniform points, L = 1000: build, then 20 steps of displacement + repair, float64
    n, L = 1_000_000, 1000.0
    P = torch.from_numpy(W.uniform_points(n, L, 31)).to(dev)
    d = DelaunayGPU(n, 16, 1.0, (L, L))
    d.setPrecision(False)
    tri = torch.zeros(16 * n, dtype=torch.int32, device=dev)
    nn = torch.zeros(n, dtype=torch.int32, device=dev)
    d.globalDelaunayTriangulation(P, tri, nn)
    b_ms = _timed_call(lambda: d.globalDelaunayTriangulation(P, tri, nn))
    rep = []

    def steps():
        for k in range(20):
            d.displace(P, 0.02, seed=32, step=k)
            d.testAndRepairDelaunayTriangulation(P, tri, nn)
            rep.append(d.stats()["repaired"])

    s_ms = _timed_call(steps) / 20
    out["uniform_1m_fp64_20_steps"] = {"points": n, "build_ms": b_ms, "repair_step_ms": s_ms,
                                       "build_mpts": n / b_ms / 1e3, "repair_step_mpts": n / s_ms / 1e3,
                                       "repaired_per_step": float(np.mean(rep)),
                                       "sum_ring_sizes_is_6n": int(nn.sum().item()) == 6 * n}
    d.close()
    # near-degenerate lattice and clustered mixture, float32 filter, autotuned
    lat, Lx, Ly = W.triangular_lattice(1024, 1024, 1.0, 1e-4, seed=3)
    mix, Lm = W.gaussian_mixture(1 << 20, components=64, sigma=2.0, L=1024.0, seed=5)
    for name, pts, bx, by in (("lattice_1m_fp32", lat, Lx, Ly), ("mixture_1m_fp32", mix, Lm, Lm)):
        n = len(pts)
        P = torch.from_numpy(pts).to(dev)
        d = DelaunayGPU(n, 16, 0.0, (bx, by))
        tri = torch.zeros(16 * n, dtype=torch.int32, device=dev)
        nn = torch.zeros(n, dtype=torch.int32, device=dev)
        tune = d.autotune(P, tri, nn)
        # one untimed call at the chosen settings, then the median of five (the deferred
        # phase of the mixture varies with where its slowest point is scheduled)
        d.globalDelaunayTriangulation(P, tri, nn)
        b_ms = float(np.median([_timed_call(lambda: d.globalDelaunayTriangulation(P, tri, nn)) for _ in range(5)]))
        d.setCheckMode(True)
        d.globalDelaunayTriangulation(P, tri, nn)
        st = d.stats()
        out[name] = {"points": n, "build_ms": b_ms, "build_mpts": n / b_ms / 1e3, "tuning": tune,
                     "fp32_undecided_frac": st["fp32_undecided"] / max(1, st["tests"]),
                     "fp64_undecided": st["fp64_undecided"], "exact_points": st["exact_points"],
                     "mismatches": st["mismatches"], "flags": st["error_flags"], "max_ring": st["max_ring"],
                     "sum_ring_sizes_is_6n": int(nn[: n].sum().item()) == 6 * n}
        d.close()
    # general periodic box: 1,048,576 uniform points in a 60-degree box at unit density, float32
    # filter; build, one repair after a sigma = 0.02 displacement, device validation
    n = 1 << 20
    s = float(np.sqrt(n / (np.sqrt(3.0) / 2.0)))
    box = (s, 0.5 * s, 0.0, s * np.sqrt(3.0) / 2.0)
    M = np.array([[box[0], box[1]], [box[2], box[3]]])
    hp = np.ascontiguousarray(np.random.default_rng(61).uniform(0.0, 1.0, (n, 2)) @ M.T)
    P = torch.from_numpy(hp).to(dev)
    d = DelaunayGPU(n, 16, 1.0, box)
    tri = torch.zeros(16 * n, dtype=torch.int32, device=dev)
    nn = torch.zeros(n, dtype=torch.int32, device=dev)
    d.globalDelaunayTriangulation(P, tri, nn)
    b_ms = _timed_call(lambda: d.globalDelaunayTriangulation(P, tri, nn))
    # repair steps: sigma = 0.02 per axis, left unwrapped (any position is valid in a general
    # box); one warm-up step, then 5 timed ones (displacements drawn outside the timed calls)
    gen = torch.Generator(device=dev).manual_seed(62)
    r_ms, rep = [], []
    for k in range(6):
        P.add_(torch.randn(P.shape, generator=gen, device=dev, dtype=torch.float64), alpha=0.02)
        ms = _timed_call(lambda: d.testAndRepairDelaunayTriangulation(P, tri, nn))
        if k > 0:
            r_ms.append(ms)
            rep.append(d.stats()["repaired"])
    st = d.stats()
    v = d.validate(P, tri, nn)
    rm = float(np.mean(r_ms))
    out["hex_box_1m_fp32"] = {"points": n, "box": [float(x) for x in d.kernelBox()], "build_ms": b_ms,
                              "build_mpts": n / b_ms / 1e3, "repair_step_ms": rm, "repair_step_mpts": n / rm / 1e3,
                              "repaired_per_step": float(np.mean(rep)), "flags": st["error_flags"],
                              "valid": v["valid"]}
    d.close()
    return out


def run_ours(args):
    import torch
    import torch.distributed as dist

    from gpudelaunaytriangulation_b200.delaunay import DelaunayGPU

    world, rank, local = dist_setup()
    torch.cuda.set_device(local)
    if world > 1:
        dist.init_process_group("nccl", timeout=__import__("datetime").timedelta(seconds=600),
                                device_id=torch.device("cuda", local))
    dev = torch.device("cuda", local)
    n, L, sigma, cell, maxn = WORKLOADS[args.workload]
    if args.n:
        n, L = args.n, float(np.sqrt(args.n))
    group = ReplicaGroup(world, rank, dev)
    seed = replica_seed(2026, rank)
    p0 = W.uniform_points(n, L, seed)
    p1 = W.displace(p0, sigma, L, L, seed + 1)
    P0 = torch.from_numpy(p0).to(dev)
    P1 = torch.from_numpy(p1).to(dev)
    tri = torch.zeros(maxn * n, dtype=torch.int32, device=dev)
    nn = torch.zeros(n, dtype=torch.int32, device=dev)
    d = DelaunayGPU(n, maxn, cell, (L, L))
    d.setTiming(True)
    stream = torch.cuda.current_stream()

    barrier = group.barrier
    max_over_ranks = group.max_over_ranks

    def timed(precision_fp32: bool, steps: int, warmup: int, sample_clocks=False):
        d.setPrecision(precision_fp32)
        for _ in range(warmup):
            d.globalDelaunayTriangulation(P0, tri, nn)
            d.testAndRepairDelaunayTriangulation(P1, tri, nn)
        build_ms, launches, repaired, rounds = [], 0, 0, []
        clocks = ClockSampler(local) if sample_clocks else None
        barrier()
        torch.cuda.synchronize()
        if clocks:
            clocks.start()
            time.sleep(0.3)
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(steps):
            d.globalDelaunayTriangulation(P0, tri, nn)
            build_ms.append(d.phaseTimes()["build"])
            launches += d.stats()["launches"]
            d.testAndRepairDelaunayTriangulation(P1, tri, nn)
            st = d.stats()
            launches += st["launches"]
            repaired += st["repaired"]
            rounds.append(st["repair_rounds"])
        e1.record(stream)
        torch.cuda.synchronize()
        barrier()
        ck = clocks.stop() if clocks else None
        ms = e0.elapsed_time(e1) / steps
        return max_over_ranks(ms), build_ms, launches, repaired / steps, rounds, ck

    # headline: float32 filter
    ms, build_ms, launches, repaired, rounds, clocks = timed(True, args.steps, args.warmup, sample_clocks=True)
    value, _ = group.throughput(n, ms)
    # phase split of one extra step (outside the timed region)
    d.globalDelaunayTriangulation(P0, tri, nn)
    ph_build = d.phaseTimes()
    d.testAndRepairDelaunayTriangulation(P1, tri, nn)
    ph_rep = d.phaseTimes()
    st_rep = d.stats()
    # float64-plain variant, same workload
    ms64, build_ms64, _, _, _, _ = timed(False, max(2, args.steps // 2), 1)
    value64 = world * n / (ms64 / 1e3) / 1e6
    # check mode (outside timing): every float32 decision re-evaluated in float64
    d.setPrecision(True)
    d.setCheckMode(True)
    d.globalDelaunayTriangulation(P0, tri, nn)
    chk_b = d.stats()
    d.testAndRepairDelaunayTriangulation(P1, tri, nn)
    chk_r = d.stats()
    d.setCheckMode(False)

    # End to end through the public API with host buffers (pinned), every copy inside the
    # timed region, pipelined the way a caller would: each step's inputs (initial and
    # displaced positions) upload on one copy stream, its result (the repaired rings and
    # ring lengths) downloads on another, the calls run on the compute stream; ring buffers
    # alternate between steps, so a step's result downloads while the next step computes.
    e2e = None
    if not args.no_e2e:
        h0 = torch.from_numpy(p0).pin_memory()
        h1 = torch.from_numpy(p1).pin_memory()
        htri_r = torch.empty(tri.numel(), dtype=torch.int32).pin_memory()
        hnn_r = torch.empty(n, dtype=torch.int32).pin_memory()
        cin = torch.cuda.Stream(device=dev)
        cout = torch.cuda.Stream(device=dev)
        Pa = [torch.empty_like(P0) for _ in range(2)]
        Pb = [torch.empty_like(P0) for _ in range(2)]
        tb = [torch.empty_like(tri) for _ in range(2)]
        nb = [torch.empty_like(nn) for _ in range(2)]
        used = [None, None]   # compute finished with the step's positions
        out = [None, None]    # downloads of the step's results finished
        ready = [None, None]  # the step's positions uploaded
        e_steps = max(40, args.steps)   # pipeline fill + drain (one upload, one download) amortised

        def upload(k):
            # issued one step ahead, so it overlaps the previous step's calls
            b = k % 2
            with torch.cuda.stream(cin):
                if used[b] is not None:
                    cin.wait_event(used[b])
                Pa[b].copy_(h0, non_blocking=True)
                Pb[b].copy_(h1, non_blocking=True)
                up = torch.cuda.Event()
                up.record(cin)
                ready[b] = up

        def compute(k):
            b = k % 2
            stream.wait_event(ready[b])
            if out[b] is not None:
                stream.wait_event(out[b])
            d.globalDelaunayTriangulation(Pa[b], tb[b], nb[b])
            d.testAndRepairDelaunayTriangulation(Pb[b], tb[b], nb[b])
            er = torch.cuda.Event()
            er.record(stream)
            used[b] = er
            with torch.cuda.stream(cout):
                cout.wait_event(er)
                htri_r.copy_(tb[b], non_blocking=True)
                hnn_r.copy_(nb[b], non_blocking=True)
                ev = torch.cuda.Event()
                ev.record(cout)
                out[b] = ev

        def run(steps):
            upload(0)
            for k in range(steps):
                if k + 1 < steps:
                    upload(k + 1)
                compute(k)

        run(2)
        torch.cuda.synchronize()
        barrier()
        f0 = torch.cuda.Event(enable_timing=True)
        f1 = torch.cuda.Event(enable_timing=True)
        f0.record(stream)
        run(e_steps)
        stream.wait_stream(cout)
        stream.wait_stream(cin)
        f1.record(stream)
        torch.cuda.synchronize()
        barrier()
        ems = max_over_ranks(f0.elapsed_time(f1) / e_steps)
        # the last step's results are the host's: they must equal the device-timed run's
        valid = torch.arange(maxn)[None, :] < hnn_r[:, None]
        assert torch.equal(hnn_r, nn.cpu()) and torch.equal(htri_r.view(n, maxn)[valid], tri.cpu().view(n, maxn)[valid]), \
            "e2e result differs"
        e2e = {"value": world * n / (ems / 1e3) / 1e6, "unit": UNIT,
               "h2d_bytes_per_step": 2 * P0.numel() * 8,
               "d2h_bytes_per_step": (tri.numel() + nn.numel()) * 4, "ms_per_step": ems,
               "inputs": "initial + displaced positions uploaded every step",
               "result": "repaired rings + ring lengths downloaded every step",
               "pipelining": "uploads / downloads on two copy streams overlapping the calls; rings double-buffered",
               "steps": e_steps}

    ens = None
    if not args.no_ensemble:
        ens = ensemble_md_measure(dev)
    other = None
    if not args.no_configs and world == 1:
        other = configs_measure(dev)

    peak, peak_kind = measured_peaks()
    avg_build_s = (sum(build_ms) / len(build_ms)) / 1e3
    bytes_launch = n * BUILD_BYTES_PER_POINT
    achieved = bytes_launch / avg_build_s / 1e9
    traffic = None if BUILD_DRAM_BYTES_PER_POINT_NCU is None else BUILD_DRAM_BYTES_PER_POINT_NCU * n

    ref_gpu = None
    if rank == 0 and world == 1 and not args.no_reference_gpu:
        # this library's rings for both inputs, for the comparison (outside every timing)
        d.setPrecision(True)
        d.globalDelaunayTriangulation(P0, tri, nn)
        ours0 = (tri.view(n, -1).cpu().numpy(), nn.cpu().numpy())
        d.testAndRepairDelaunayTriangulation(P1, tri, nn)
        ours1 = (tri.view(n, -1).cpu().numpy(), nn.cpu().numpy())
        try:
            ref_gpu = reference_gpu_run(n, L, sigma, cell, p0, p1, steps=3, warmup=1, ours=(ours0, ours1))
        except Exception as e:   # reported, never fatal for this arm
            ref_gpu = {"unavailable": f"{type(e).__name__}: {e}"}

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        r = reference_cpu_run(n, L, sigma, cell, maxn, steps=1, warmup=0, seed=seed, budget_s=30)
        cpu = {"value": n / (sum(r["seconds"]) / len(r["seconds"])) / 1e6, "unit": UNIT, "cores": r["threads"],
               "kind": r["kind"], "cpu": cpu_model(),
               "sample": f"one full step (build + one repair of {n} points) of the same workload"}

    out = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded uniform periodic points)",
        "config": {"workload": args.workload, "n_points": n, "box": L, "sigma": sigma, "cell_size": cell,
                   "max_neighs": maxn, "precision": "fp32 filter -> fp64 -> exact",
                   "l2": "working set (positions 64 MB x2 + rings 268 MB) larger than the 126 MB L2",
                   "parallelism": f"{world} independent replica(s)"},
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                     "traffic": traffic, "kernel": "k_build<float,14,64> (one-ring construction)",
                     "bytes_per_point": BUILD_BYTES_PER_POINT, "avg_launch_ms": avg_build_s * 1e3,
                     "peak_source": f"{peak_kind} hbm_gbs"},
        "cpu_baseline": cpu,
        "reference_gpu": ref_gpu,
        "e2e": e2e,
        "gpu_launches": launches,
        "clocks": clocks,
        "fp64_plain": {"value": value64, "unit": UNIT, "ms_per_step": ms64,
                       "build_kernel_ms": sum(build_ms64) / len(build_ms64)},
        "phases_ms": {"build_call": ph_build, "repair_call": ph_rep},
        "repair": {"repaired_per_step": repaired, "rounds": rounds, "flagged": st_rep["flagged"]},
        "fallback": {"fp32_undecided_frac": chk_b["fp32_undecided"] / max(1, chk_b["tests"]),
                     "fp64_undecided": chk_b["fp64_undecided"] + chk_r["fp64_undecided"],
                     "exact_points": chk_b["exact_points"] + chk_r["exact_points"],
                     "tests": chk_b["tests"] + chk_r["tests"]},
        "mismatches": chk_b["mismatches"] + chk_r["mismatches"],
        "ensemble_md": ens,
        "configs": other,
    }
    if rank == 0:
        print(json.dumps(out))
    d.close()
    if world > 1:
        dist.destroy_process_group()
    return 0


def run_profile_case(args):
    """A fixed, small sequence of library calls for Nsight Compute captures.  `--reps` global
    triangulations of n seeded uniform points at unit density (build, repair), or in a
    general 60-degree box at unit density (hex); with `repair`, one test-and-repair after a
    sigma = 0.02 displacement.  Launch order per triangulation: 6 binning kernels, k_build,
    k_build_warp.  `md`: the 256-set ensemble, one build, then `--reps` MD steps.  `mixture`:
    the 1M-point 64-cluster mixture at its tuned settings.  Prints the counters of the calls."""
    import math

    import torch

    from gpudelaunaytriangulation_b200.delaunay import DelaunayBatch, DelaunayGPU

    if args.profile == "md":
        # the batched ensemble of the ensemble_md measurement: 256 sets, one build, then
        # `--reps` MD steps (sigma 0.01, 4 rebuild rounds) launched directly, not from a graph
        pts, sizes, boxes = W.ensemble(256, 1000, 65536, seed=7)
        n = len(pts)
        b = DelaunayBatch(sizes, boxes, 16, 1.0)
        P = torch.from_numpy(pts).cuda()
        tri = torch.zeros(16 * n, dtype=torch.int32, device="cuda")
        nn = torch.zeros(n, dtype=torch.int32, device="cuda")
        b.globalDelaunayTriangulation(P, tri, nn)
        stream = torch.cuda.Stream()
        stream.wait_stream(torch.cuda.current_stream())
        with torch.cuda.stream(stream):
            for _ in range(args.reps):
                b.mdStep(P, tri, nn, 0.01, seed=8, rounds=4, stream=stream)
            stream.synchronize()
        print(json.dumps({"md": b.stats()}))
        return 0
    if args.profile == "mixture":
        # the clustered workload of the mixture_1m_fp32 measurement (1,048,576 points, 64
        # Gaussian clusters of std 2 in a 1024 box) at the settings the autotuner picks for it
        # (cell edge 0.25 of the mean spacing, work budget 512, 14-entry ring at 32 threads per
        # block), `--reps` global triangulations
        pts, L = W.gaussian_mixture(1 << 20, components=64, sigma=2.0, L=1024.0, seed=5)
        n = len(pts)
        d = DelaunayGPU(n, 24, 0.25 * L / math.sqrt(n), (L, L))
        d.setKernelShape(3)
        d.setWorkBudget(512)
        d.setTiming(True)
        P = torch.from_numpy(pts).cuda()
        tri = torch.zeros(24 * n, dtype=torch.int32, device="cuda")
        nn = torch.zeros(n, dtype=torch.int32, device="cuda")
        for _ in range(args.reps):
            tri, nn = d.globalDelaunayTriangulation(P, tri, nn)
        print(json.dumps({"mixture": d.stats(), "build_ms": d.phaseTimes()}))
        return 0
    n = args.n or (1 << 20)
    L = math.sqrt(n)
    if args.profile == "hex":
        s = math.sqrt(n / (math.sqrt(3.0) / 2.0))
        box = (s, 0.5 * s, 0.0, s * math.sqrt(3.0) / 2.0)
        M = np.array([[box[0], box[1]], [box[2], box[3]]])
        pts = np.ascontiguousarray(np.random.default_rng(7).uniform(0.0, 1.0, (n, 2)) @ M.T)
    else:
        box = (L, L)
        pts = W.uniform_points(n, L, seed=7)
    P = torch.from_numpy(pts).cuda()
    d = DelaunayGPU(n, 16, 1.0, box)
    d.setTiming(True)
    tri = torch.zeros(16 * n, dtype=torch.int32, device="cuda")
    nn = torch.zeros(n, dtype=torch.int32, device="cuda")
    for _ in range(args.reps):
        d.globalDelaunayTriangulation(P, tri, nn)
    out = {"build": d.stats(), "build_ms": d.phaseTimes()}
    if args.profile == "repair":
        P1 = torch.from_numpy(W.displace(pts, 0.02, L, L, seed=8)).cuda()
        d.testAndRepairDelaunayTriangulation(P1, tri, nn)
        out["repair"] = d.stats()
        out["repair_ms"] = d.phaseTimes()
    torch.cuda.synchronize()
    print(json.dumps(out))
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--workload", choices=sorted(WORKLOADS), default="build_repair_4m")
    ap.add_argument("--n", type=int, default=0, help="override the point count (box side sqrt(n))")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-ensemble", action="store_true", help="skip the batched-ensemble MD measurement")
    ap.add_argument("--no-configs", action="store_true", help="skip the other workload families")
    ap.add_argument("--no-reference-gpu", action="store_true", help="skip timing the reference's own CUDA kernels")
    ap.add_argument("--profile", choices=["build", "repair", "hex", "md", "mixture"], default=None,
                    help="profiling case for Nsight Compute: a fixed, small sequence of calls (no timing)")
    ap.add_argument("--reps", type=int, default=2, help="global triangulations per --profile run")
    args = ap.parse_args()
    if args.profile:
        return run_profile_case(args)
    if args.warmup < 3 and args.impl == "ours":
        args.warmup = 3
    if args.impl == "reference":
        return run_reference(args)
    return run_ours(args)


if __name__ == "__main__":
    sys.exit(main())
