"""Profiling driver: a fixed, small sequence of library calls for Nsight Compute captures.

    python -m gpudelaunaytriangulation_b200.profile --n 1048576 [--fp64] [--repair]

Runs `--reps` global triangulations of n seeded uniform points at unit density (and, with
--repair, one test-and-repair after a sigma=0.02 displacement), then prints the counters of
the last call.  Launch order per rep: 6 binning kernels, k_build, k_build_warp.
"""
import argparse
import json
import math

import torch

from . import workloads as W
from .delaunay import DelaunayGPU


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--n", type=int, default=1 << 20)
    ap.add_argument("--reps", type=int, default=2)
    ap.add_argument("--cell", type=float, default=1.0)
    ap.add_argument("--fp64", action="store_true")
    ap.add_argument("--repair", action="store_true")
    a = ap.parse_args()
    L = math.sqrt(a.n)
    pts = W.uniform_points(a.n, L, seed=7)
    P = torch.from_numpy(pts).cuda()
    d = DelaunayGPU(a.n, 16, a.cell, (L, L))
    d.setPrecision(not a.fp64)
    d.setTiming(True)
    tri = torch.zeros(16 * a.n, dtype=torch.int32, device="cuda")
    nn = torch.zeros(a.n, dtype=torch.int32, device="cuda")
    for _ in range(a.reps):
        d.globalDelaunayTriangulation(P, tri, nn)
    out = {"build": d.stats(), "build_ms": d.phaseTimes()}
    if a.repair:
        P1 = torch.from_numpy(W.displace(pts, 0.02, L, L, seed=8)).cuda()
        d.testAndRepairDelaunayTriangulation(P1, tri, nn)
        out["repair"] = d.stats()
        out["repair_ms"] = d.phaseTimes()
    torch.cuda.synchronize()
    print(json.dumps(out))


if __name__ == "__main__":
    main()
