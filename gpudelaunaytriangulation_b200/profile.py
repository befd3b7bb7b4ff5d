"""Profiling driver: a fixed, small sequence of library calls for Nsight Compute captures.

    python -m gpudelaunaytriangulation_b200.profile --n 1048576 [--fp64] [--repair] [--hex]

Runs `--reps` global triangulations of n seeded uniform points at unit density (and, with
--repair, one test-and-repair after a sigma=0.02 displacement), then prints the counters of
the last call.  Launch order per rep: 6 binning kernels, k_build, k_build_warp.
"""
import argparse
import json
import math

import numpy as np
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
    ap.add_argument("--hex", action="store_true", help="a general 60-degree periodic box at unit density")
    a = ap.parse_args()
    L = math.sqrt(a.n)
    if a.hex:
        s = math.sqrt(a.n / (math.sqrt(3.0) / 2.0))
        box = (s, 0.5 * s, 0.0, s * math.sqrt(3.0) / 2.0)
        M = np.array([[box[0], box[1]], [box[2], box[3]]])
        pts = np.ascontiguousarray(np.random.default_rng(7).uniform(0.0, 1.0, (a.n, 2)) @ M.T)
    else:
        box = (L, L)
        pts = W.uniform_points(a.n, L, seed=7)
    P = torch.from_numpy(pts).cuda()
    d = DelaunayGPU(a.n, 16, a.cell, box)
    d.setPrecision(not a.fp64)
    d.setTiming(True)
    tri = torch.zeros(16 * a.n, dtype=torch.int32, device="cuda")
    nn = torch.zeros(a.n, dtype=torch.int32, device="cuda")
    for _ in range(a.reps):
        d.globalDelaunayTriangulation(P, tri, nn)
    out = {"build": d.stats(), "build_ms": d.phaseTimes()}
    if a.repair:
        if a.hex:
            moved = pts + np.random.default_rng(8).normal(0.0, 0.02, pts.shape)
        else:
            moved = W.displace(pts, 0.02, L, L, seed=8)
        P1 = torch.from_numpy(moved).cuda()
        d.testAndRepairDelaunayTriangulation(P1, tri, nn)
        out["repair"] = d.stats()
        out["repair_ms"] = d.phaseTimes()
    torch.cuda.synchronize()
    print(json.dumps(out))


if __name__ == "__main__":
    main()
