"""Generates tests/golden/*.npz from the reference's own CPU path (oracle/_ref, built from
the reference sources by oracle/build_ref.sh).  Run in a container where the reference is
present:  python tests/golden/make_golden.py

Each fixture holds the seeded points, the box, the cell size and the reference's rings in
canonical rotation (smallest index first), flattened with their lengths.  Repair fixtures
also hold the displaced points and the reference's rings after testAndRepair.
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from gpudelaunaytriangulation_b200 import workloads as W  # noqa: E402
from oracle import oracle as O  # noqa: E402


def flat(tri, nn):
    c = O.canonical(tri, nn)
    return np.concatenate([c[i, : nn[i]] for i in range(len(nn))]).astype(np.int32)


def main():
    cases = [("uniform_n200_s1", 200, 1), ("uniform_n2000_s2", 2000, 2), ("uniform_n10000_s3", 10000, 3)]
    for name, n, seed in cases:
        L = float(np.sqrt(n))
        pts = W.uniform_points(n, L, seed)
        ref = O.reference_global(pts, L, L, 1.0, 32)
        out = dict(points=pts, L=np.array([L, L]), cell_size=np.array(1.0), nn=ref.nn.astype(np.int32),
                   rings=flat(ref.tri, ref.nn))
        if n <= 2000:
            moved = W.displace(pts, 0.02, L, L, seed + 1000)
            rep, flags = O.reference_test_and_repair(moved, L, L, ref, 1.0)
            out.update(moved=moved, repair_nn=rep.nn.astype(np.int32), repair_rings=flat(rep.tri, rep.nn),
                       repair_flags=flags.astype(np.int32))
        np.savez_compressed(os.path.join(HERE, name + ".npz"), **out)
        print(name, "max ring", int(ref.nn.max()))


if __name__ == "__main__":
    main()
