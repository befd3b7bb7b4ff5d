"""Device-side validation (dgt_validate) against the oracle's exact verifier.

The validator's counts -- malformed rows, asymmetric spokes, non-positive fan triangles,
fans not winding once, spokes failing the exact local Delaunay test, and the ring-size sum
-- must equal those of the oracle verifier (oracle/dgt_oracle.c, orc_verify) on a valid
triangulation, on one whose points moved without repair, and on rows with planted faults
(faults planted in the arrays' data, in range: the validator reads them, it never follows
an index it has not checked)."""
import numpy as np
import pytest

from gpudelaunaytriangulation_b200 import workloads as W
from oracle import oracle as O

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu


def build(n, seed):
    from gpudelaunaytriangulation_b200.delaunay import DelaunayGPU

    L = float(np.sqrt(n))
    pts = W.uniform_points(n, L, seed)
    d = DelaunayGPU(n, 16, 1.0, (L, L))
    P = torch.from_numpy(pts).cuda()
    tri, nn = d.globalDelaunayTriangulation(P)
    return d, P, tri, nn, pts, L


def same_as_oracle(v, pts, L, tri, nn):
    n = len(pts)
    t = tri.view(n, -1).cpu().numpy()
    k = nn.cpu().numpy()
    ok, rep = O.verify(pts, L, L, t, k, global_scan=False)
    assert v["points"] == n
    assert v["sum_neighbors"] == rep["sum_deg"], (v, rep)
    assert v["bad_rows"] == rep["bad_index"], (v, rep)
    assert v["asymmetric"] == rep["asym"], (v, rep)
    assert v["not_ccw"] == rep["nonpositive"], (v, rep)
    assert v["winding"] == rep["winding"], (v, rep)
    assert v["not_delaunay"] == rep["not_local_dt"], (v, rep)
    assert bool(v["valid"]) == ok, (v, rep)


def test_valid_then_moved_then_repaired():
    n = 20000
    d, P, tri, nn, pts, L = build(n, 5)
    v = d.validate(P, tri, nn)
    assert v["valid"] == 1 and v["sum_neighbors"] == 6 * n, v
    same_as_oracle(v, pts, L, tri, nn)
    moved = W.displace(pts, 0.2, L, L, 6)
    P.copy_(torch.from_numpy(moved))
    v = d.validate(P, tri, nn)
    assert v["valid"] == 0 and v["not_delaunay"] > 0 and v["not_ccw"] > 0, v
    same_as_oracle(v, moved, L, tri, nn)
    d.testAndRepairDelaunayTriangulation(P, tri, nn)
    v = d.validate(P, tri, nn)
    assert v["valid"] == 1, v
    same_as_oracle(v, moved, L, tri, nn)


def test_planted_faults_are_counted():
    n = 20000
    d, P, tri, nn, pts, L = build(n, 7)
    t = tri.view(n, -1)
    # two adjacent entries swapped (an inverted triangle and two asymmetric spokes)
    t[11, 1], t[11, 2] = t[11, 2].clone(), t[11, 1].clone()
    # a repeated entry (malformed row)
    t[23, 0] = t[23, 1]
    # a ring length too short (malformed row)
    nn[37] = 2
    # a neighbour replaced by a far point (asymmetric, not Delaunay)
    t[51, 0] = (int(t[51, 0]) + n // 2) % n
    torch.cuda.synchronize()
    v = d.validate(P, tri, nn)
    assert v["valid"] == 0 and v["bad_rows"] == 2 and v["asymmetric"] > 0 and v["not_ccw"] > 0, v
    same_as_oracle(v, pts, L, tri, nn)


def test_cell_order_renumbering():
    # the order from the last binning is a permutation along which the cell index never
    # decreases; triangulating the renumbered points gives the same rings, relabelled
    n = 30000
    d, P, tri, nn, pts, L = build(n, 9)
    order = d.cellOrder().cpu().numpy().astype(np.int64)
    assert np.array_equal(np.sort(order), np.arange(n))
    xs = int(np.floor(L / 1.0))
    cw = L / xs
    cell = np.minimum(np.floor(pts[order, 1] / cw), xs - 1) * xs + np.minimum(np.floor(pts[order, 0] / cw), xs - 1)
    assert (np.diff(cell) >= 0).all()
    d2, P2, tri2, nn2, _, _ = build(n, 9)
    P2.copy_(torch.from_numpy(np.ascontiguousarray(pts[order])))
    d2.globalDelaunayTriangulation(P2, tri2, nn2)
    t2 = tri2.view(n, -1).cpu().numpy()
    k2 = nn2.cpu().numpy()
    back = np.full_like(t2, -1)
    kk = np.zeros(n, np.int32)
    for new in range(n):
        back[order[new], : k2[new]] = order[t2[new, : k2[new]]]
        kk[order[new]] = k2[new]
    t = tri.view(n, -1).cpu().numpy()
    k = nn.cpu().numpy()
    assert np.array_equal(kk, k)
    assert np.array_equal(O.canonical(back, kk), O.canonical(t, k))
