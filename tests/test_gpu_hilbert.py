"""Hilbert-curve order of the points (dgt_get_hilbert_order) against the oracle's
restatement (oracle.hilbert_order, whose curve index equals the reference's own xy2d,
tests/test_oracle.py): equal orders for uniform, clustered and batched inputs, a locality
check for a general box, and renumbered points triangulate to the same rings, relabelled.
Integer output: the bar is equality."""
import numpy as np
import pytest

from gpudelaunaytriangulation_b200 import workloads as W
from oracle import oracle as O

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu


def _dg():
    from gpudelaunaytriangulation_b200.delaunay import DelaunayGPU

    return DelaunayGPU


@pytest.mark.parametrize("case", ["uniform", "mixture", "rectangle", "small"])
def test_hilbert_order_matches_oracle(case):
    if case == "uniform":
        n = 100000
        L = float(np.sqrt(n))
        pts, Lx, Ly = W.uniform_points(n, L, 71), L, L
    elif case == "mixture":
        pts, L = W.gaussian_mixture(65536, components=64, sigma=2.0, L=256.0, seed=9)
        Lx = Ly = L
    elif case == "rectangle":
        pts, Lx, Ly = W.triangular_lattice(200, 150, 1.0, 1e-4, seed=4)
    else:
        pts, Lx, Ly = W.uniform_points(5, 3.0, 72), 3.0, 3.0
    n = len(pts)
    d = _dg()(n, 16, 1.0, (Lx, Ly))
    P = torch.from_numpy(np.ascontiguousarray(pts)).cuda()
    order = d.hilbertOrder(P).cpu().numpy().astype(np.int64)
    ref = O.hilbert_order(pts, [n], [(Lx, Ly)])
    assert np.array_equal(order, ref)
    d.close()


def test_hilbert_order_batched_sets():
    from gpudelaunaytriangulation_b200.delaunay import DelaunayBatch

    pts, sizes, boxes = W.ensemble(12, 200, 5000, seed=13)
    b = DelaunayBatch(sizes, boxes, 16, 1.0)
    P = torch.from_numpy(pts).cuda()
    order = b.hilbertOrder(P).cpu().numpy().astype(np.int64)
    assert np.array_equal(order, O.hilbert_order(pts, sizes, boxes))
    b.close()


def test_hilbert_order_general_box_is_local():
    # a 60-degree box: the curve runs over the fractional frame; consecutive points of the
    # order lie close together (a random order averages about a third of the box apart)
    n = 40000
    s = float(np.sqrt(n / (np.sqrt(3.0) / 2.0)))
    box = (s, 0.5 * s, 0.0, s * np.sqrt(3.0) / 2.0)
    M = np.array([[box[0], box[1]], [box[2], box[3]]])
    pts = np.ascontiguousarray(np.random.default_rng(73).uniform(0.0, 1.0, (n, 2)) @ M.T)
    d = _dg()(n, 16, 1.0, box)
    P = torch.from_numpy(pts).cuda()
    order = d.hilbertOrder(P).cpu().numpy().astype(np.int64)
    assert np.array_equal(np.sort(order), np.arange(n))
    frac = pts @ np.linalg.inv(M).T
    steps = np.abs(np.diff(frac[order], axis=0))
    steps = np.minimum(steps, 1.0 - steps)   # periodic
    assert np.sqrt((steps ** 2).sum(axis=1)).mean() * np.sqrt(n) < 2.0
    d.close()


def test_hilbert_renumbering_gives_same_rings_relabelled():
    n = 30000
    L = float(np.sqrt(n))
    pts = W.uniform_points(n, L, 74)
    d = _dg()(n, 16, 1.0, (L, L))
    P = torch.from_numpy(pts).cuda()
    tri, nn = d.globalDelaunayTriangulation(P)
    order = d.hilbertOrder(P).cpu().numpy().astype(np.int64)
    d2 = _dg()(n, 16, 1.0, (L, L))
    P2 = torch.from_numpy(np.ascontiguousarray(pts[order])).cuda()
    tri2, nn2 = d2.globalDelaunayTriangulation(P2)
    t2, k2 = tri2.view(n, -1).cpu().numpy(), nn2.cpu().numpy()
    back = np.full_like(t2, -1)
    kk = np.zeros(n, np.int32)
    for new in range(n):
        back[order[new], : k2[new]] = order[t2[new, : k2[new]]]
        kk[order[new]] = k2[new]
    t, k = tri.view(n, -1).cpu().numpy(), nn.cpu().numpy()
    assert np.array_equal(kk, k)
    assert np.array_equal(O.canonical(back, kk), O.canonical(t, k))
    # renumbered, Delaunay neighbours sit at nearby indices
    span = np.abs(t2[:, :6] - np.arange(n)[:, None])
    assert np.median(span) < n / 50
    d.close()
    d2.close()


def test_hilbert_sort_points_in_place():
    # the reference driver's hilbertSortArray: points reordered in place along the curve
    n = 20000
    L = float(np.sqrt(n))
    pts = W.uniform_points(n, L, 75)
    d = _dg()(n, 16, 1.0, (L, L))
    P = torch.from_numpy(pts.copy()).cuda()
    order = d.hilbertSort(P).cpu().numpy().astype(np.int64)
    ref = O.hilbert_order(pts, [n], [(L, L)])
    assert np.array_equal(order, ref)
    assert np.array_equal(P.cpu().numpy(), pts[ref])
    # sorted again: already in curve order
    again = d.hilbertSort(P).cpu().numpy()
    assert np.array_equal(again, np.arange(n))
    d.close()
