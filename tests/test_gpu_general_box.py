"""General (non-rectangular) periodic boxes on the GPU (dgt_set_box_general).

The reference's box class supports general boxes (periodicBoundaries.h:86-101, 165-178) but
its cell list and Delaunay kernels do not (cellListGPU.h:14-16), so there is no reference
output to compare with.  Parity is anchored instead on the rectangular path, which matches the
reference bit for bit: a rotated rectangle and a sheared basis of a rectangular lattice must
give the same rings, and in genuinely oblique boxes every result must pass the oracle's exact
verifier (rings mutually consistent, CCW, winding once, every edge locally Delaunay, every
circumcircle empty under a global scan), which for points in general position pins the unique
Delaunay triangulation."""
import math

import numpy as np
import pytest

from gpudelaunaytriangulation_b200 import workloads as W
from oracle import oracle as O

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu


def _dgpu():
    from gpudelaunaytriangulation_b200.delaunay import DelaunayGPU, PeriodicBox

    return DelaunayGPU, PeriodicBox


def _build(pts, box, cell=1.0, fp32=True):
    DelaunayGPU, _ = _dgpu()
    n = len(pts)
    d = DelaunayGPU(n, 16, cell, box)
    d.setPrecision(fp32)
    P = torch.from_numpy(np.ascontiguousarray(pts)).cuda()
    tri, nn = d.globalDelaunayTriangulation(P)
    torch.cuda.synchronize()
    t = tri.view(n, -1).cpu().numpy()
    k = nn.cpu().numpy()
    return d, P, tri, nn, t, k


def _same_rings(t0, k0, t1, k1):
    w = min(t0.shape[1], t1.shape[1])
    return np.array_equal(k0, k1) and np.array_equal(O.canonical(t0, k0)[:, :w], O.canonical(t1, k1)[:, :w])


def _oblique_points(n, box, seed):
    M = np.array([[box[0], box[1]], [box[2], box[3]]])
    u = np.random.default_rng(seed).uniform(0.0, 1.0, (n, 2))
    return np.ascontiguousarray(u @ M.T)


def _box_of_area(n, shape):
    # scale a box shape (xx, xy, yx, yy) to unit density for n points
    det = abs(shape[0] * shape[3] - shape[1] * shape[2])
    s = math.sqrt(n / det)
    return tuple(s * v for v in shape)


HEX = (1.0, 0.5, 0.0, math.sqrt(3.0) / 2.0)   # 60-degree lattice
OBLIQUE = (40.0, 13.0, 3.0, 35.0)              # an arbitrary oblique lattice


@pytest.mark.parametrize("theta", [0.37, 1.1])
def test_rotated_rectangle_matches_the_rectangular_path(theta):
    n = 20000
    L = math.sqrt(n)
    pts = W.uniform_points(n, L, 41)
    _, _, _, _, t0, k0 = _build(pts, (L, L))
    R = np.array([[math.cos(theta), -math.sin(theta)], [math.sin(theta), math.cos(theta)]])
    box = R @ np.diag([L, L])
    rbox = (box[0, 0], box[0, 1], box[1, 0], box[1, 1])
    d, P, tri, nn, t1, k1 = _build(pts @ R.T, rbox)
    st = d.stats()
    assert st["error_flags"] == 0 and st["mismatches"] == 0, st
    assert _same_rings(t0, k0, t1, k1)
    assert d.validate(P, tri, nn)["valid"] == 1
    ok, rep = O.verify_general(pts @ R.T, d.kernelBox(), t1, k1)
    assert ok, rep


def test_sheared_basis_of_a_rectangular_lattice_and_shifted_images():
    n = 20000
    L = math.sqrt(n)
    pts = W.uniform_points(n, L, 42)
    _, _, _, _, t0, k0 = _build(pts, (L, L))
    # lattice vectors (L, 0) and (2L, L): the square lattice through a sheared basis
    DelaunayGPU, PeriodicBox = _dgpu()
    d, P, tri, nn, t1, k1 = _build(pts, PeriodicBox.general(L, 2 * L, 0.0, L))
    kb = d.kernelBox()
    assert abs(abs(kb[0] * kb[3] - kb[1] * kb[2]) - L * L) < 1e-9 * L * L
    assert _same_rings(t0, k0, t1, k1)
    # every point moved by a lattice vector: the same periodic point set
    shifted = pts + np.outer(np.arange(n) % 5 - 2, [L, 0.0]) + np.outer(np.arange(n) % 3 - 1, [2 * L, L])
    _, _, _, _, t2, k2 = _build(shifted, (L, 2 * L, 0.0, L))
    assert _same_rings(t0, k0, t2, k2)


@pytest.mark.parametrize("shape", [HEX, OBLIQUE], ids=["hex", "oblique"])
def test_oblique_box_is_delaunay_in_both_precisions(shape):
    n = 30000
    box = _box_of_area(n, shape)
    pts = _oblique_points(n, box, 43)
    d, P, tri, nn, t, k = _build(pts, box)
    st = d.stats()
    assert st["error_flags"] == 0 and st["mismatches"] == 0, st
    assert int(k.sum()) == 6 * n
    assert d.validate(P, tri, nn)["valid"] == 1
    ok, rep = O.verify_general(pts, d.kernelBox(), t, k)
    assert ok, rep
    _, _, _, _, t64, k64 = _build(pts, box, fp32=False)
    assert _same_rings(t, k, t64, k64)


@pytest.mark.parametrize("flip", [True, False], ids=["flips", "rebuild"])
def test_oblique_box_repair_matches_a_fresh_build(flip):
    n = 30000
    box = _box_of_area(n, OBLIQUE)
    pts = _oblique_points(n, box, 44)
    d, P, tri, nn, _, _ = _build(pts, box)
    d.setFlipRepair(flip)
    rng = np.random.default_rng(45)
    for step in range(3):
        pts = pts + rng.normal(0.0, 0.05, pts.shape)   # left unwrapped: any position is valid
        P.copy_(torch.from_numpy(pts))
        d.testAndRepairDelaunayTriangulation(P, tri, nn)
        torch.cuda.synchronize()
        assert d.stats()["error_flags"] == 0
    t = tri.view(n, -1).cpu().numpy()
    k = nn.cpu().numpy()
    _, _, _, _, tf, kf = _build(pts, box)
    assert _same_rings(t, k, tf, kf)
    ok, rep = O.verify_general(pts, d.kernelBox(), t, k)
    assert ok, rep


def test_oblique_box_md_steps_wrap_into_the_unit_cell():
    n = 20000
    box = _box_of_area(n, HEX)
    pts = _oblique_points(n, box, 46)
    d, P, tri, nn, _, _ = _build(pts, box)
    for _ in range(5):
        d.mdStep(P, tri, nn, 0.02, 47)
    torch.cuda.synchronize()
    assert d.stats()["error_flags"] == 0
    q = P.cpu().numpy()
    kb = d.kernelBox()
    Mi = np.linalg.inv(np.array([[kb[0], kb[1]], [kb[2], kb[3]]]))
    u = q @ Mi.T
    assert np.all(u >= -1e-9) and np.all(u < 1.0 + 1e-9)
    assert d.validate(P, tri, nn)["valid"] == 1
    ok, rep = O.verify_general(q, kb, tri.view(n, -1).cpu().numpy(), nn.cpu().numpy())
    assert ok, rep


def test_batch_of_general_and_rectangular_boxes_matches_single_sets():
    from gpudelaunaytriangulation_b200.delaunay import DelaunayBatch

    rng = np.random.default_rng(48)
    hexb = _box_of_area(5000, HEX)
    obl = _box_of_area(3000, OBLIQUE)
    Lr = math.sqrt(4000)
    th = 0.6
    R = np.array([[math.cos(th), -math.sin(th)], [math.sin(th), math.cos(th)]]) @ np.diag([math.sqrt(2000)] * 2)
    rot = (R[0, 0], R[0, 1], R[1, 0], R[1, 1])
    sizes = [5000, 3000, 4000, 0, 2000]
    boxes = [hexb, obl, (Lr, Lr), (10.0, 10.0), rot]
    sets = [_oblique_points(5000, hexb, 49), _oblique_points(3000, obl, 50), W.uniform_points(4000, Lr, 51),
            np.zeros((0, 2)), _oblique_points(2000, rot, 52)]
    pts = np.ascontiguousarray(np.concatenate(sets))
    off = np.concatenate([[0], np.cumsum(sizes)])
    b = DelaunayBatch(sizes, boxes, 16, 1.0)
    P = torch.from_numpy(pts).cuda()
    for step in range(2):
        if step == 1:
            # drift every set, then repair the batch in place
            pts = pts + rng.normal(0.0, 0.03, pts.shape)
            sets = [pts[off[s]:off[s + 1]] for s in range(len(sizes))]
            P.copy_(torch.from_numpy(pts))
            b.testAndRepairDelaunayTriangulation(P, tri, nn)
        else:
            tri, nn = b.globalDelaunayTriangulation(P)
        torch.cuda.synchronize()
        assert b.stats()["error_flags"] == 0
        t = tri.view(len(pts), -1).cpu().numpy()
        k = nn.cpu().numpy()
        for s in range(len(sizes)):
            lo, hi = off[s], off[s + 1]
            if hi == lo:
                continue
            ts = t[lo:hi].copy()
            ts[np.arange(ts.shape[1])[None, :] < k[lo:hi, None]] -= lo
            box = boxes[s] if len(boxes[s]) == 4 else (boxes[s][0], 0.0, 0.0, boxes[s][1])
            if len(boxes[s]) == 2:
                sets[s] = np.mod(sets[s], Lr)   # the single-set rectangular path wants [0, L)
            _, _, _, _, t1, k1 = _build(sets[s], boxes[s])
            assert _same_rings(ts, k[lo:hi], t1, k1), (step, s)
            ok, rep = O.verify_general(sets[s], box, ts, k[lo:hi])
            assert ok, (step, s, rep)


def test_general_box_argument_and_input_errors():
    from gpudelaunaytriangulation_b200 import _native as N

    DelaunayGPU, PeriodicBox = _dgpu()
    n = 2000
    box = _box_of_area(n, OBLIQUE)
    # degenerate (parallel lattice vectors) and non-finite matrices are refused
    for bad in [(10.0, 20.0, 5.0, 10.0), (10.0, 0.0, float("nan"), 10.0), (float("inf"), 1.0, 0.0, 10.0)]:
        with pytest.raises(N.DgtError) as e:
            DelaunayGPU(n, 16, 1.0, PeriodicBox.general(*bad))
        assert e.value.code == N.DGT_ERR_INVALID_ARGUMENT
    # a non-finite coordinate is reported, and the context stays usable
    pts = _oblique_points(n, box, 53)
    d = DelaunayGPU(n, 16, 1.0, box)
    bad_pts = pts.copy()
    bad_pts[7, 0] = float("nan")
    with pytest.raises(N.DgtError) as e:
        d.globalDelaunayTriangulation(torch.from_numpy(bad_pts).cuda())
    assert e.value.code == N.DGT_ERR_BAD_POINTS
    P = torch.from_numpy(pts).cuda()
    tri, nn = d.globalDelaunayTriangulation(P)
    assert d.validate(P, tri, nn)["valid"] == 1
    # too few points to close a ring, as in a rectangular box
    small = _box_of_area(3, HEX)
    d3 = DelaunayGPU(3, 16, 1.0, small)
    with pytest.raises(N.DgtError) as e:
        d3.globalDelaunayTriangulation(torch.from_numpy(_oblique_points(3, small, 54)).cuda())
    assert e.value.code == N.DGT_ERR_DEGENERATE


def test_kernel_box_is_the_oracle_reduction():
    DelaunayGPU, PeriodicBox = _dgpu()
    rng = np.random.default_rng(55)
    for _ in range(20):
        a = rng.uniform(-30, 30, 2)
        b = rng.uniform(-30, 30, 2)
        box = (a[0], b[0], a[1], b[1])
        if abs(a[0] * b[1] - a[1] * b[0]) < 50.0 or (box[1] == 0.0 and box[2] == 0.0):
            continue
        d = DelaunayGPU(100, 16, 1.0, PeriodicBox.general(*box))
        assert d.kernelBox() == O.reduce_basis(box)
        d.close()


@pytest.mark.parametrize("shape", [HEX, OBLIQUE], ids=["hex", "oblique"])
def test_oblique_box_deferred_points_in_pieces(shape):
    # work budget 16 sends most points to the warp-per-point kernel (its general-box tile
    # walk), and the build runs in 1 or 5 overlapped pieces: the same rings as the default
    # build, accepted by the exact verifier
    DelaunayGPU, _ = _dgpu()
    n = 20000
    box = _box_of_area(n, shape)
    pts = _oblique_points(n, box, 47)
    _, _, _, _, t0, k0 = _build(pts, box)
    P = torch.from_numpy(pts).cuda()
    for pieces in (1, 5):
        d = DelaunayGPU(n, 16, 1.0, box)
        d.setWorkBudget(16)
        d.setDeferredOverlap(pieces)
        tri, nn = d.globalDelaunayTriangulation(P)
        st = d.stats()
        assert st["error_flags"] == 0 and st["exact_points"] > n // 4, (pieces, st)
        t = tri.view(n, -1).cpu().numpy()
        k = nn.cpu().numpy()
        assert _same_rings(t0, k0, t, k), pieces
        assert d.validate(P, tri, nn)["valid"] == 1
        d.close()
