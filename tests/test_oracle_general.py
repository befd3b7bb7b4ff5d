"""CPU tests of the oracle's general (non-rectangular) periodic box: the minimum-image offset,
the basis reduction and the exact verifier.  The reference's cell list and Delaunay kernels
are rectangular-only (cellListGPU.h:14-16), so its box class (periodicBoundaries.h:86-101,
165-178) is the specification, and the rectangular path -- pinned against the reference's own
output -- anchors these checks: a rotated rectangle, or a sheared basis of the same lattice,
must keep the triangulation."""
from fractions import Fraction as F

import numpy as np
import pytest

from gpudelaunaytriangulation_b200 import workloads as W
from oracle import oracle as O


def _rect_offset(c, p, L):
    out = np.zeros(2)
    c = np.ascontiguousarray(c, np.float64)
    p = np.ascontiguousarray(p, np.float64)
    O.lib().orc_offset(c.ctypes.data_as(O._P_D), p.ctypes.data_as(O._P_D), L, L, out.ctypes.data_as(O._P_D))
    return out


def test_general_offset_of_a_diagonal_box_is_the_rectangular_offset():
    rng = np.random.default_rng(11)
    L = 64.0
    for _ in range(2000):
        c, p = rng.uniform(0, L, 2), rng.uniform(0, L, 2)
        if np.any(np.abs(np.abs(c - p) - 0.5 * L) < 1e-6):
            continue
        g = O.offset_general(c, p, (L, 0.0, 0.0, L))
        r = _rect_offset(c, p, L)
        assert g[0] == r[0] and g[1] == r[1]


def test_general_offset_is_the_fractional_minimum_image():
    rng = np.random.default_rng(12)
    box = (40.0, 13.0, 3.0, 35.0)   # lattice vectors (40, 3) and (13, 35)
    M = np.array([[box[0], box[1]], [box[2], box[3]]])
    Mi = np.linalg.inv(M)
    for _ in range(2000):
        c = M @ rng.uniform(-0.5, 1.5, 2)
        p = M @ rng.uniform(0.0, 1.0, 2)
        d = O.offset_general(c, p, box)
        shift = Mi @ ((c - p) - d)   # a lattice vector in fractional coordinates: integers
        assert np.allclose(shift, np.round(shift), atol=1e-9)
        assert np.all(np.abs(Mi @ d) <= 0.5 + 1e-9)


def test_general_offset_single_shift_rounding():
    # a shift that is positive is taken off the far coordinate first (exact, Sterbenz), so
    # the result is the exact difference rounded once
    box = (2048.0, 0.0, 0.0, 2048.0)
    c, p = np.array([2047.8, 0.3]), np.array([0.3, 2047.9])
    d = O.offset_general(c, p, box)
    ex = [F(2047.8) - F(2048.0) - F(0.3), F(0.3) - (F(2047.9) - F(2048.0))]
    assert d[0] == float(ex[0]) and d[1] == float(ex[1])


def test_basis_reduction():
    # (10, 0), (23, 9) -> (3, 9), (10, 0): the same lattice (|det| kept), reduced, idempotent
    r = O.reduce_basis((10.0, 23.0, 0.0, 9.0))
    assert r == (3.0, 10.0, 9.0, 0.0)
    assert O.reduce_basis(r) == r
    rng = np.random.default_rng(13)
    for _ in range(200):
        a = rng.uniform(-5, 5, 2)
        b = rng.uniform(-5, 5, 2)
        box = (a[0], b[0], a[1], b[1])
        det = a[0] * b[1] - a[1] * b[0]
        if abs(det) < 1.0:
            continue
        r = O.reduce_basis(box)
        ra, rb = np.array([r[0], r[2]]), np.array([r[1], r[3]])
        assert abs(abs(r[0] * r[3] - r[1] * r[2]) - abs(det)) < 1e-9 * abs(det)
        assert ra @ ra <= rb @ rb * (1 + 1e-12)
        assert abs(ra @ rb) <= 0.5 * (ra @ ra) * (1 + 1e-12)


def _rotated(pts, L, theta):
    R = np.array([[np.cos(theta), -np.sin(theta)], [np.sin(theta), np.cos(theta)]])
    box = R @ np.diag([L, L])
    return pts @ R.T, (box[0, 0], box[0, 1], box[1, 0], box[1, 1])


def test_verifier_general_box_invariances_and_planted_faults():
    n = 3000
    L = float(np.sqrt(n))
    pts = W.uniform_points(n, L, 5)
    t = O.restated_global(pts, L, L, 1.0, 32)
    ok, rep = O.verify(pts, L, L, t.tri, t.nn)
    assert ok, rep
    # the same lattice through a sheared basis: (L, 0) and (L, L)
    ok, rep = O.verify_general(pts, (L, L, 0.0, L), t.tri, t.nn)
    assert ok, rep
    # rotated points in the rotated box: rotation keeps every circle
    rp, rbox = _rotated(pts, L, 0.37)
    ok, rep = O.verify_general(rp, rbox, t.tri, t.nn)
    assert ok, rep
    # points moved by lattice vectors: the same periodic point set
    shifted = rp + np.outer(np.arange(n) % 3 - 1, [rbox[0], rbox[2]])
    ok, rep = O.verify_general(shifted, rbox, t.tri, t.nn)
    assert ok, rep
    # planted faults, as for the rectangular verifier
    bad = t.tri.copy()
    bad[10, : t.nn[10]] = bad[10, : t.nn[10]][::-1]
    ok, rep = O.verify_general(rp, rbox, bad, t.nn)
    assert not ok and rep["nonpositive"] > 0
    nn = t.nn.copy()
    nn[20] -= 1
    ok, rep = O.verify_general(rp, rbox, t.tri, nn)
    assert not ok and rep["sum_deg"] == 6 * n - 1 and rep["asym"] > 0
    moved = rp.copy()
    moved[30] += 0.3
    ok, rep = O.verify_general(moved, rbox, t.tri, t.nn)
    assert not ok and (rep["not_local_dt"] > 0 or rep["nonpositive"] > 0)


def test_python_box_mirror_wraps_into_the_unit_cell():
    # PeriodicBox (the host mirror of periodicBoundaries) on the CPU: the same box from a
    # tuple, the reference's getBoxDims order, and putInBoxReal for a general box keeping
    # each point's lattice class
    torch = pytest.importorskip("torch")
    from gpudelaunaytriangulation_b200.delaunay import PeriodicBox

    b = PeriodicBox.of((10.0, 4.0, 1.0, 8.0))
    assert not b.isBoxSquare() and b.getBoxDims() == (10.0, 4.0, 1.0, 8.0)
    assert PeriodicBox.of((5.0, 6.0)).isBoxSquare()
    rng = np.random.default_rng(14)
    p = torch.from_numpy(rng.uniform(-40.0, 40.0, (500, 2)))
    q = b.putInBoxReal(p).numpy()
    M = np.array([[10.0, 4.0], [1.0, 8.0]])
    u = q @ np.linalg.inv(M).T
    assert np.all(u >= -1e-12) and np.all(u < 1.0 + 1e-12)
    shift = (p.numpy() - q) @ np.linalg.inv(M).T
    assert np.allclose(shift, np.round(shift), atol=1e-9)
