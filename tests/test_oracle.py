"""CPU tests of the oracle: the C restatement of the reference's host path must reproduce the
reference's own output (golden fixtures made from oracle/_ref, and oracle/_ref itself when it
is built here), and the exact verifier must accept Delaunay triangulations and reject
planted faults."""
import glob
import os

import numpy as np
import pytest

from gpudelaunaytriangulation_b200 import workloads as W
from oracle import oracle as O

GOLDEN = sorted(glob.glob(os.path.join(os.path.dirname(__file__), "golden", "*.npz")))


def flat(tri, nn):
    c = O.canonical(tri, nn)
    return np.concatenate([c[i, : nn[i]] for i in range(len(nn))]).astype(np.int32)


def unflat(rings, nn, stride=32):
    tri = np.zeros((len(nn), stride), np.int32)
    off = np.concatenate([[0], np.cumsum(nn)])
    for i in range(len(nn)):
        tri[i, : nn[i]] = rings[off[i]: off[i + 1]]
    return tri


@pytest.mark.parametrize("path", GOLDEN, ids=[os.path.basename(p) for p in GOLDEN])
def test_restatement_matches_reference_golden(path):
    g = np.load(path)
    L = g["L"]
    res = O.restated_global(g["points"], L[0], L[1], float(g["cell_size"]), 32)
    assert np.array_equal(res.nn, g["nn"])
    assert np.array_equal(flat(res.tri, res.nn), g["rings"])
    if "moved" in g:
        rep, flags = O.restated_test_and_repair(g["moved"], L[0], L[1], res, float(g["cell_size"]))
        assert np.array_equal(flags, g["repair_flags"])
        assert np.array_equal(rep.nn, g["repair_nn"])
        assert np.array_equal(flat(rep.tri, rep.nn), g["repair_rings"])


@pytest.mark.parametrize("path", GOLDEN, ids=[os.path.basename(p) for p in GOLDEN])
def test_golden_is_delaunay(path):
    g = np.load(path)
    L = g["L"]
    ok, rep = O.verify(g["points"], L[0], L[1], unflat(g["rings"], g["nn"]), g["nn"])
    assert ok, rep
    assert rep["sum_deg"] == 6 * len(g["nn"])
    if "moved" in g:
        ok, rep = O.verify(g["moved"], L[0], L[1], unflat(g["repair_rings"], g["repair_nn"]), g["repair_nn"])
        assert ok, rep


@pytest.mark.skipif(O.ref_lib() is None, reason="oracle/_ref not built (reference sources absent)")
@pytest.mark.parametrize("n,seed", [(300, 11), (5000, 12), (30000, 13)])
def test_restatement_raw_identical_to_reference(n, seed):
    L = float(np.sqrt(n))
    pts = W.uniform_points(n, L, seed)
    a = O.restated_global(pts, L, L, 1.0, 32)
    b = O.reference_global(pts, L, L, 1.0, 32)
    mask = np.arange(32)[None, :] < a.nn[:, None]
    assert np.array_equal(a.nn, b.nn)
    # same rings including where each starts: same arithmetic in the same order
    assert np.array_equal(np.where(mask, a.tri, -1), np.where(mask, b.tri, -1))
    moved = W.displace(pts, 0.05, L, L, seed + 7)
    ra, fa = O.restated_test_and_repair(moved, L, L, a)
    rb, fb = O.reference_test_and_repair(moved, L, L, b)
    assert np.array_equal(fa, fb)
    assert np.array_equal(O.canonical(ra.tri, ra.nn), O.canonical(rb.tri, rb.nn))


def test_restatement_cell_size_independent():
    n = 4000
    L = float(np.sqrt(n))
    pts = W.uniform_points(n, L, 21)
    a = O.restated_global(pts, L, L, 1.0, 32)
    b = O.restated_global(pts, L, L, 2.5, 32)
    assert np.array_equal(O.canonical(a.tri, a.nn), O.canonical(b.tri, b.nn))


def test_verifier_rejects_planted_faults():
    n = 3000
    L = float(np.sqrt(n))
    pts = W.uniform_points(n, L, 5)
    t = O.restated_global(pts, L, L, 1.0, 32)
    ok, rep = O.verify(pts, L, L, t.tri, t.nn)
    assert ok, rep
    # reversed ring (CW): orientation and winding fail
    bad = t.tri.copy()
    bad[10, : t.nn[10]] = bad[10, : t.nn[10]][::-1]
    ok, rep = O.verify(pts, L, L, bad, t.nn)
    assert not ok and rep["nonpositive"] > 0
    # dropped neighbour: Euler sum and symmetry fail
    nn = t.nn.copy()
    nn[20] -= 1
    ok, rep = O.verify(pts, L, L, t.tri, nn)
    assert not ok and rep["sum_deg"] == 6 * n - 1 and rep["asym"] > 0
    # a point moved off its Delaunay position: the old rings are no longer Delaunay
    moved = pts.copy()
    moved[30] += 0.3
    moved = W.wrap(moved, L, L)
    ok, rep = O.verify(moved, L, L, t.tri, t.nn)
    assert not ok and (rep["not_local_dt"] > 0 or rep["nonpositive"] > 0)


def test_exact_predicates_known_answers():
    # circle through (0,0), (1,0), (0,1): centre (0.5, 0.5)
    a, b = [1.0, 0.0], [0.0, 1.0]
    assert O.incircle0(a, b, [0.5, 0.5]) == 1
    assert O.incircle0(a, b, [2.0, 2.0]) == -1
    assert O.incircle0(a, b, [1.0, 1.0]) == 0          # exactly cocircular
    assert O.orient0(a, b) == 1 and O.orient0(b, a) == -1
    assert O.orient0([1.0, 1.0], [2.0, 2.0]) == 0
    # near-degenerate: one ulp off the circle, below the resolution of a naive float64 sum
    assert O.incircle0(a, b, [1.0, 1.0 - 2.0 ** -53]) == 1
    assert O.incircle0(a, b, [1.0, 1.0 + 2.0 ** -52]) == -1
    big = 2.0 ** 40   # magnitudes where the naive determinant loses all bits
    assert O.incircle0([big, 0.0], [0.0, big], [big, big - 2.0 ** -12]) == 1


def test_incircle_sign_matches_rational_arithmetic():
    from fractions import Fraction as F

    rng = np.random.default_rng(3)
    for _ in range(300):
        a, b, d = rng.normal(size=(3, 2)) * rng.choice([1e-3, 1.0, 1e3])
        if rng.random() < 0.3:   # nearly cocircular d
            c = np.array([(a @ a) * b[1] - (b @ b) * a[1], (b @ b) * a[0] - (a @ a) * b[0]]) / (2 * (a[0] * b[1] - a[1] * b[0]))
            th = rng.uniform(0, 2 * np.pi)
            d = c + np.linalg.norm(c) * np.array([np.cos(th), np.sin(th)])
        fa = [F(x) for x in a]
        fb = [F(x) for x in b]
        fd = [F(x) for x in d]
        na, nb, nd = (fa[0] ** 2 + fa[1] ** 2, fb[0] ** 2 + fb[1] ** 2, fd[0] ** 2 + fd[1] ** 2)
        v = na * (fd[0] * fb[1] - fd[1] * fb[0]) + nb * (fa[0] * fd[1] - fa[1] * fd[0]) + nd * (fb[0] * fa[1] - fb[1] * fa[0])
        want = (v > 0) - (v < 0)
        assert O.incircle0(a, b, d) == want


def test_offsets_single_rounding():
    L = 2048.0
    c = np.array([2047.8, 0.3])
    p = np.array([0.3, 2047.9])
    out = np.zeros(2)
    O.lib().orc_offset(c.ctypes.data_as(O._P_D), p.ctypes.data_as(O._P_D), L, L, out.ctypes.data_as(O._P_D))
    from fractions import Fraction as F

    ex = [F(2047.8) - F(L) - F(0.3), F(0.3) - (F(2047.9) - F(L))]
    assert out[0] == float(ex[0]) and out[1] == float(ex[1])


@pytest.mark.skipif(O.ref_lib() is None, reason="oracle/_ref not built (reference sources absent)")
def test_reference_seed_pass_guard_measures_polygons():
    # the guard bench.py runs before the reference's own CUDA kernels: the reference's seed
    # pass, on the host, over the same points; its polygons must stay well inside the
    # reference's rows (it has no capacity check there), and the measurement must flag a row
    # width it reaches
    n = 20000
    L = float(np.sqrt(n))
    pts = W.uniform_points(n, L, 2026)
    mx = O.reference_seed_max(pts, L, L, 1.0, 64)
    assert 4 <= mx <= 12
    assert O.reference_seed_max(pts, L, L, 1.0, mx) == -1


@pytest.mark.skipif(O.ref_lib() is None, reason="oracle/_ref not built (reference sources absent)")
def test_hilbert_index_matches_reference_xy2d():
    # the restated curve index equals the reference's own xy2d (hilbert_curve.cpp:229) at every
    # grid order the device ordering uses
    rng = np.random.default_rng(5)
    for m in range(1, 16):
        g = 1 << m
        xs, ys = rng.integers(0, g, 300), rng.integers(0, g, 300)
        mine = O.hilbert_index(m, xs, ys)
        ref = np.array([O.reference_xy2d(m, a, b) for a, b in zip(xs, ys)])
        assert np.array_equal(mine, ref), m


def test_hilbert_index_is_a_continuous_curve():
    # known answers of the curve: on a 2^m grid the index is a bijection onto [0, 4^m), and
    # squares with consecutive indices share an edge
    for m in (1, 2, 3, 5):
        g = 1 << m
        x, y = np.meshgrid(np.arange(g), np.arange(g))
        d = O.hilbert_index(m, x.ravel(), y.ravel())
        assert np.array_equal(np.sort(d), np.arange(g * g))
        at = np.argsort(d)
        step = np.abs(np.diff(x.ravel()[at])) + np.abs(np.diff(y.ravel()[at]))
        assert (step == 1).all(), m
    # the first-order curve: (0,0) -> (0,1) -> (1,1) -> (1,0)
    assert O.hilbert_index(1, [0, 0, 1, 1], [0, 1, 1, 0]).tolist() == [0, 1, 2, 3]
