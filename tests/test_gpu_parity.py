"""GPU parity: the CUDA path (through the C ABI) against the oracle.

Bar: rings bit-identical after canonical rotation to the reference's own output (golden
fixtures made from oracle/_ref) and to the C restatement of the reference, every
triangulation accepted by the exact verifier (consistent rings, CCW fans winding once,
every edge locally Delaunay, every circumcircle empty, sum of ring sizes = 6N), and zero
float32-filter decisions contradicted by float64 in check mode."""
import glob
import os

import numpy as np
import pytest

from gpudelaunaytriangulation_b200 import _native as N
from gpudelaunaytriangulation_b200 import workloads as W
from oracle import oracle as O

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

GOLDEN = sorted(glob.glob(os.path.join(os.path.dirname(__file__), "golden", "*.npz")))


def _dg():
    from gpudelaunaytriangulation_b200.delaunay import DelaunayGPU

    return DelaunayGPU


def flat(tri, nn):
    c = O.canonical(tri, nn)
    return np.concatenate([c[i, : nn[i]] for i in range(len(nn))]).astype(np.int32)


def gpu_build(pts, Lx, Ly, cell=1.0, maxn=16, fp32=True, check=False):
    n = len(pts)
    d = _dg()(n, maxn, cell, (Lx, Ly))
    d.setPrecision(fp32)
    d.setCheckMode(check)
    P = torch.from_numpy(np.ascontiguousarray(pts)).cuda()
    tri, nn = d.globalDelaunayTriangulation(P)
    torch.cuda.synchronize()
    return d, P, tri, nn


def host(tri, nn):
    n = nn.numel()
    return tri.view(n, -1).cpu().numpy(), nn.cpu().numpy()


def assert_delaunay(pts, Lx, Ly, t, nn, scan=True):
    ok, rep = O.verify(pts, Lx, Ly, t, nn, global_scan=scan)
    assert ok, rep
    assert rep["sum_deg"] == 6 * len(pts)


@pytest.mark.parametrize("path", GOLDEN, ids=[os.path.basename(p) for p in GOLDEN])
@pytest.mark.parametrize("fp32", [True, False], ids=["fp32filter", "fp64"])
def test_build_matches_reference_golden(path, fp32):
    g = np.load(path)
    L = g["L"]
    d, P, tri, nn = gpu_build(g["points"], L[0], L[1], float(g["cell_size"]), 16, fp32, check=True)
    t, k = host(tri, nn)
    assert np.array_equal(k, g["nn"])
    assert np.array_equal(flat(t, k), g["rings"])
    st = d.stats()
    assert st["mismatches"] == 0 and st["error_flags"] == 0
    assert_delaunay(g["points"], L[0], L[1], t, k)


@pytest.mark.parametrize("path", [p for p in GOLDEN if "n10000" not in p], ids=lambda p: os.path.basename(p))
def test_repair_matches_reference_golden(path):
    g = np.load(path)
    L = g["L"]
    d, P, tri, nn = gpu_build(g["points"], L[0], L[1], float(g["cell_size"]))
    P.copy_(torch.from_numpy(g["moved"]))
    d.testAndRepairDelaunayTriangulation(P, tri, nn)
    t, k = host(tri, nn)
    assert np.array_equal(k, g["repair_nn"])
    assert np.array_equal(flat(t, k), g["repair_rings"])


@pytest.mark.parametrize("n,seed,cell", [(1000, 31, 1.0), (50000, 32, 1.0), (50000, 33, 0.6), (50000, 34, 2.0)])
def test_build_matches_restated_reference(n, seed, cell):
    L = float(np.sqrt(n))
    pts = W.uniform_points(n, L, seed)
    ref = O.restated_global(pts, L, L, 1.0, 32)
    for fp32 in (True, False):
        d, P, tri, nn = gpu_build(pts, L, L, cell, 16, fp32, check=True)
        t, k = host(tri, nn)
        assert np.array_equal(k, ref.nn)
        assert np.array_equal(O.canonical(t, k)[:, :16], O.canonical(ref.tri, ref.nn)[:, :16])
        st = d.stats()
        assert st["mismatches"] == 0, st
        assert st["points"] + st["exact_points"] >= n


def test_fp32_filter_and_fp64_identical_and_counted():
    n = 200000
    L = float(np.sqrt(n))
    pts = W.uniform_points(n, L, 41)
    d1, _, t1, k1 = gpu_build(pts, L, L, 1.0, 16, True, check=True)
    s1 = d1.stats()
    d2, _, t2, k2 = gpu_build(pts, L, L, 1.0, 16, False)
    assert torch.equal(k1, k2) and torch.equal(t1, t2)
    assert s1["mismatches"] == 0
    assert s1["tests"] > 0 and s1["fp32_undecided"] < 1e-3 * s1["tests"]
    t, k = host(t1, k1)
    assert_delaunay(pts, L, L, t, k, scan=False)


@pytest.mark.parametrize("sigma,steps", [(0.02, 4), (0.1, 2)])
def test_repair_steps_match_fresh_triangulation(sigma, steps):
    n = 30000
    L = float(np.sqrt(n))
    pts = W.uniform_points(n, L, 51)
    d, P, tri, nn = gpu_build(pts, L, L)
    cur = pts
    for s in range(steps):
        cur = W.displace(cur, sigma, L, L, 900 + s)
        P.copy_(torch.from_numpy(cur))
        d.testAndRepairDelaunayTriangulation(P, tri, nn)
        t, k = host(tri, nn)
        ref = O.restated_global(cur, L, L, 1.0, 32)
        assert np.array_equal(k, ref.nn)
        assert np.array_equal(O.canonical(t, k)[:, :16], O.canonical(ref.tri, ref.nn)[:, :16])
        st = d.stats()
        assert st["flagged"] + st["flips"] > 0 and st["error_flags"] == 0


@pytest.mark.parametrize("flip", [True, False], ids=["flips", "rebuild_only"])
def test_repair_reuses_cell_lists_until_points_drift(flip):
    # small moves keep the last binning's cell lists (certification widened by the largest
    # move); once the accumulated move passes half a cell the call rebins; every step must
    # equal a fresh triangulation
    n = 30000
    L = float(np.sqrt(n))
    pts = W.uniform_points(n, L, 57)
    d, P, tri, nn = gpu_build(pts, L, L)
    d.setFlipRepair(flip)
    cur = pts
    seen = []
    for s in range(8):
        cur = W.displace(cur, 0.06, L, L, 800 + s)
        P.copy_(torch.from_numpy(cur))
        d.testAndRepairDelaunayTriangulation(P, tri, nn)
        st = d.stats()
        assert st["error_flags"] == 0, st
        seen.append(st["rebinned"])
        t, k = host(tri, nn)
        ref = O.restated_global(cur, L, L, 1.0, 32)
        assert np.array_equal(k, ref.nn), s
        assert np.array_equal(O.canonical(t, k)[:, :16], O.canonical(ref.tri, ref.nn)[:, :16]), s
    assert seen[0] == 0 and 1 in seen, seen


@pytest.mark.parametrize("sigma", [0.02, 0.3])
def test_flip_and_rebuild_repairs_agree(sigma):
    # flip-first repair (default) and rebuild-only repair (the reference's strategy) must give
    # the fresh triangulation of the moved points; sigma 0.3 inverts many fans (rebuild path)
    n = 30000
    L = float(np.sqrt(n))
    pts = W.uniform_points(n, L, 53)
    runs = {}
    for flip in (True, False):
        d, P, tri, nn = gpu_build(pts, L, L)
        d.setFlipRepair(flip)
        cur = pts
        for s in range(3):
            cur = W.displace(cur, sigma, L, L, 700 + s)
            P.copy_(torch.from_numpy(cur))
            d.testAndRepairDelaunayTriangulation(P, tri, nn)
            st = d.stats()
            assert st["error_flags"] == 0, st
            if flip:
                assert st["flips"] > 0, st
            else:
                assert st["flips"] == 0 and st["flagged"] > 0, st
        runs[flip] = host(tri, nn)
    ref = O.restated_global(cur, L, L, 1.0, 32)
    for flip, (t, k) in runs.items():
        assert np.array_equal(k, ref.nn), flip
        assert np.array_equal(O.canonical(t, k)[:, :16], O.canonical(ref.tri, ref.nn)[:, :16]), flip


def test_repair_of_reference_style_local_moves():
    # triangulation.cpp:322-364: a random 5% of points each moved by U(-0.1, 0.1) per axis
    n = 20000
    L = float(np.sqrt(n))
    pts = W.uniform_points(n, L, 61)
    d, P, tri, nn = gpu_build(pts, L, L)
    rng = np.random.default_rng(61)
    idx = rng.permutation(n)[: n // 20]
    moved = pts.copy()
    moved[idx] += rng.uniform(-0.1, 0.1, size=(len(idx), 2))
    moved = W.wrap(moved, L, L)
    P.copy_(torch.from_numpy(moved))
    d.testAndRepairDelaunayTriangulation(P, tri, nn)
    t, k = host(tri, nn)
    ref = O.restated_global(moved, L, L, 1.0, 32)
    assert np.array_equal(O.canonical(t, k)[:, :16], O.canonical(ref.tri, ref.nn)[:, :16])
    assert d.stats()["repaired"] < n // 2


def test_gpu_displacement_then_repair():
    n = 40000
    L = float(np.sqrt(n))
    pts = W.uniform_points(n, L, 71)
    d, P, tri, nn = gpu_build(pts, L, L)
    for step in range(3):
        d.displace(P, 0.02, seed=7, step=step)
        d.testAndRepairDelaunayTriangulation(P, tri, nn)
    cur = P.cpu().numpy()
    assert (cur >= 0).all() and (cur < L).all()
    t, k = host(tri, nn)
    ref = O.restated_global(cur, L, L, 1.0, 32)
    assert np.array_equal(O.canonical(t, k)[:, :16], O.canonical(ref.tri, ref.nn)[:, :16])


@pytest.mark.parametrize("n", [40, 100, 333])
def test_small_sets(n):
    L = float(np.sqrt(n))
    pts = W.uniform_points(n, L, 81 + n)
    d, P, tri, nn = gpu_build(pts, L, L, 1.0, 16)
    t, k = host(tri, nn)
    ref = O.restated_global(pts, L, L, 1.0, 32)
    assert (ref.tri[np.arange(32)[None, :] < ref.nn[:, None]] >= 0).all()
    assert np.array_equal(O.canonical(t, k)[:, :16], O.canonical(ref.tri, ref.nn)[:, :16])


def test_tiny_box_rings_are_closed():
    # 12 points in a 3.5-wide box: cells see their own periodic images, the minimum-image
    # one-ring is not a torus triangulation any more; the reference keeps virtual corners
    # (index -1) in such rings, this library closes every ring with real points
    n = 12
    L = float(np.sqrt(n))
    pts = W.uniform_points(n, L, 93)
    d, P, tri, nn = gpu_build(pts, L, L, 1.0, 16)
    t, k = host(tri, nn)
    assert (k >= 3).all()
    for i in range(n):
        assert ((t[i, : k[i]] >= 0) & (t[i, : k[i]] < n) & (t[i, : k[i]] != i)).all()


def test_rectangular_lattice_box():
    pts, Lx, Ly = W.triangular_lattice(64, 64, 1.0, 1e-4, seed=3)
    for fp32 in (True, False):
        d, P, tri, nn = gpu_build(pts, Lx, Ly, 0.0, 16, fp32, check=True)
        t, k = host(tri, nn)
        assert (k == 6).all()
        assert_delaunay(pts, Lx, Ly, t, k)
        assert d.stats()["mismatches"] == 0


def test_clustered_gaussian_mixture():
    # cluster spacing / box as in the 1M-point 64-cluster workload (voids well below L/2)
    pts, L = W.gaussian_mixture(65536, components=64, sigma=2.0, L=256.0, seed=9)
    d, P, tri, nn = gpu_build(pts, L, L, 0.0, 16, True, check=True)
    st = d.stats()
    assert st["error_flags"] == 0 and st["mismatches"] == 0, st
    t, k = host(tri, nn)
    assert_delaunay(pts, L, L, t, k)
    ref = O.restated_global(pts, L, L, 1.0, 64)
    assert np.array_equal(O.canonical(t, k)[:, : t.shape[1]], O.canonical(ref.tri, ref.nn)[:, : t.shape[1]])


@pytest.mark.parametrize("case", ["uniform", "lattice", "mixture"])
def test_warp_per_point_kernel_same_rings(case):
    # work budget 0 sends every point to the warp-per-point kernel (float64 + exact, shared
    # ring): its rings must equal the restated reference and the per-thread kernel's
    if case == "uniform":
        n = 30000
        L = float(np.sqrt(n))
        pts, Lx, Ly = W.uniform_points(n, L, 21), L, L
    elif case == "lattice":
        pts, Lx, Ly = W.triangular_lattice(96, 96, 1.0, 1e-4, seed=4)
    else:
        pts, L = W.gaussian_mixture(65536, components=64, sigma=2.0, L=256.0, seed=9)
        Lx = Ly = L
    n = len(pts)
    out = {}
    for budget in (None, 0):
        d = _dg()(n, 32, 0.0 if case != "uniform" else 1.0, (Lx, Ly))
        if budget is not None:
            d.setWorkBudget(budget)
        P = torch.from_numpy(np.ascontiguousarray(pts)).cuda()
        tri = torch.zeros(32 * n, dtype=torch.int32, device="cuda")
        nn = torch.zeros(n, dtype=torch.int32, device="cuda")
        d.globalDelaunayTriangulation(P, tri, nn)
        st = d.stats()
        assert st["error_flags"] == 0, st
        if budget == 0:
            assert st["heavy_points"] == n and st["exact_points"] == n
        out[budget] = host(tri, nn)
        d.close()
    (t0, k0), (t1, k1) = out[None], out[0]
    assert np.array_equal(k0, k1)
    assert np.array_equal(O.canonical(t0, k0), O.canonical(t1, k1))
    assert_delaunay(pts, Lx, Ly, t1, k1, scan=(case != "mixture"))
    if case == "uniform":
        ref = O.restated_global(pts, Lx, Ly, 1.0, 32)
        assert np.array_equal(O.canonical(t1, k1), O.canonical(ref.tri, ref.nn)[:, :32])


def test_clustered_input_defers_only_long_scans():
    # 1M-point mixture layout at 1/16 size: rim points go to the warp-per-point kernel
    pts, L = W.gaussian_mixture(65536, components=64, sigma=2.0, L=256.0, seed=9)
    n = len(pts)
    d = _dg()(n, 32, 1.0, (L, L))
    P = torch.from_numpy(pts).cuda()
    tri = torch.zeros(32 * n, dtype=torch.int32, device="cuda")
    nn = torch.zeros(n, dtype=torch.int32, device="cuda")
    d.globalDelaunayTriangulation(P, tri, nn)
    st = d.stats()
    assert st["error_flags"] == 0 and 0 < st["heavy_points"] < n // 4, st
    t, k = host(tri, nn)
    assert_delaunay(pts, L, L, t, k, scan=False)


def test_box_too_small_is_flagged():
    # 16 tight clusters in a 200-wide box: void circles reach past L/2
    pts, L = W.gaussian_mixture(40000, components=16, sigma=2.0, seed=9)
    d, P, tri, nn = gpu_build(pts, L, L, 0.0, 16)
    assert d.stats()["error_flags"] & 32


def test_safety_mode_grows_stride():
    n = 5000
    L = float(np.sqrt(n))
    pts = W.uniform_points(n, L, 91)
    d, P, tri, nn = gpu_build(pts, L, L, 1.0, 4)   # 4 slots: every point overflows first
    t, k = host(tri, nn)
    assert d.MaxSize == int(k.max()) and t.shape[1] == d.MaxSize
    assert_delaunay(pts, L, L, t, k)


def test_no_safety_mode_raises_instead_of_truncating():
    from gpudelaunaytriangulation_b200 import _native as N

    n = 5000
    L = float(np.sqrt(n))
    pts = W.uniform_points(n, L, 92)
    d = _dg()(n, 5, 1.0, (L, L))
    P = torch.from_numpy(pts).cuda()
    tri = torch.zeros(5 * n, dtype=torch.int32, device="cuda")
    nn = torch.zeros(n, dtype=torch.int32, device="cuda")
    d.safetyMode = False   # python-side growth off, library still reports
    with pytest.raises(N.DgtError) as e:
        d.globalDelaunayTriangulation(P, tri, nn)
    assert e.value.code == N.DGT_ERR_NEED_RESIZE
    assert d.MaxSize > 5


def test_bad_points_rejected():
    from gpudelaunaytriangulation_b200 import _native as N

    n = 1000
    L = float(np.sqrt(n))
    pts = W.uniform_points(n, L, 93)
    pts[5, 0] = L   # outside [0, L)
    with pytest.raises(N.DgtError) as e:
        gpu_build(pts, L, L)
    assert e.value.code == N.DGT_ERR_BAD_POINTS


def test_batched_sets_match_per_set_oracle():
    from gpudelaunaytriangulation_b200.delaunay import DelaunayBatch

    pts, sizes, boxes = W.ensemble(12, 200, 5000, seed=13)
    b = DelaunayBatch(sizes, boxes, 16, 1.0)
    b.setCheckMode(True)
    P = torch.from_numpy(pts).cuda()
    tri, nn = b.globalDelaunayTriangulation(P)
    t, k = host(tri, nn)
    off = np.concatenate([[0], np.cumsum(sizes)])
    for s in range(len(sizes)):
        lo, hi = off[s], off[s + 1]
        ref = O.restated_global(pts[lo:hi], boxes[s][0], boxes[s][1], 1.0, 32)
        ts = t[lo:hi].copy()
        ts[np.arange(ts.shape[1])[None, :] < k[lo:hi, None]] -= lo
        assert np.array_equal(k[lo:hi], ref.nn)
        assert np.array_equal(O.canonical(ts, k[lo:hi])[:, :16], O.canonical(ref.tri, ref.nn)[:, :16])
    assert b.stats()["mismatches"] == 0
    # batched repair after a displacement of every set
    for step in range(2):
        b.displace(P, 0.01, seed=3, step=step)
        b.testAndRepairDelaunayTriangulation(P, tri, nn)
    cur = P.cpu().numpy()
    t, k = host(tri, nn)
    for s in range(len(sizes)):
        lo, hi = off[s], off[s + 1]
        ref = O.restated_global(cur[lo:hi], boxes[s][0], boxes[s][1], 1.0, 32)
        ts = t[lo:hi].copy()
        ts[np.arange(ts.shape[1])[None, :] < k[lo:hi, None]] -= lo
        assert np.array_equal(O.canonical(ts, k[lo:hi])[:, :16], O.canonical(ref.tri, ref.nn)[:, :16])


def test_batched_clustered_sets_through_warp_kernel_match_oracle():
    # clustered sets of different sizes and boxes in one batch, at a quarter of each set's
    # mean spacing and a small work budget: many points go to the warp-per-point kernel, whose
    # scans of the voids between clusters cross strips of thousands of cells and so are judged
    # on both occupancy levels (8 x 8-cell blocks and 64 x 64-cell super-blocks, the latter
    # filled per set from the block counts)
    from gpudelaunaytriangulation_b200.delaunay import DelaunayBatch

    # clusters ~32 units apart, as in the 1M-point workload (wider voids let circles pass half
    # the box, where the reference's minimum-image search itself fails)
    specs = [(32768, 32, 181.0, 33), (24000, 24, 156.0, 34), (32768, 32, 181.0, 36)]
    sets = [W.gaussian_mixture(n, components=c, sigma=2.0, L=L, seed=s) for n, c, L, s in specs]
    pts = np.concatenate([p for p, _ in sets], axis=0)
    sizes = np.array([len(p) for p, _ in sets])
    boxes = np.array([[L, L] for _, L in sets])
    b = DelaunayBatch(sizes, boxes, 32, 0.25)
    b.setWorkBudget(64)
    P = torch.from_numpy(pts).cuda()
    tri = torch.zeros(32 * len(pts), dtype=torch.int32, device="cuda")
    nn = torch.zeros(len(pts), dtype=torch.int32, device="cuda")
    b.globalDelaunayTriangulation(P, tri, nn)
    st = b.stats()
    assert st["error_flags"] == 0 and st["heavy_points"] > 1000, st
    t, k = host(tri, nn)
    off = np.concatenate([[0], np.cumsum(sizes)])
    for s in range(len(sizes)):
        lo, hi = off[s], off[s + 1]
        ref = O.restated_global(pts[lo:hi], boxes[s][0], boxes[s][1], 1.0, 32)
        ts = t[lo:hi].copy()
        ts[np.arange(ts.shape[1])[None, :] < k[lo:hi, None]] -= lo
        assert np.array_equal(k[lo:hi], ref.nn), s
        assert np.array_equal(O.canonical(ts, k[lo:hi]), O.canonical(ref.tri, ref.nn)[:, :32]), s
    b.close()


@pytest.mark.parametrize("n", [10000, 9000])
def test_square_lattice_input_matches_reference(n):
    # the reference driver's squareLattice input (jittered square lattice, near-cocircular
    # squares; 9000 leaves the last column partly empty), build and one repair
    pts, L = W.square_lattice(n, seed=11)
    d, P, tri, nn = gpu_build(pts, L, L, 1.0, 16, True, check=True)
    st = d.stats()
    assert st["error_flags"] == 0 and st["mismatches"] == 0, st
    t, k = host(tri, nn)
    ref = O.restated_global(pts, L, L, 1.0, 32)
    assert np.array_equal(k, ref.nn)
    assert np.array_equal(O.canonical(t, k)[:, :16], O.canonical(ref.tri, ref.nn)[:, :16])
    moved = W.displace(pts, 0.05, L, L, 12)
    P.copy_(torch.from_numpy(moved))
    d.testAndRepairDelaunayTriangulation(P, tri, nn)
    t, k = host(tri, nn)
    ref = O.restated_global(moved, L, L, 1.0, 32)
    assert np.array_equal(k, ref.nn)
    assert np.array_equal(O.canonical(t, k)[:, :16], O.canonical(ref.tri, ref.nn)[:, :16])


def test_deferred_overlap_same_rings():
    # the global build in 1, 2, 3 or 8 pieces, each piece's deferred points rebuilt on a stream
    # of their own while the next pieces build: the same rings as the restated reference, with
    # many points deferred (clustered input, fine cells, small work budget)
    pts, L = W.gaussian_mixture(65536, components=64, sigma=2.0, L=256.0, seed=9)
    n = len(pts)
    ref = O.restated_global(pts, L, L, 1.0, 32)
    P = torch.from_numpy(pts).cuda()
    for chunks in (1, 2, 3, 8):
        d = _dg()(n, 32, 0.25 * L / np.sqrt(n), (L, L))
        d.setWorkBudget(64)
        d.setDeferredOverlap(chunks)
        tri = torch.zeros(32 * n, dtype=torch.int32, device="cuda")
        nn = torch.zeros(n, dtype=torch.int32, device="cuda")
        for _ in range(2):
            d.globalDelaunayTriangulation(P, tri, nn)
        st = d.stats()
        assert st["error_flags"] == 0 and st["exact_points"] > 1000, (chunks, st)
        t, k = host(tri, nn)
        assert np.array_equal(k, ref.nn), chunks
        assert np.array_equal(O.canonical(t, k), O.canonical(ref.tri, ref.nn)), chunks
        for bad in (0, 9):
            with pytest.raises(N.DgtError):
                d.setDeferredOverlap(bad)
        d.close()


def test_million_points_properties():
    n = 1_000_000
    L = 1000.0
    pts = W.uniform_points(n, L, 101)
    d, P, tri, nn = gpu_build(pts, L, L, 1.0, 16)
    t, k = host(tri, nn)
    assert int(k.sum()) == 6 * n
    assert_delaunay(pts, L, L, t, k, scan=False)
    moved = W.displace(pts, 0.02, L, L, 102)
    P.copy_(torch.from_numpy(moved))
    d.testAndRepairDelaunayTriangulation(P, tri, nn)
    t, k = host(tri, nn)
    assert int(k.sum()) == 6 * n
    assert_delaunay(moved, L, L, t, k, scan=False)


def test_every_kernel_shape_same_output():
    n = 60000
    L = float(np.sqrt(n))
    pts = W.uniform_points(n, L, 111)
    ref = O.restated_global(pts, L, L, 1.0, 32)
    for shape in range(N.KERNEL_SHAPES):
        d = _dg()(n, 16, 1.0, (L, L))
        d.setKernelShape(shape)
        P = torch.from_numpy(pts).cuda()
        tri, nn = d.globalDelaunayTriangulation(P)
        t, k = host(tri, nn)
        assert np.array_equal(k, ref.nn), shape
        assert np.array_equal(O.canonical(t, k)[:, :16], O.canonical(ref.tri, ref.nn)[:, :16]), shape


def test_autotune_result_is_correct_and_cached():
    n = 100000
    L = float(np.sqrt(n))
    pts = W.uniform_points(n, L, 112)
    d = _dg()(n, 16, 1.0, (L, L))
    P = torch.from_numpy(pts).cuda()
    tri = torch.zeros(16 * n, dtype=torch.int32, device="cuda")
    nn = torch.zeros(n, dtype=torch.int32, device="cuda")
    res = d.autotune(P, tri, nn)
    assert res["trials"] >= 5 and 0 <= res["shape"] < N.KERNEL_SHAPES and res["best_ms"] <= res["default_ms"] * 1.05
    t, k = host(tri, nn)
    assert_delaunay(pts, L, L, t, k, scan=False)
    d2 = _dg()(n, 16, 1.0, (L, L))
    res2 = d2.autotune(P, tri, nn)
    assert res2["from_cache"] == 1 and res2["shape"] == res["shape"]
