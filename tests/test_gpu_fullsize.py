"""Ring-for-ring parity at the benchmarked sizes: every workload that bench.py times is
compared here, at its full size and with its own seeds and settings, against the C
restatement of the reference (oracle/dgt_oracle.c, pinned raw-identical to the reference's
own output by tests/test_oracle.py) -- the comparison the reference makes itself with
compareTriangulation (triangulation.cpp:91-143: rings rotated to a common start, then
compared entry by entry).

- 4,194,304 uniform points, L = 2048: the build (float32 filter, and float64 plain), then
  one test-and-repair after a sigma = 0.02 displacement, against the reference's own repair
  sequence (triangle test + local rebuild, DelaunayGPU.cpp:567-602) run on the oracle's
  build.
- 1,000,000 uniform points, L = 1000, float64 predicates: 20 device displacements
  (sigma = 0.02) each followed by test-and-repair, compared after every step against the
  reference's repair of its own previous state.
- 1,048,576-site jittered triangular lattice (rectangular box) and 1,048,576-point
  64-cluster Gaussian mixture, both at their autotuned settings.  The lattice oracle runs at
  cell size 0.5, where the reference's square-cell binning of a rectangular box stays in
  range (at 1.0 it clamps y bins with the x count, cellListGPU.cu:41-42).
- 256 independent sets (sizes log-uniform in [1000, 65536]), autotuned, built in one
  launch sequence, then 100 MD steps (sigma = 0.01) replayed from a captured CUDA graph;
  every set compared after the build and after the 100 steps.

Integer output: the bar is equality.  The oracle is test infrastructure only."""
import numpy as np
import pytest

from gpudelaunaytriangulation_b200 import workloads as W
from oracle import oracle as O

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu


def _dg():
    from gpudelaunaytriangulation_b200.delaunay import DelaunayGPU

    return DelaunayGPU


def host(tri, nn):
    n = nn.numel()
    return tri.view(n, -1).cpu().numpy(), nn.cpu().numpy()


def assert_same_rings(t, k, ref, what=""):
    """Ring lengths equal and every ring equal after rotation to its smallest index."""
    assert np.array_equal(k, ref.nn), (what, int((k != ref.nn).sum()))
    w = max(t.shape[1], ref.tri.shape[1])
    a = np.full((len(k), w), -1, np.int32)
    b = np.full((len(k), w), -1, np.int32)
    a[:, : t.shape[1]] = O.canonical(t, k)
    b[:, : ref.tri.shape[1]] = O.canonical(ref.tri, ref.nn)
    bad = np.nonzero((a != b).any(axis=1))[0]
    assert len(bad) == 0, (what, len(bad), bad[:8].tolist())


def test_build_repair_4m_matches_reference_ring_for_ring():
    # bench.py's headline workload: same points (seed 2026), same displacement (seed 2027)
    n, L = 4_194_304, 2048.0
    p0 = W.uniform_points(n, L, 2026)
    p1 = W.displace(p0, 0.02, L, L, 2027)
    d = _dg()(n, 16, 1.0, (L, L))
    d.setCheckMode(True)
    P = torch.from_numpy(p0).cuda()
    tri, nn = d.globalDelaunayTriangulation(P)
    st = d.stats()
    assert st["mismatches"] == 0 and st["error_flags"] == 0, st
    t, k = host(tri, nn)
    ref0 = O.restated_global(p0, L, L, 1.0, 24)
    assert_same_rings(t, k, ref0, "build")
    # float64-plain predicates give the same rings
    d64 = _dg()(n, 16, 1.0, (L, L))
    d64.setPrecision(False)
    tri64, nn64 = d64.globalDelaunayTriangulation(P)
    assert torch.equal(nn64, nn) and torch.equal(tri64, tri)
    d64.close()
    # one repair step against the reference's repair of its own build
    P.copy_(torch.from_numpy(p1))
    d.testAndRepairDelaunayTriangulation(P, tri, nn)
    st = d.stats()
    assert st["mismatches"] == 0 and st["error_flags"] == 0, st
    t, k = host(tri, nn)
    ref1, flags = O.restated_test_and_repair(p1, L, L, ref0, 1.0)
    assert (flags >= 0).sum() > 0
    assert_same_rings(t, k, ref1, "repair")
    d.close()


def test_uniform_1m_fp64_twenty_repair_steps_match_reference_chain():
    # bench.py's 1M float64 configuration: points seed 31, device displacement seed 32
    n, L = 1_000_000, 1000.0
    pts = W.uniform_points(n, L, 31)
    d = _dg()(n, 16, 1.0, (L, L))
    d.setPrecision(False)
    P = torch.from_numpy(pts).cuda()
    tri, nn = d.globalDelaunayTriangulation(P)
    ref = O.restated_global(pts, L, L, 1.0, 24)
    t, k = host(tri, nn)
    assert_same_rings(t, k, ref, "build")
    for step in range(20):
        d.displace(P, 0.02, seed=32, step=step)
        d.testAndRepairDelaunayTriangulation(P, tri, nn)
        st = d.stats()
        assert st["error_flags"] == 0, (step, st)
        cur = P.cpu().numpy()
        assert (cur >= 0).all() and (cur[:, 0] < L).all() and (cur[:, 1] < L).all()
        ref, _ = O.restated_test_and_repair(cur, L, L, ref, 1.0)
        t, k = host(tri, nn)
        assert_same_rings(t, k, ref, f"step {step}")
    assert_same_rings(t, k, O.restated_global(cur, L, L, 1.0, 24), "fresh after 20 steps")
    d.close()


def test_lattice_1m_autotuned_matches_reference():
    pts, Lx, Ly = W.triangular_lattice(1024, 1024, 1.0, 1e-4, seed=3)
    n = len(pts)
    d = _dg()(n, 16, 0.0, (Lx, Ly))
    P = torch.from_numpy(pts).cuda()
    tri = torch.zeros(16 * n, dtype=torch.int32, device="cuda")
    nn = torch.zeros(n, dtype=torch.int32, device="cuda")
    d.autotune(P, tri, nn)
    d.setCheckMode(True)
    d.globalDelaunayTriangulation(P, tri, nn)
    st = d.stats()
    assert st["mismatches"] == 0 and st["error_flags"] == 0, st
    t, k = host(tri, nn)
    ref = O.restated_global(pts, Lx, Ly, 0.5, 24)
    assert_same_rings(t, k, ref, "lattice")
    ok, rep = O.verify(pts, Lx, Ly, t, k, global_scan=True)
    assert ok and rep["sum_deg"] == 6 * n, rep
    d.close()


def test_mixture_1m_autotuned_matches_reference():
    # 64 Gaussian clusters (sigma 2) in a 1024 box: 20x density contrast, rings up to 19
    pts, L = W.gaussian_mixture(1 << 20, components=64, sigma=2.0, L=1024.0, seed=5)
    n = len(pts)
    d = _dg()(n, 16, 0.0, (L, L))
    P = torch.from_numpy(pts).cuda()
    tri = torch.zeros(16 * n, dtype=torch.int32, device="cuda")
    nn = torch.zeros(n, dtype=torch.int32, device="cuda")
    tune = d.autotune(P, tri, nn)
    d.setCheckMode(True)
    tri, nn = d.globalDelaunayTriangulation(P, tri, nn)
    st = d.stats()
    assert st["mismatches"] == 0 and st["error_flags"] == 0, (st, tune)
    t, k = host(tri, nn)
    ref = O.restated_global(pts, L, L, 1.0, 24)
    assert_same_rings(t, k, ref, "mixture")
    d.close()


def _check_sets(P, tri, nn, sizes, boxes, what):
    cur = P.cpu().numpy()
    n = nn.numel()
    t = tri.view(n, -1).cpu().numpy()
    k = nn.cpu().numpy()
    off = np.concatenate([[0], np.cumsum(sizes)])
    for s in range(len(sizes)):
        lo, hi = off[s], off[s + 1]
        ref = O.restated_global(cur[lo:hi], boxes[s][0], boxes[s][1], 1.0, 24)
        ts = t[lo:hi].copy()
        ts[np.arange(ts.shape[1])[None, :] < k[lo:hi, None]] -= lo
        assert_same_rings(ts, k[lo:hi], ref, f"{what}: set {s}")


def test_ensemble_256_sets_100_graph_steps_match_reference():
    # bench.py's batched ensemble: 256 sets (seed 7), autotuned, graph of 10 steps replayed
    # 10 times, sigma 0.01, 4 repair rounds per step
    from gpudelaunaytriangulation_b200.delaunay import DelaunayBatch

    pts, sizes, boxes = W.ensemble(256, 1000, 65536, seed=7)
    n = len(pts)
    b = DelaunayBatch(sizes, boxes, 16, 1.0)
    P = torch.from_numpy(pts).cuda()
    tri = torch.zeros(16 * n, dtype=torch.int32, device="cuda")
    nn = torch.zeros(n, dtype=torch.int32, device="cuda")
    b.autotune(P, tri, nn)
    P.copy_(torch.from_numpy(pts))
    b.globalDelaunayTriangulation(P, tri, nn)
    _check_sets(P, tri, nn, sizes, boxes, "build")
    stream = torch.cuda.Stream()
    stream.wait_stream(torch.cuda.current_stream())
    with torch.cuda.stream(stream):
        g = b.mdGraph(P, tri, nn, 0.01, seed=8, steps=10, rounds=4, stream=stream)
        for _ in range(10):
            g.launch(stream)
        stream.synchronize()
    st = b.stats()
    assert st["sticky_flags"] == 0 and st["md_step"] == 100, st
    g.close()
    _check_sets(P, tri, nn, sizes, boxes, "after 100 steps")
    b.close()
