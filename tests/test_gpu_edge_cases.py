"""Edge cases of the point sets: empty sets, sets too small to close a ring, batches mixing
empty and tiny sets with normal ones, and coordinates on the box edges.  Results are checked
against the oracle (restated reference and exact verifier) where a triangulation exists,
and as clean error codes where it does not."""
import numpy as np
import pytest

from gpudelaunaytriangulation_b200 import _native as N
from gpudelaunaytriangulation_b200 import workloads as W
from oracle import oracle as O

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu


def _dg():
    from gpudelaunaytriangulation_b200.delaunay import DelaunayBatch, DelaunayGPU

    return DelaunayGPU, DelaunayBatch


def test_empty_set_is_a_no_op():
    DelaunayGPU, _ = _dg()
    d = DelaunayGPU(0, 16, 1.0, (10.0, 10.0))
    P = torch.zeros((0, 2), dtype=torch.float64, device="cuda")
    tri, nn = d.globalDelaunayTriangulation(P)
    assert nn.numel() == 0
    d.testAndRepairDelaunayTriangulation(P, tri, nn)
    assert d.validate(P, tri, nn)["valid"] == 1


@pytest.mark.parametrize("n", [1, 2, 3])
def test_too_few_points_report_an_error_and_leave_the_library_usable(n):
    # a ring needs three distinct neighbours; the minimum image of 1-3 points cannot close one
    DelaunayGPU, _ = _dg()
    L = float(np.sqrt(n)) + 1.0
    pts = W.uniform_points(n, L, 90 + n)
    d = DelaunayGPU(n, 16, 1.0, (L, L))
    P = torch.from_numpy(pts).cuda()
    with pytest.raises(N.DgtError) as e:
        d.globalDelaunayTriangulation(P)
    assert e.value.code == N.DGT_ERR_DEGENERATE
    # the device is still fine: a normal set right after
    m = 5000
    Lm = float(np.sqrt(m))
    q = W.uniform_points(m, Lm, 95)
    d2 = DelaunayGPU(m, 16, 1.0, (Lm, Lm))
    Q = torch.from_numpy(q).cuda()
    tri, nn = d2.globalDelaunayTriangulation(Q)
    assert d2.validate(Q, tri, nn)["valid"] == 1


@pytest.mark.parametrize("pieces", [1, 8])
def test_batch_with_empty_and_tiny_sets(pieces):
    # pieces > 1: the global build split into pieces of the cell order that straddle the sets
    _, DelaunayBatch = _dg()
    sizes = np.array([0, 500, 0, 2000, 40], dtype=np.int64)
    boxes = np.stack([np.sqrt(np.maximum(sizes, 1).astype(np.float64))] * 2, axis=1)
    pts = np.concatenate([W.uniform_points(int(n), float(L), 300 + s)
                          for s, (n, L) in enumerate(zip(sizes, boxes[:, 0])) if n > 0])
    b = DelaunayBatch(sizes, boxes, 16, 1.0)
    b.setDeferredOverlap(pieces)
    P = torch.from_numpy(pts).cuda()
    tri, nn = b.globalDelaunayTriangulation(P)
    t = tri.view(len(pts), -1).cpu().numpy()
    k = nn.cpu().numpy()
    off = np.concatenate([[0], np.cumsum(sizes)])
    for s in range(len(sizes)):
        lo, hi = off[s], off[s + 1]
        if hi == lo:
            continue
        ref = O.restated_global(pts[lo:hi], boxes[s][0], boxes[s][1], 1.0, 32)
        ts = t[lo:hi].copy()
        ts[np.arange(ts.shape[1])[None, :] < k[lo:hi, None]] -= lo
        assert np.array_equal(k[lo:hi], ref.nn), s
        assert np.array_equal(O.canonical(ts, k[lo:hi])[:, : t.shape[1]],
                              O.canonical(ref.tri, ref.nn)[:, : t.shape[1]]), s


def test_few_points_in_many_pieces():
    # 40 points in 8 pieces of 5 and 12 points in 8 pieces of 2 (the pieces past the last
    # point are not launched): the same rings as in one piece, and the restated reference's
    DelaunayGPU, _ = _dg()
    for n, L, seed in ((40, 5.0, 3), (12, float(np.sqrt(12)), 93)):
        pts = W.uniform_points(n, L, seed)
        P = torch.from_numpy(pts).cuda()
        out = []
        for pieces in (1, 8):
            d = DelaunayGPU(n, 16, 1.0, (L, L))
            d.setDeferredOverlap(pieces)
            tri, nn = d.globalDelaunayTriangulation(P)
            out.append((tri.view(n, -1).cpu().numpy(), nn.cpu().numpy()))
            d.close()
        assert np.array_equal(out[0][1], out[1][1]) and np.array_equal(out[0][0], out[1][0]), n
        assert (out[1][1] >= 3).all()
        if n == 40:
            ref = O.restated_global(pts, L, L, 1.0, 32)
            t, k = out[1]
            assert np.array_equal(k, ref.nn)
            assert np.array_equal(O.canonical(t, k)[:, :16], O.canonical(ref.tri, ref.nn)[:, :16])


def test_coordinates_on_the_box_edges():
    # x = 0 and y = 0 exactly, and coordinates one ulp below L: valid, equal to the oracle
    DelaunayGPU, _ = _dg()
    n = 4000
    L = float(np.sqrt(n))
    pts = W.uniform_points(n, L, 97)
    pts[:20, 0] = 0.0
    pts[20:40, 1] = 0.0
    pts[40:60, 0] = np.nextafter(L, 0.0)
    pts[60:80, 1] = np.nextafter(L, 0.0)
    d = DelaunayGPU(n, 16, 1.0, (L, L))
    P = torch.from_numpy(pts).cuda()
    tri, nn = d.globalDelaunayTriangulation(P)
    assert d.validate(P, tri, nn)["valid"] == 1
    t = tri.view(n, -1).cpu().numpy()
    k = nn.cpu().numpy()
    ok, rep = O.verify(pts, L, L, t, k)
    assert ok, rep
    ref = O.restated_global(pts, L, L, 1.0, 32)
    assert np.array_equal(O.canonical(t, k)[:, :16], O.canonical(ref.tri, ref.nn)[:, :16])


def test_largest_single_set_and_repair():
    # 2^24 points (4x the largest benchmark set): index arithmetic and grid sizes past 2^24
    # cells; checked on the device (validator) and by the ring-size sum, which is 6N exactly
    # on the torus
    DelaunayGPU, _ = _dg()
    n = 1 << 24
    L = float(np.sqrt(n))
    g = torch.Generator(device="cuda").manual_seed(77)
    P = torch.rand((n, 2), generator=g, device="cuda", dtype=torch.float64) * L
    d = DelaunayGPU(n, 16, 1.0, (L, L))
    tri, nn = d.globalDelaunayTriangulation(P)
    st = d.stats()
    assert st["error_flags"] == 0 and st["mismatches"] == 0
    assert int(nn.sum().item()) == 6 * n
    assert d.validate(P, tri, nn)["valid"] == 1
    P.add_(torch.randn((n, 2), generator=g, device="cuda", dtype=torch.float64), alpha=0.02)
    P.remainder_(L)
    P.masked_fill_(P >= L, 0.0)   # a tiny negative coordinate plus L rounds to L
    d.testAndRepairDelaunayTriangulation(P, tri, nn)
    assert d.stats()["error_flags"] == 0
    assert d.validate(P, tri, nn)["valid"] == 1
