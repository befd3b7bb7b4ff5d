"""Device-only MD steps on a batched ensemble: displacement + fixed-round repair, directly
and replayed from a captured CUDA graph; every set's rings must equal a fresh oracle
triangulation of the displaced points."""
import numpy as np
import pytest

from gpudelaunaytriangulation_b200 import workloads as W
from oracle import oracle as O

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu


def check_sets(P, tri, nn, sizes, boxes):
    cur = P.cpu().numpy()
    n = nn.numel()
    t = tri.view(n, -1).cpu().numpy()
    k = nn.cpu().numpy()
    off = np.concatenate([[0], np.cumsum(sizes)])
    for s in range(len(sizes)):
        lo, hi = off[s], off[s + 1]
        ref = O.restated_global(cur[lo:hi], boxes[s][0], boxes[s][1], 1.0, 32)
        ts = t[lo:hi].copy()
        ts[np.arange(ts.shape[1])[None, :] < k[lo:hi, None]] -= lo
        assert np.array_equal(k[lo:hi], ref.nn), s
        assert np.array_equal(O.canonical(ts, k[lo:hi])[:, : t.shape[1]],
                              O.canonical(ref.tri, ref.nn)[:, : t.shape[1]]), s


def setup(num_sets=10, lo=500, hi=8000, seed=21):
    from gpudelaunaytriangulation_b200.delaunay import DelaunayBatch

    pts, sizes, boxes = W.ensemble(num_sets, lo, hi, seed=seed)
    b = DelaunayBatch(sizes, boxes, 16, 1.0)
    P = torch.from_numpy(pts).cuda()
    tri, nn = b.globalDelaunayTriangulation(P)
    return b, P, tri, nn, sizes, boxes


def test_md_steps_without_graph():
    b, P, tri, nn, sizes, boxes = setup()
    for _ in range(3):
        b.mdStep(P, tri, nn, 0.01, seed=5, rounds=4)
    torch.cuda.synchronize()
    st = b.stats()
    assert st["sticky_flags"] == 0 and st["md_step"] == 3
    check_sets(P, tri, nn, sizes, boxes)


@pytest.mark.parametrize("flip_rounds", [0, 6])
def test_md_steps_with_other_flip_round_counts(flip_rounds):
    # every flagged edge rebuilt (0 flip rounds) or flipped longer (6): same triangulation
    b, P, tri, nn, sizes, boxes = setup(seed=22)
    b.setGraphFlipRounds(flip_rounds)
    for _ in range(3):
        b.mdStep(P, tri, nn, 0.03, seed=6, rounds=6)
    torch.cuda.synchronize()
    assert b.stats()["sticky_flags"] == 0
    check_sets(P, tri, nn, sizes, boxes)


def test_md_graph_replays_fresh_noise_and_matches_oracle():
    b, P, tri, nn, sizes, boxes = setup(seed=22)
    stream = torch.cuda.Stream()
    with torch.cuda.stream(stream):
        g = b.mdGraph(P, tri, nn, 0.01, seed=9, steps=4, rounds=4, stream=stream)
        before = P.clone()
        g.launch(stream)
        stream.synchronize()
        mid = P.clone()
        g.launch(stream)
        stream.synchronize()
    assert not torch.equal(before, mid) and not torch.equal(mid, P)
    st = b.stats()
    assert st["sticky_flags"] == 0 and st["md_step"] == 8 and st["repair_calls"] == 8
    check_sets(P, tri, nn, sizes, boxes)
    g.close()


def test_unfinished_repair_is_flagged_not_hidden():
    # one round only and a large move: the queue cannot drain, the device flag must say so
    b, P, tri, nn, sizes, boxes = setup(num_sets=3, lo=2000, hi=4000, seed=23)
    b.mdStep(P, tri, nn, 0.3, seed=1, rounds=1)
    torch.cuda.synchronize()
    assert b.stats()["sticky_flags"] & 64


def test_fused_md_step_equals_displacement_then_repair():
    # dgt_md_step moves the points inside the repair call (one kernel: move, wrap, distance
    # outside the listing cell); a separate dgt_displace followed by test-and-repair must
    # give the same positions and the same rings, step after step
    b1, P1, tri1, nn1, sizes, boxes = setup(num_sets=6, lo=1000, hi=6000, seed=24)
    b2, P2, tri2, nn2, _, _ = setup(num_sets=6, lo=1000, hi=6000, seed=24)
    for step in range(4):
        b1.mdStep(P1, tri1, nn1, 0.02, seed=11, rounds=6)
        b2.displace(P2, 0.02, seed=11, step=step)
        b2.testAndRepairDelaunayTriangulation(P2, tri2, nn2)
        torch.cuda.synchronize()
        assert torch.equal(P1, P2), step
        assert torch.equal(nn1, nn2), step
    assert b1.stats()["sticky_flags"] == 0 and b1.stats()["md_step"] == 4
    check_sets(P1, tri1, nn1, sizes, boxes)
    n = nn1.numel()
    t1 = tri1.view(n, -1).cpu().numpy()
    t2 = tri2.view(n, -1).cpu().numpy()
    k = nn1.cpu().numpy()
    assert np.array_equal(O.canonical(t1, k), O.canonical(t2, k))
