"""The allocation-free global triangulation (dgt_global_triangulation_noalloc).

It serves callers that cannot call cudaMalloc (the GPU allocator belongs to a host
application, or the memory budget is fixed before the library loads): all its scratch is a
fixed device array inside the library.  Here it must give exactly the rings and ring
lengths of the regular entry point and of the oracle (integer output, so the bar is
equality), on two calls in a row with different sets -- the second call starts from
whatever the first left in the shared array -- leave the device's free memory unchanged
across a call, and refuse inputs beyond its fixed size (points, or a grid too wide for its
cell array) without writing.  This file is collected last on purpose (file name) and needs
nothing from other tests.
"""
import ctypes

import numpy as np
import pytest

from gpudelaunaytriangulation_b200 import _native as N
from gpudelaunaytriangulation_b200 import workloads as W
from oracle import oracle as O

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu


def _vp(t):
    return ctypes.c_void_p(t.data_ptr())


def call(P, tri, nn, n, Lx, Ly, stride, cell=1.0):
    """One call through the C ABI on tensors the caller already holds; returns (code, stride needed)."""
    need = ctypes.c_int(-1)
    stream = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    code = N.lib().dgt_global_triangulation_noalloc(_vp(P), n, Lx, Ly, cell, _vp(tri), _vp(nn), stride,
                                                     ctypes.byref(need), stream)
    torch.cuda.synchronize()
    return code, need.value


def buffers(pts, stride):
    n = len(pts)
    P = torch.from_numpy(np.ascontiguousarray(pts)).cuda()
    tri = torch.full((max(n, 1) * stride,), -7, dtype=torch.int32, device="cuda")
    nn = torch.full((max(n, 1),), -7, dtype=torch.int32, device="cuda")
    return P, tri, nn


def noalloc(pts, L, stride=16, cell=1.0, Ly=None):
    n = len(pts)
    P, tri, nn = buffers(pts, stride)
    code, need = call(P, tri, nn, n, L, L if Ly is None else Ly, stride, cell)
    return code, tri.view(-1, stride).cpu().numpy(), nn.cpu().numpy(), need


def with_context(pts, L, stride=16, cell=1.0):
    from gpudelaunaytriangulation_b200.delaunay import DelaunayGPU

    n = len(pts)
    d = DelaunayGPU(n, stride, cell, (L, L))
    P = torch.from_numpy(np.ascontiguousarray(pts)).cuda()
    tri = torch.zeros(n * stride, dtype=torch.int32, device="cuda")
    nn = torch.zeros(n, dtype=torch.int32, device="cuda")
    d.globalDelaunayTriangulation(P, tri, nn)
    torch.cuda.synchronize()
    out = tri.view(n, -1).cpu().numpy(), nn.cpu().numpy()
    d.close()
    return out


def same_rings(a_tri, a_nn, b_tri, b_nn):
    if not np.array_equal(a_nn, b_nn):
        return False
    w = int(a_nn.max())
    cols = np.arange(w)[None, :]
    return np.array_equal(np.where(cols < a_nn[:, None], a_tri[:, :w], -1),
                          np.where(cols < b_nn[:, None], b_tri[:, :w], -1))


def test_noalloc_matches_regular_entry_point_twice_in_a_row():
    cases = [(60000, 11), (20000, 12)]   # second call: smaller set on the leftovers of the first
    for n, seed in cases:
        L = float(np.sqrt(n))
        pts = W.uniform_points(n, L, seed)
        code, t, k, need = noalloc(pts, L)
        assert code == N.DGT_OK, N.lib().dgt_error_string(code)
        rt, rk = with_context(pts, L)
        assert same_rings(t, k, rt, rk)
        assert int(k.sum()) == 6 * n


def test_noalloc_matches_oracle_and_allocates_nothing():
    # the first call sets up (loads the library's kernels and the array on this device); the
    # second, identical call must leave the device's free memory exactly where it was
    n = 50000
    L = float(np.sqrt(n))
    pts = W.uniform_points(n, L, 15)
    P, tri, nn = buffers(pts, 16)
    code, _ = call(P, tri, nn, n, L, L, 16)
    assert code == N.DGT_OK, N.lib().dgt_error_string(code)
    first = tri.view(n, 16).cpu().numpy().copy(), nn.cpu().numpy().copy()
    tri.fill_(-7)
    nn.fill_(-7)
    torch.cuda.synchronize()
    free_before = torch.cuda.mem_get_info()[0]
    code, _ = call(P, tri, nn, n, L, L, 16)
    free_after = torch.cuda.mem_get_info()[0]
    assert code == N.DGT_OK
    assert free_after == free_before, (free_before, free_after)
    t, k = tri.view(n, 16).cpu().numpy(), nn.cpu().numpy()
    assert same_rings(t, k, *first)
    ref = O.restated_global(pts, L, L, 1.0, 32)
    assert np.array_equal(k, ref.nn)
    assert np.array_equal(O.canonical(t, k)[:, :16], O.canonical(ref.tri, ref.nn)[:, :16])


def test_noalloc_small_grid_then_larger_grid():
    # the second call's grid is larger than the first's: every count it reads must have been
    # cleared by the call itself, not left from the first
    for n, seed in [(3000, 16), (65536, 17)]:
        L = float(np.sqrt(n))
        pts = W.uniform_points(n, L, seed)
        code, t, k, _ = noalloc(pts, L, cell=0.5)
        assert code == N.DGT_OK, N.lib().dgt_error_string(code)
        rt, rk = with_context(pts, L)
        assert same_rings(t, k, rt, rk)


def test_noalloc_empty_input_is_a_no_op():
    pts = np.zeros((0, 2), np.float64)
    code, t, k, need = noalloc(pts, 10.0)
    assert code == N.DGT_OK and need == 0
    assert (k == -7).all() and (t == -7).all()


@pytest.mark.parametrize("Lx,Ly", [(1.0e6, 0.01), (1.0e12, 1.0e-9)], ids=["wide", "int_overflow"])
def test_noalloc_rejects_grid_beyond_its_cell_array(Lx, Ly):
    # a box of extreme aspect ratio asks for more cells along x than the array holds (the
    # second case for more than an int holds): refused before any work, nothing written
    n = 1000
    u = W.splitmix64_uniform(18, 2 * n).reshape(n, 2)
    pts = np.stack([u[:, 0] * Lx, u[:, 1] * Ly], axis=1)
    code, t, k, need = noalloc(pts, Lx, Ly=Ly)
    assert code == N.DGT_ERR_INVALID_ARGUMENT
    assert (k == -7).all() and (t == -7).all()


def test_noalloc_rejects_oversized_input_without_writing():
    n = N.NOALLOC_MAX_POINTS + 1
    L = float(np.sqrt(n))
    pts = W.uniform_points(n, L, 13)
    code, t, k, need = noalloc(pts, L)
    assert code == N.DGT_ERR_INVALID_ARGUMENT
    assert (k == -7).all() and (t == -7).all()


def test_noalloc_reports_required_stride():
    n = 5000
    L = float(np.sqrt(n))
    pts = W.uniform_points(n, L, 14)
    code, t, k, need = noalloc(pts, L, stride=5)
    assert code == N.DGT_ERR_NEED_RESIZE and need > 5
    code, t, k, _ = noalloc(pts, L, stride=need)
    assert code == N.DGT_OK
    rt, rk = with_context(pts, L, stride=need)
    assert same_rings(t, k, rt, rk)
