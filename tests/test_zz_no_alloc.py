"""The allocation-free global triangulation (dgt_global_triangulation_noalloc).

It serves callers that cannot call cudaMalloc (the GPU allocator belongs to a host
application, or the memory budget is fixed before the library loads): all its scratch is a
fixed device array inside the library.  Here it must give exactly the rings and ring
lengths of the regular entry point (integer output, so the bar is equality), on two calls
in a row with different sets -- the second call starts from whatever the first left in
the shared array -- and it must refuse inputs beyond its fixed size without writing.
This file is collected last on purpose (file name) and needs nothing from other tests.
"""
import ctypes

import numpy as np
import pytest

from gpudelaunaytriangulation_b200 import _native as N
from gpudelaunaytriangulation_b200 import workloads as W

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu


def _vp(t):
    return ctypes.c_void_p(t.data_ptr())


def noalloc(pts, L, stride=16, cell=1.0):
    n = len(pts)
    P = torch.from_numpy(np.ascontiguousarray(pts)).cuda()
    tri = torch.full((n * stride,), -7, dtype=torch.int32, device="cuda")
    nn = torch.full((n,), -7, dtype=torch.int32, device="cuda")
    need = ctypes.c_int(-1)
    stream = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    code = N.lib().dgt_global_triangulation_noalloc(_vp(P), n, L, L, cell, _vp(tri), _vp(nn), stride,
                                                     ctypes.byref(need), stream)
    torch.cuda.synchronize()
    return code, tri.view(n, stride).cpu().numpy(), nn.cpu().numpy(), need.value


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
