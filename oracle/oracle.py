"""ctypes front end of the CPU oracle -- TEST INFRASTRUCTURE ONLY.

Only tests/, ``__graft_entry__.smoke()`` and bench.py's CPU-baseline / reference legs import
this module.  It wraps

- ``oracle/liboracle.so`` (``dgt_oracle.c``): a C restatement of the reference's CPU path
  (src/model/DelaunayGPU.cu:318-608, :680-943, :192-284; src/model/DelaunayGPU.cpp:118-157,
  :567-602, :673-705; src/utilities/cellListGPU.cpp:97-117, :289-330) and an independent
  exact-arithmetic Delaunay verifier;
- ``oracle/_ref/libdgtref.so`` (``ref_harness.cu`` linked with the reference's own sources):
  the reference itself, run through its CPU/OpenMP callers (no device needed) or through its
  public ``DelaunayGPU`` class (needs a device).
"""
from __future__ import annotations

import ctypes
import os
import subprocess
from dataclasses import dataclass

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))


def reference_dir() -> str:
    """The reference project's sources: $DGT_REFERENCE_DIR, else a checkout named
    ``reference`` beside this repository."""
    return os.environ.get("DGT_REFERENCE_DIR") or os.path.join(os.path.dirname(os.path.dirname(HERE)), "reference")


LIB_PATH = os.path.join(HERE, "liboracle.so")
REF_PATH = os.path.join(HERE, "_ref", "libdgtref.so")

_P_D = ctypes.POINTER(ctypes.c_double)
_P_I = ctypes.POINTER(ctypes.c_int)


class OrcReport(ctypes.Structure):
    _fields_ = [
        ("sum_deg", ctypes.c_longlong),
        ("bad_index", ctypes.c_longlong),
        ("asym", ctypes.c_longlong),
        ("nonpositive", ctypes.c_longlong),
        ("winding", ctypes.c_longlong),
        ("not_local_dt", ctypes.c_longlong),
        ("circle_intruders", ctypes.c_longlong),
        ("triangles", ctypes.c_longlong),
        ("min_deg", ctypes.c_int),
        ("max_deg", ctypes.c_int),
    ]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


def build(force: bool = False) -> str:
    """Compile liboracle.so with the Makefile next to this file (gcc; seconds)."""
    if force or not os.path.exists(LIB_PATH) or os.path.getmtime(LIB_PATH) < os.path.getmtime(
        os.path.join(HERE, "dgt_oracle.c")
    ):
        subprocess.run(["make", "-s", "-C", HERE], check=True)
    return LIB_PATH


def build_ref() -> str | None:
    """Compile oracle/_ref/libdgtref.so from the reference's sources when they are present."""
    if not os.path.isdir(os.path.join(reference_dir(), "src", "model")):
        return REF_PATH if os.path.exists(REF_PATH) else None
    harness = os.path.join(HERE, "ref_harness.cu")
    if not os.path.exists(REF_PATH) or os.path.getmtime(REF_PATH) < os.path.getmtime(harness):
        env = dict(os.environ, DGT_REFERENCE_DIR=reference_dir())
        subprocess.run(["bash", os.path.join(HERE, "build_ref.sh")], check=True, capture_output=True, env=env)
    return REF_PATH


_lib = None
_ref = None


def lib():
    global _lib
    if _lib is None:
        build()
        L = ctypes.CDLL(LIB_PATH)
        L.orc_ref_global.restype = ctypes.c_int
        L.orc_ref_global.argtypes = [_P_D, ctypes.c_int, ctypes.c_double, ctypes.c_double, ctypes.c_double,
                                     ctypes.c_int, ctypes.c_int, _P_I, _P_I]
        L.orc_ref_test_and_repair.restype = ctypes.c_int
        L.orc_ref_test_and_repair.argtypes = [_P_D, ctypes.c_int, ctypes.c_double, ctypes.c_double,
                                              ctypes.c_double, ctypes.c_int, ctypes.c_int, _P_I, _P_I, _P_I]
        L.orc_verify.restype = ctypes.c_int
        L.orc_verify.argtypes = [_P_D, ctypes.c_int, ctypes.c_double, ctypes.c_double, _P_I, _P_I, ctypes.c_int,
                                 ctypes.c_int, ctypes.c_int, ctypes.POINTER(OrcReport)]
        L.orc_incircle0.restype = ctypes.c_int
        L.orc_incircle0.argtypes = [_P_D, _P_D, _P_D]
        L.orc_orient0.restype = ctypes.c_int
        L.orc_orient0.argtypes = [_P_D, _P_D]
        L.orc_offset.restype = None
        L.orc_offset.argtypes = [_P_D, _P_D, ctypes.c_double, ctypes.c_double, _P_D]
        L.orc_offset_general.restype = None
        L.orc_offset_general.argtypes = [_P_D, _P_D, _P_D, _P_D]
        L.orc_reduce_basis.restype = None
        L.orc_reduce_basis.argtypes = [_P_D]
        L.orc_verify_general.restype = ctypes.c_int
        L.orc_verify_general.argtypes = [_P_D, ctypes.c_int, _P_D, _P_I, _P_I, ctypes.c_int, ctypes.c_int,
                                         ctypes.c_int, ctypes.POINTER(OrcReport)]
        L.orc_canonical_rotate.restype = None
        L.orc_canonical_rotate.argtypes = [_P_I, _P_I, ctypes.c_int, ctypes.c_int]
        _lib = L
    return _lib


def ref_lib():
    """The reference itself (oracle/_ref), or None when it was not built."""
    global _ref
    if _ref is None:
        path = build_ref()
        if path is None or not os.path.exists(path):
            return None
        R = ctypes.CDLL(path)
        R.ref_fn_global.restype = ctypes.c_int
        R.ref_fn_global.argtypes = [_P_D, ctypes.c_int, ctypes.c_double, ctypes.c_double, ctypes.c_double,
                                    ctypes.c_int, ctypes.c_int, _P_I, _P_I]
        R.ref_fn_test_and_repair.restype = ctypes.c_int
        R.ref_fn_test_and_repair.argtypes = [_P_D, ctypes.c_int, ctypes.c_double, ctypes.c_double,
                                             ctypes.c_double, ctypes.c_int, ctypes.c_int, _P_I, _P_I, _P_I]
        R.ref_cls_create.restype = ctypes.c_void_p
        R.ref_cls_create.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_double, ctypes.c_double,
                                     ctypes.c_double, ctypes.c_int]
        R.ref_cls_global.restype = ctypes.c_int
        R.ref_cls_global.argtypes = [ctypes.c_void_p, _P_D, _P_I, _P_I, ctypes.c_int]
        R.ref_cls_test_and_repair.restype = ctypes.c_int
        R.ref_cls_test_and_repair.argtypes = [ctypes.c_void_p, _P_D, _P_I, _P_I, ctypes.c_int]
        R.ref_cls_destroy.restype = None
        R.ref_cls_destroy.argtypes = [ctypes.c_void_p]
        R.ref_omp_max_threads.restype = ctypes.c_int
        R.ref_fn_seed_max.restype = ctypes.c_int
        R.ref_fn_seed_max.argtypes = [_P_D, ctypes.c_int, ctypes.c_double, ctypes.c_double, ctypes.c_double,
                                      ctypes.c_int, ctypes.c_int]
        R.ref_gpu_create.restype = ctypes.c_void_p
        R.ref_gpu_create.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_double, ctypes.c_double,
                                     ctypes.c_double, _P_D, _P_D]
        _P_F = ctypes.POINTER(ctypes.c_float)
        R.ref_gpu_build.restype = ctypes.c_int
        R.ref_gpu_build.argtypes = [ctypes.c_void_p, _P_F]
        R.ref_gpu_repair.restype = ctypes.c_int
        R.ref_gpu_repair.argtypes = [ctypes.c_void_p, _P_F]
        R.ref_gpu_triangles_ok.restype = ctypes.c_int
        R.ref_gpu_triangles_ok.argtypes = [ctypes.c_void_p]
        R.ref_gpu_fetch.restype = ctypes.c_int
        R.ref_gpu_fetch.argtypes = [ctypes.c_void_p, _P_I, _P_I, ctypes.c_int]
        R.ref_gpu_destroy.restype = None
        R.ref_gpu_destroy.argtypes = [ctypes.c_void_p]
        R.ref_xy2d.restype = ctypes.c_int
        R.ref_xy2d.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_int]
        _ref = R
    return _ref


def _pd(a):
    return a.ctypes.data_as(_P_D)


def _pi(a):
    return a.ctypes.data_as(_P_I)


@dataclass
class Triangulation:
    tri: np.ndarray  # (n, stride) int32, rows hold the CCW ring in their first nn[i] entries
    nn: np.ndarray   # (n,) int32
    max_ring: int

    @property
    def stride(self) -> int:
        return self.tri.shape[1]


def _prep(points):
    pts = np.ascontiguousarray(points, dtype=np.float64)
    assert pts.ndim == 2 and pts.shape[1] == 2
    return pts


def default_threads() -> int:
    return max(1, os.cpu_count() or 1)


def restated_global(points, Lx, Ly, cell_size=1.0, stride=32, threads=None) -> Triangulation:
    """The C restatement of the reference's global triangulation (host path)."""
    pts = _prep(points)
    n = len(pts)
    tri = np.zeros((n, stride), np.int32)
    nn = np.zeros(n, np.int32)
    r = lib().orc_ref_global(_pd(pts), n, Lx, Ly, cell_size, stride, threads or default_threads(), _pi(tri), _pi(nn))
    if r < 0:
        raise RuntimeError(f"restated global triangulation failed ({r})")
    return Triangulation(tri, nn, r)


def restated_test_and_repair(points, Lx, Ly, tri: Triangulation, cell_size=1.0, threads=None):
    """The C restatement of the reference's test-and-repair, on a copy of ``tri``.
    Returns (Triangulation, repair flags)."""
    pts = _prep(points)
    n = len(pts)
    t = np.ascontiguousarray(tri.tri.copy())
    nn = np.ascontiguousarray(tri.nn.copy())
    rep = np.zeros(n, np.int32)
    r = lib().orc_ref_test_and_repair(_pd(pts), n, Lx, Ly, cell_size, t.shape[1], threads or default_threads(),
                                      _pi(t), _pi(nn), _pi(rep))
    if r < 0:
        raise RuntimeError(f"restated test-and-repair failed ({r})")
    return Triangulation(t, nn, int(nn.max())), rep


def reference_global(points, Lx, Ly, cell_size=1.0, stride=32, threads=None) -> Triangulation:
    """The reference's own host path (oracle/_ref, callers with GPUcompute=false)."""
    R = ref_lib()
    if R is None:
        raise RuntimeError("oracle/_ref/libdgtref.so is not built")
    pts = _prep(points)
    n = len(pts)
    tri = np.zeros((n, stride), np.int32)
    nn = np.zeros(n, np.int32)
    r = R.ref_fn_global(_pd(pts), n, Lx, Ly, cell_size, stride, threads or default_threads(), _pi(tri), _pi(nn))
    return Triangulation(tri, nn, r)


def reference_test_and_repair(points, Lx, Ly, tri: Triangulation, cell_size=1.0, threads=None):
    R = ref_lib()
    if R is None:
        raise RuntimeError("oracle/_ref/libdgtref.so is not built")
    pts = _prep(points)
    n = len(pts)
    t = np.ascontiguousarray(tri.tri.copy())
    nn = np.ascontiguousarray(tri.nn.copy())
    rep = np.zeros(n, np.int32)
    r = R.ref_fn_test_and_repair(_pd(pts), n, Lx, Ly, cell_size, t.shape[1], threads or default_threads(),
                                 _pi(t), _pi(nn), _pi(rep))
    if r < 0:
        raise RuntimeError(f"reference test-and-repair failed ({r})")
    return Triangulation(t, nn, int(nn.max())), rep


class ReferenceClass:
    """The reference's public DelaunayGPU class on its host path (needs a CUDA device)."""

    def __init__(self, n, max_neighs, cell_size, Lx, Ly, threads=None):
        R = ref_lib()
        if R is None:
            raise RuntimeError("oracle/_ref/libdgtref.so is not built")
        self.R = R
        self.n = n
        self.h = R.ref_cls_create(n, max_neighs, cell_size, Lx, Ly, threads or default_threads())
        if not self.h:
            raise RuntimeError("reference DelaunayGPU construction failed")

    def global_triangulation(self, points, stride=32, fetch=True):
        pts = _prep(points)
        tri = np.zeros((self.n, stride), np.int32) if fetch else None
        nn = np.zeros(self.n, np.int32) if fetch else None
        r = self.R.ref_cls_global(self.h, _pd(pts), _pi(tri) if fetch else None, _pi(nn) if fetch else None, stride)
        if r < 0:
            raise RuntimeError("reference globalDelaunayTriangulation failed")
        return Triangulation(tri, nn, r) if fetch else None

    def test_and_repair(self, points, stride=32, fetch=True):
        pts = _prep(points)
        tri = np.zeros((self.n, stride), np.int32) if fetch else None
        nn = np.zeros(self.n, np.int32) if fetch else None
        r = self.R.ref_cls_test_and_repair(self.h, _pd(pts), _pi(tri) if fetch else None,
                                           _pi(nn) if fetch else None, stride)
        if r < 0:
            raise RuntimeError("reference testAndRepairDelaunayTriangulation failed")
        return Triangulation(tri, nn, r) if fetch else None

    def close(self):
        if self.h:
            self.R.ref_cls_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def reference_seed_max(points, Lx, Ly, cell_size=1.0, stride=64, threads=None) -> int:
    """Largest candidate polygon of the reference's seed pass over ``points`` (run on the
    host); -1 if it reaches ``stride``."""
    R = ref_lib()
    if R is None:
        raise RuntimeError("oracle/_ref/libdgtref.so is not built")
    pts = _prep(points)
    return R.ref_fn_seed_max(_pd(pts), len(pts), Lx, Ly, cell_size, stride, threads or default_threads())


class ReferenceGPU:
    """The reference's public DelaunayGPU class on its GPU path (its own CUDA kernels,
    setGPUcompute(true), safety mode on): a global triangulation of ``p0`` and a
    test-and-repair with the moved points ``p1``, each timed on the device."""

    def __init__(self, p0, p1, Lx, Ly, max_neighs=24, cell_size=1.0):
        R = ref_lib()
        if R is None:
            raise RuntimeError("oracle/_ref/libdgtref.so is not built")
        self.R = R
        a, b = _prep(p0), _prep(p1)
        self.n = len(a)
        self.h = R.ref_gpu_create(self.n, max_neighs, cell_size, Lx, Ly, _pd(a), _pd(b))
        if not self.h:
            raise RuntimeError("reference DelaunayGPU (GPU path) construction failed")

    def build(self) -> float:
        ms = ctypes.c_float(0.0)
        if self.R.ref_gpu_build(self.h, ctypes.byref(ms)) != 0:
            raise RuntimeError("reference GPU globalDelaunayTriangulation failed")
        return ms.value

    def triangles_ok(self) -> bool:
        return self.R.ref_gpu_triangles_ok(self.h) == 1

    def repair(self) -> float:
        ms = ctypes.c_float(0.0)
        r = self.R.ref_gpu_repair(self.h, ctypes.byref(ms))
        if r == -2:
            raise RuntimeError("reference GPU repair refused: the triangulation does not have exactly 2N triangles")
        if r != 0:
            raise RuntimeError("reference GPU testAndRepairDelaunayTriangulation failed")
        return ms.value

    def fetch(self, stride=32) -> Triangulation:
        tri = np.zeros((self.n, stride), np.int32)
        nn = np.zeros(self.n, np.int32)
        if self.R.ref_gpu_fetch(self.h, _pi(tri), _pi(nn), stride) < 0:
            raise RuntimeError("reference GPU fetch failed")
        return Triangulation(tri, nn, int(nn.max()))

    def close(self):
        if self.h:
            self.R.ref_gpu_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def verify(points, Lx, Ly, tri, nn, global_scan=True, threads=None):
    """Exact check that (tri, nn) is the Delaunay triangulation.  Returns (ok, report dict)."""
    pts = _prep(points)
    t = np.ascontiguousarray(tri, dtype=np.int32)
    nnv = np.ascontiguousarray(nn, dtype=np.int32)
    rep = OrcReport()
    r = lib().orc_verify(_pd(pts), len(pts), Lx, Ly, _pi(t), _pi(nnv), t.shape[1], 1 if global_scan else 0,
                         threads or default_threads(), ctypes.byref(rep))
    return r == 0, rep.as_dict()


def verify_general(points, box, tri, nn, global_scan=True, threads=None):
    """verify() in a general periodic box, box = (xx, xy, yx, yy) (periodicBoundaries(a, b, c, d);
    lattice vectors (xx, yx) and (xy, yy)).  Returns (ok, report dict)."""
    pts = _prep(points)
    bx = np.ascontiguousarray(box, dtype=np.float64)
    t = np.ascontiguousarray(tri, dtype=np.int32)
    nnv = np.ascontiguousarray(nn, dtype=np.int32)
    rep = OrcReport()
    r = lib().orc_verify_general(_pd(pts), len(pts), _pd(bx), _pi(t), _pi(nnv), t.shape[1],
                                 1 if global_scan else 0, threads or default_threads(), ctypes.byref(rep))
    return r == 0, rep.as_dict()


def offset_general(c, p, box):
    """Offset c - p to the image whose fractional offset lies in [-1/2, 1/2] (general box)."""
    c = np.ascontiguousarray(c, np.float64)
    p = np.ascontiguousarray(p, np.float64)
    bx = np.ascontiguousarray(box, np.float64)
    out = np.zeros(2, np.float64)
    lib().orc_offset_general(_pd(c), _pd(p), _pd(bx), _pd(out))
    return out


def reduce_basis(box):
    """Lagrange-Gauss reduced basis of the lattice of box = (xx, xy, yx, yy)."""
    bx = np.array(box, dtype=np.float64)
    lib().orc_reduce_basis(_pd(bx))
    return tuple(float(v) for v in bx)


def hilbert_index(k, x, y):
    """Hilbert-curve index of grid squares (x, y) of a 2^k x 2^k grid (integer arrays): the
    standard conversion the reference's xy2d performs (src/utilities/hilbert_curve.cpp:229,
    with its quadrant rotation rot, :137), restated level by level from the coarsest."""
    x = np.asarray(x, dtype=np.int64).copy()
    y = np.asarray(y, dtype=np.int64).copy()
    d = np.zeros(np.broadcast(x, y).shape, dtype=np.int64)
    for lv in range(k - 1, -1, -1):
        s = 1 << lv
        rx = (x >> lv) & 1
        ry = (y >> lv) & 1
        d += s * s * ((3 * rx) ^ ry)
        x &= s - 1
        y &= s - 1
        refl = (ry == 0) & (rx == 1)
        x = np.where(refl, s - 1 - x, x)
        y = np.where(refl, s - 1 - y, y)
        swap = ry == 0
        x, y = np.where(swap, y, x), np.where(swap, x, y)
    return d


def reference_xy2d(m, x, y) -> int:
    """The reference's own xy2d (oracle/_ref), or None when it was not built."""
    R = ref_lib()
    return None if R is None else int(R.ref_xy2d(int(m), int(x), int(y)))


def hilbert_order(points, sizes, boxes):
    """Order of the points along a Hilbert curve over each set's rectangular box, set by set:
    a 2^k x 2^k grid per set (the smallest with 4^k >= its points, 1 <= k <= 15), square
    (floor(x * (2^k / Lx)), floor(y * (2^k / Ly))) clamped to the grid, points sorted by
    square index then by point index."""
    points = np.asarray(points, dtype=np.float64)
    out, off = [], 0
    for n, (Lx, Ly) in zip(sizes, boxes):
        n = int(n)
        k = 1
        while k < 15 and (1 << (2 * k)) < n:
            k += 1
        g = 1 << k
        p = points[off:off + n]

        def square(u):
            q = np.zeros(len(u), dtype=np.int64)
            ok = u >= 0.0
            q[ok] = np.where(u[ok] < g, np.floor(u[ok]), g - 1).astype(np.int64)
            return q

        key = hilbert_index(k, square(p[:, 0] * (g / Lx)), square(p[:, 1] * (g / Ly)))
        out.append(np.lexsort((np.arange(n), key)) + off)
        off += n
    return np.concatenate(out) if out else np.zeros(0, dtype=np.int64)


def canonical(tri, nn):
    """Copy of the rings rotated so each starts at its smallest index; unused slots -> -1."""
    t = np.ascontiguousarray(np.array(tri, dtype=np.int32, copy=True))
    nnv = np.ascontiguousarray(nn, dtype=np.int32)
    lib().orc_canonical_rotate(_pi(t), _pi(nnv), t.shape[0], t.shape[1])
    cols = np.arange(t.shape[1])[None, :]
    t[cols >= nnv[:, None]] = -1
    return t


def incircle0(a, b, d) -> int:
    a = np.ascontiguousarray(a, np.float64)
    b = np.ascontiguousarray(b, np.float64)
    d = np.ascontiguousarray(d, np.float64)
    return lib().orc_incircle0(_pd(a), _pd(b), _pd(d))


def orient0(a, b) -> int:
    a = np.ascontiguousarray(a, np.float64)
    b = np.ascontiguousarray(b, np.float64)
    return lib().orc_orient0(_pd(a), _pd(b))
