"""Python mirror of the reference's DelaunayGPU class (src/model/DelaunayGPU.h:18-130) over
the C ABI.  Device memory is held in torch CUDA tensors (plumbing only); every call goes to
libdgt.so and fails loudly when the library or a GPU is missing.

    box = PeriodicBox(L, L)
    delGPU = DelaunayGPU(N, maxNeighs, cellSize, box)             # DelaunayGPU.h:25
    tri = torch.zeros(maxNeighs * N, dtype=torch.int32, device="cuda")
    nn = torch.zeros(N, dtype=torch.int32, device="cuda")
    delGPU.globalDelaunayTriangulation(pts, tri, nn)              # DelaunayGPU.h:30
    delGPU.testAndRepairDelaunayTriangulation(pts, tri, nn)       # DelaunayGPU.h:33

As in the reference the callee may resize the caller's triangulation array to MaxSize*N
(DelaunayGPU.cpp:126-132, :152-155); the row stride is tri.numel() // N.  With safety mode
off an overflowing ring raises instead of silently corrupting the output (the reference's
GPU path returns early without writing, DelaunayGPU.cu:874-879).
"""
from __future__ import annotations

import ctypes
from dataclasses import dataclass

import torch

from . import _native as _nat


@dataclass
class PeriodicBox:
    """Periodic box (src/utilities/periodicBoundaries.h).  PeriodicBox(Lx, Ly) is the
    rectangle [0, Lx) x [0, Ly) (periodicBoundaries(x, y), :30); PeriodicBox(xx, yy, xy, yx),
    or PeriodicBox.general(xx, xy, yx, yy) in the reference's argument order, is the general
    box of periodicBoundaries(a, b, c, d) (:32, setGeneral :86-101): a point is
    (xx u + xy v, yx u + yy v) for fractional coordinates (u, v)."""

    Lx: float
    Ly: float
    xy: float = 0.0
    yx: float = 0.0

    @classmethod
    def general(cls, xx: float, xy: float, yx: float, yy: float) -> "PeriodicBox":
        return cls(float(xx), float(yy), float(xy), float(yx))

    @classmethod
    def of(cls, box) -> "PeriodicBox":
        """A PeriodicBox, an (Lx, Ly) pair or a general (xx, xy, yx, yy) matrix."""
        if isinstance(box, PeriodicBox):
            return box
        box = tuple(float(v) for v in box)
        if len(box) == 2:
            return cls(*box)
        if len(box) == 4:
            return cls.general(*box)
        raise ValueError("a box is (Lx, Ly) or (xx, xy, yx, yy)")

    def isBoxSquare(self) -> bool:
        """periodicBoundaries::isBoxSquare (:39): rectangular."""
        return self.xy == 0.0 and self.yx == 0.0

    def getBoxDims(self):
        """periodicBoundaries::getBoxDims (:36): (xx, xy, yx, yy)."""
        return self.Lx, self.xy, self.yx, self.Ly

    def putInBoxReal(self, p: torch.Tensor) -> torch.Tensor:
        """Wrap points into the primary cell (periodicBoundaries.h:131-152)."""
        out = p.clone()
        if not self.isBoxSquare():
            xx, xy, yx, yy = self.getBoxDims()
            det = xx * yy - xy * yx
            u = (yy * out[..., 0] - xy * out[..., 1]) / det
            v = (-yx * out[..., 0] + xx * out[..., 1]) / det
            u = torch.remainder(u, 1.0)
            v = torch.remainder(v, 1.0)
            u = torch.where(u >= 1.0, torch.zeros_like(u), u)
            v = torch.where(v >= 1.0, torch.zeros_like(v), v)
            out[..., 0] = xx * u + xy * v
            out[..., 1] = yx * u + yy * v
            return out
        out[..., 0] = torch.remainder(out[..., 0], self.Lx)
        out[..., 1] = torch.remainder(out[..., 1], self.Ly)
        out[..., 0] = torch.where(out[..., 0] >= self.Lx, torch.zeros_like(out[..., 0]), out[..., 0])
        out[..., 1] = torch.where(out[..., 1] >= self.Ly, torch.zeros_like(out[..., 1]), out[..., 1])
        return out


def _ptr(t: torch.Tensor | None):
    return ctypes.c_void_p(t.data_ptr()) if t is not None else ctypes.c_void_p(0)


def _stream_ptr(stream):
    if stream is None:
        stream = torch.cuda.current_stream()
    return ctypes.c_void_p(stream.cuda_stream)


def _check_points(points: torch.Tensor, n: int):
    if not (isinstance(points, torch.Tensor) and points.is_cuda):
        raise TypeError("points must be a CUDA tensor")
    if points.dtype != torch.float64 or points.numel() != 2 * n or not points.is_contiguous():
        raise ValueError(f"points must be a contiguous float64 CUDA tensor of {n} x 2 values")


def _check_int(t: torch.Tensor, name: str):
    if not (isinstance(t, torch.Tensor) and t.is_cuda and t.dtype == torch.int32 and t.is_contiguous()):
        raise TypeError(f"{name} must be a contiguous int32 CUDA tensor")


class DelaunayGPU:
    """Per-point periodic Delaunay one-rings on the GPU (reference API names kept)."""

    def __init__(self, N: int, maximumNeighborsGuess: int = 16, cellSize: float = 1.0,
                 box: PeriodicBox | tuple | None = None, *, _batch=None):
        self._L = lib = _nat.lib()
        self._h = ctypes.c_void_p()
        if _batch is not None:
            sizes, boxes, rel_cell = _batch
            sz = (ctypes.c_int * len(sizes))(*[int(s) for s in sizes])
            pb = [PeriodicBox.of(b) for b in boxes]
            if all(b.isBoxSquare() for b in pb):
                bx = (ctypes.c_double * (2 * len(sizes)))(*[v for b in pb for v in (b.Lx, b.Ly)])
                _nat.check(lib.dgt_create_batch(len(sizes), sz, bx, float(rel_cell), int(maximumNeighborsGuess),
                                               ctypes.byref(self._h)), "dgt_create_batch")
            else:
                bx = (ctypes.c_double * (4 * len(sizes)))(*[v for b in pb for v in b.getBoxDims()])
                _nat.check(lib.dgt_create_batch_general(len(sizes), sz, bx, float(rel_cell),
                                                       int(maximumNeighborsGuess), ctypes.byref(self._h)),
                           "dgt_create_batch_general")
            self.Ncells = int(sum(int(s) for s in sizes))
            self.Box = None
        else:
            if box is None:
                raise ValueError("a periodic box is required")
            box = PeriodicBox.of(box)
            self.Box = box
            self.Ncells = int(N)
            if box.isBoxSquare():
                _nat.check(lib.dgt_create(self.Ncells, int(maximumNeighborsGuess), float(cellSize), box.Lx, box.Ly,
                                         ctypes.byref(self._h)), "dgt_create")
            else:
                # created on the bounding rectangle, then given the general box
                bx = abs(box.Lx) + abs(box.xy)
                by = abs(box.yx) + abs(box.Ly)
                _nat.check(lib.dgt_create(self.Ncells, int(maximumNeighborsGuess), float(cellSize), bx, by,
                                         ctypes.byref(self._h)), "dgt_create")
                try:
                    _nat.check(lib.dgt_set_box_general(self._h, *box.getBoxDims()), "dgt_set_box_general")
                except Exception:
                    lib.dgt_destroy(self._h)
                    self._h = ctypes.c_void_p()
                    raise
        self.safetyMode = True
        self.GPUcompute = True
        self.last_stats: dict | None = None

    # ------------------------------------------------------------------ reference setters
    @property
    def MaxSize(self) -> int:
        v = ctypes.c_int()
        _nat.check(self._L.dgt_get_max_size(self._h, ctypes.byref(v)), "dgt_get_max_size")
        return v.value

    def resize(self, nmax: int):
        """resize(nmax) (DelaunayGPU.h:38): the ring capacity MaxSize."""
        _nat.check(self._L.dgt_resize(self._h, int(nmax)), "dgt_resize")

    def setCellListSize(self, csize: float):
        _nat.check(self._L.dgt_set_cell_size(self._h, float(csize)), "dgt_set_cell_size")

    def setBox(self, box: PeriodicBox | tuple):
        """setBox(bx) (DelaunayGPU.h:44): rectangular or general box."""
        box = PeriodicBox.of(box)
        if box.isBoxSquare():
            _nat.check(self._L.dgt_set_box(self._h, box.Lx, box.Ly), "dgt_set_box")
        else:
            _nat.check(self._L.dgt_set_box_general(self._h, *box.getBoxDims()), "dgt_set_box_general")
        self.Box = box

    def kernelBox(self):
        """The box matrix (xx, xy, yx, yy) the kernels use: the reduced basis of a general box
        (the same lattice), (Lx, 0, 0, Ly) for a rectangle."""
        out = (ctypes.c_double * 4)()
        _nat.check(self._L.dgt_get_box(self._h, out), "dgt_get_box")
        return tuple(out)

    def setSafetyMode(self, flag: bool):
        self.safetyMode = bool(flag)
        _nat.check(self._L.dgt_set_safety_mode(self._h, 1 if flag else 0), "dgt_set_safety_mode")

    def setGPUcompute(self, flag: bool):
        """The reference can run its OpenMP host path instead; this library has no CPU path."""
        if not flag:
            raise NotImplementedError("no CPU path: the triangulation always runs on the GPU")
        self.GPUcompute = True

    def setOMPthreads(self, num: int):
        """Accepted for API compatibility; there is no host path to thread."""
        return None

    def setPrecision(self, fp32_filter: bool = True):
        _nat.check(self._L.dgt_set_precision(self._h, _nat.PRECISION_FP32_FILTER if fp32_filter else _nat.PRECISION_FP64),
                "dgt_set_precision")

    def setCheckMode(self, on: bool):
        _nat.check(self._L.dgt_set_check_mode(self._h, 1 if on else 0), "dgt_set_check_mode")

    # ------------------------------------------------------------------------- the path
    def updateList(self, points: torch.Tensor, stream=None):
        _check_points(points, self.Ncells)
        _nat.check(self._L.dgt_update_list(self._h, _ptr(points), _stream_ptr(stream)), "dgt_update_list")

    def _fit(self, tri: torch.Tensor | None, nn: torch.Tensor | None, device):
        n = self.Ncells
        if tri is None:
            tri = torch.zeros(self.MaxSize * n, dtype=torch.int32, device=device)
        if nn is None:
            nn = torch.zeros(n, dtype=torch.int32, device=device)
        _check_int(tri, "GPUTriangulation")
        _check_int(nn, "cellNeighborNum")
        if nn.numel() != n:
            nn.resize_(n)
        if n and (tri.numel() % n != 0 or tri.numel() // n < self.MaxSize):
            tri.resize_(self.MaxSize * n)
        return tri, nn

    def globalDelaunayTriangulation(self, points: torch.Tensor, GPUTriangulation: torch.Tensor | None = None,
                                    cellNeighborNum: torch.Tensor | None = None, stream=None):
        n = self.Ncells
        _check_points(points, n)
        tri, nn = self._fit(GPUTriangulation, cellNeighborNum, points.device)
        if n == 0:
            return tri, nn
        while True:
            stride = tri.numel() // n
            code = self._L.dgt_global_triangulation(self._h, _ptr(points), _ptr(tri), _ptr(nn), stride,
                                                    _stream_ptr(stream))
            if code == _nat.DGT_ERR_NEED_RESIZE and self.safetyMode:
                tri.resize_(self.MaxSize * n)   # DelaunayGPU.cpp:152-155 grows and recomputes
                continue
            _nat.check(code, "globalDelaunayTriangulation")
            break
        return tri, nn

    def testAndRepairDelaunayTriangulation(self, points: torch.Tensor, GPUTriangulation: torch.Tensor,
                                           cellNeighborNum: torch.Tensor, stream=None):
        n = self.Ncells
        _check_points(points, n)
        _check_int(GPUTriangulation, "GPUTriangulation")
        _check_int(cellNeighborNum, "cellNeighborNum")
        if n == 0:
            return GPUTriangulation, cellNeighborNum
        tri, nn = GPUTriangulation, cellNeighborNum
        while True:
            stride = tri.numel() // n
            code = self._L.dgt_test_and_repair(self._h, _ptr(points), _ptr(tri), _ptr(nn), stride,
                                               _stream_ptr(stream))
            if code == _nat.DGT_ERR_NEED_RESIZE and self.safetyMode:
                # re-stride every row into the larger array (rows keep their contents;
                # the reference copies linearly here, DelaunayGPU.cpp:109-112), then go on
                new = torch.zeros(self.MaxSize * n, dtype=torch.int32, device=tri.device)
                _nat.check(self._L.dgt_restride(_ptr(tri), stride, _ptr(new), self.MaxSize, _ptr(nn), n,
                                             _stream_ptr(stream)), "dgt_restride")
                tri.resize_(new.numel())
                tri.copy_(new)
                continue
            _nat.check(code, "testAndRepairDelaunayTriangulation")
            break
        return tri, nn

    def displace(self, points: torch.Tensor, sigma: float, seed: int, step: int, stream=None):
        """MD-like step helper: Gaussian displacement + periodic wrap on the device."""
        _check_points(points, self.Ncells)
        _nat.check(self._L.dgt_displace(self._h, _ptr(points), float(sigma), int(seed) & (2**64 - 1),
                                     int(step) & (2**64 - 1), _stream_ptr(stream)), "dgt_displace")

    def mdStep(self, points: torch.Tensor, tri: torch.Tensor, nn: torch.Tensor, sigma: float, seed: int,
               rounds: int = 4, stream=None):
        """One device-only MD step: Gaussian displacement (device step counter) then
        test-and-repair with a fixed number of rounds; no host synchronisation."""
        _check_points(points, self.Ncells)
        stride = tri.numel() // max(1, self.Ncells)
        _nat.check(self._L.dgt_md_step(self._h, _ptr(points), _ptr(tri), _ptr(nn), stride, float(sigma),
                                       int(seed) & (2**64 - 1), int(rounds), _stream_ptr(stream)), "dgt_md_step")

    def mdGraph(self, points: torch.Tensor, tri: torch.Tensor, nn: torch.Tensor, sigma: float, seed: int,
                steps: int, rounds: int = 4, stream=None) -> "MDGraph":
        """Capture `steps` MD steps into a CUDA graph (stream must not be the default one)."""
        _check_points(points, self.Ncells)
        if stream is None:
            raise ValueError("graph capture needs a non-default torch.cuda.Stream")
        stride = tri.numel() // max(1, self.Ncells)
        g = ctypes.c_void_p()
        _nat.check(self._L.dgt_md_graph_create(self._h, _ptr(points), _ptr(tri), _ptr(nn), stride, float(sigma),
                                               int(seed) & (2**64 - 1), int(steps), int(rounds),
                                               _stream_ptr(stream), ctypes.byref(g)), "dgt_md_graph_create")
        return MDGraph(self._L, g, steps)

    def setKernelShape(self, shape: int):
        _nat.check(self._L.dgt_set_kernel_shape(self._h, int(shape)), "dgt_set_kernel_shape")

    def validate(self, points: torch.Tensor, GPUTriangulation: torch.Tensor, cellNeighborNum: torch.Tensor,
                 stream=None) -> dict:
        """Check the triangulation on the device (exact predicates): well-formed rows, symmetric
        rings, counter-clockwise fans winding once, every edge locally Delaunay, ring sizes
        summing to 6N.  Returns the counts and `valid`."""
        n = self.Ncells
        _check_points(points, n)
        _check_int(GPUTriangulation, "GPUTriangulation")
        _check_int(cellNeighborNum, "cellNeighborNum")
        stride = GPUTriangulation.numel() // max(1, n)
        v = _nat.Validation()
        _nat.check(self._L.dgt_validate(self._h, _ptr(points), _ptr(GPUTriangulation), _ptr(cellNeighborNum), stride,
                                        ctypes.byref(v), _stream_ptr(stream)), "dgt_validate")
        return v.as_dict()

    def cellOrder(self, stream=None) -> torch.Tensor:
        """Indices of the points in the cell order of the last binning (int32, on the device):
        renumbering the points in this order puts Delaunay neighbours at nearby indices."""
        n = self.Ncells
        out = torch.empty(n, dtype=torch.int32, device="cuda")
        if n:
            _nat.check(self._L.dgt_get_cell_order(self._h, _ptr(out), _stream_ptr(stream)), "dgt_get_cell_order")
        return out

    def hilbertOrder(self, points: torch.Tensor, stream=None) -> torch.Tensor:
        """Indices of the points along a Hilbert curve over each set's box (int32, on the
        device; the reference's hilbertSortArray pre-pass, triangulation.cpp:63-88):
        renumbering the points in this order puts Delaunay neighbours at nearby indices."""
        n = self.Ncells
        _check_points(points, n)
        out = torch.empty(n, dtype=torch.int32, device=points.device)
        if n:
            _nat.check(self._L.dgt_get_hilbert_order(self._h, _ptr(points), _ptr(out), _stream_ptr(stream)),
                       "dgt_get_hilbert_order")
        return out

    def hilbertSort(self, points: torch.Tensor, stream=None) -> torch.Tensor:
        """Reorder `points` in place along hilbertOrder (the reference's hilbertSortArray,
        triangulation.cpp:63-88); returns the order (point k is the old point order[k])."""
        n = self.Ncells
        _check_points(points, n)
        out = torch.empty(n, dtype=torch.int32, device=points.device)
        if n:
            _nat.check(self._L.dgt_hilbert_sort_points(self._h, _ptr(points), _ptr(out), _stream_ptr(stream)),
                       "dgt_hilbert_sort_points")
        return out

    def setFlipRepair(self, on: bool):
        """Test-and-repair by Lawson flips first (default) or by rebuilding every flagged point."""
        _nat.check(self._L.dgt_set_flip_repair(self._h, int(bool(on))), "dgt_set_flip_repair")

    def setGraphFlipRounds(self, rounds: int):
        """Flip rounds of mdStep / mdGraph repairs (0..24, default 3; more pay off for larger
        displacements).  A graph keeps the value it was captured with."""
        _nat.check(self._L.dgt_set_graph_flip_rounds(self._h, int(rounds)), "dgt_set_graph_flip_rounds")

    def setWorkBudget(self, budget: int):
        """Cells + candidates a point may scan in the thread-per-point kernel before the
        warp-per-point kernel takes it over (0: every point goes to the warp kernel)."""
        _nat.check(self._L.dgt_set_work_budget(self._h, int(budget)), "dgt_set_work_budget")

    def setDeferredOverlap(self, chunks: int):
        """Global triangulations in `chunks` (1-8) pieces whose deferred points are rebuilt
        while the next pieces build (same output; see dgt_set_deferred_overlap)."""
        _nat.check(self._L.dgt_set_deferred_overlap(self._h, int(chunks)), "dgt_set_deferred_overlap")

    def tuning(self) -> dict:
        cs, sh, cap, blk = ctypes.c_double(), ctypes.c_int(), ctypes.c_int(), ctypes.c_int()
        _nat.check(self._L.dgt_get_tuning(self._h, ctypes.byref(cs), ctypes.byref(sh), ctypes.byref(cap),
                                          ctypes.byref(blk)), "dgt_get_tuning")
        return {"cell_size": cs.value, "shape": sh.value, "ring_capacity": cap.value, "block": blk.value}

    def autotune(self, points: torch.Tensor, tri: torch.Tensor, nn: torch.Tensor, stream=None) -> dict:
        """Pick cell size and kernel shape by timing builds of `points` (see dgt_autotune)."""
        _check_points(points, self.Ncells)
        stride = tri.numel() // max(1, self.Ncells)
        res = _nat.TuneResult()
        while True:
            stride = tri.numel() // max(1, self.Ncells)
            code = self._L.dgt_autotune(self._h, _ptr(points), _ptr(tri), _ptr(nn), stride, _stream_ptr(stream),
                                        ctypes.byref(res))
            if code == _nat.DGT_ERR_NEED_RESIZE and self.safetyMode:
                tri.resize_(self.MaxSize * self.Ncells)   # grow like the triangulation calls, tune again
                continue
            _nat.check(code, "dgt_autotune")
            break
        out = res.as_dict()
        out.update(self.tuning())
        return out

    def clearFlags(self, stream=None):
        _nat.check(self._L.dgt_clear_flags(self._h, _stream_ptr(stream)), "dgt_clear_flags")

    def setTiming(self, on: bool):
        """Record CUDA events around each phase of every call (see phaseTimes)."""
        _nat.check(self._L.dgt_set_timing(self._h, 1 if on else 0), "dgt_set_timing")

    def phaseTimes(self) -> dict:
        """Milliseconds per phase of the last call (None for phases it did not run)."""
        out = (ctypes.c_double * len(_nat.PHASES))()
        _nat.check(self._L.dgt_get_phase_times(self._h, out), "dgt_get_phase_times")
        return {name: (v if v >= 0 else None) for name, v in zip(_nat.PHASES, out)}

    def stats(self) -> dict:
        s = _nat.Stats()
        _nat.check(self._L.dgt_get_stats(self._h, ctypes.byref(s)), "dgt_get_stats")
        self.last_stats = s.as_dict()
        return self.last_stats

    def close(self):
        if getattr(self, "_h", None) and self._h.value:
            self._L.dgt_destroy(self._h)
            self._h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class MDGraph:
    """An instantiated CUDA graph of MD steps (see DelaunayGPU.mdGraph)."""

    def __init__(self, lib, handle, steps):
        self._L = lib
        self._g = handle
        self.steps = steps

    def launch(self, stream=None):
        _nat.check(self._L.dgt_md_graph_launch(self._g, _stream_ptr(stream)), "dgt_md_graph_launch")

    def close(self):
        if self._g and self._g.value:
            self._L.dgt_md_graph_destroy(self._g)
            self._g = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class DelaunayBatch(DelaunayGPU):
    """Many independent periodic sets triangulated / repaired by the same launches.
    Points of all sets are concatenated; rings hold global point indices."""

    def __init__(self, sizes, boxes, maximumNeighborsGuess: int = 16, cellSizeRelative: float = 1.0):
        super().__init__(0, maximumNeighborsGuess, 0.0, None, _batch=(list(sizes), list(boxes), cellSizeRelative))
        self.sizes = [int(s) for s in sizes]
        self.boxes = [PeriodicBox.of(b) for b in boxes]
