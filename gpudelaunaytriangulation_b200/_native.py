"""ctypes binding of libdgt.so (the C ABI declared in include/dgt.h).

There is no fallback: if the library is missing or cannot be loaded this module raises.
"""
from __future__ import annotations

import ctypes
import os

from . import build as _build

P_D = ctypes.POINTER(ctypes.c_double)
P_I = ctypes.POINTER(ctypes.c_int)

DGT_OK = 0
DGT_ERR_INVALID_ARGUMENT = 1
DGT_ERR_CUDA = 2
DGT_ERR_NEED_RESIZE = 3
DGT_ERR_DEGENERATE = 4
DGT_ERR_OUT_OF_MEMORY = 5
DGT_ERR_BAD_POINTS = 6
DGT_ERR_NOT_CONVERGED = 7

PRECISION_FP32_FILTER = 0
PRECISION_FP64 = 1

# every symbol include/dgt.h declares (checked by the CPU test suite)
EXPORTED = [
    "dgt_create", "dgt_create_batch", "dgt_destroy", "dgt_global_triangulation", "dgt_test_and_repair",
    "dgt_update_list", "dgt_set_cell_size", "dgt_set_box", "dgt_set_safety_mode", "dgt_set_precision",
    "dgt_set_check_mode", "dgt_resize", "dgt_get_max_size", "dgt_get_num_points", "dgt_restride",
    "dgt_get_stats", "dgt_displace", "dgt_error_string", "dgt_version", "dgt_set_timing",
    "dgt_get_phase_times", "dgt_global_triangulation_noalloc", "dgt_md_step", "dgt_md_graph_create",
    "dgt_md_graph_launch", "dgt_md_graph_destroy", "dgt_clear_flags", "dgt_set_kernel_shape",
    "dgt_get_tuning", "dgt_autotune", "dgt_set_work_budget", "dgt_set_flip_repair",
    "dgt_validate", "dgt_get_cell_order", "dgt_set_box_general", "dgt_get_box", "dgt_create_batch_general",
    "dgt_set_graph_flip_rounds", "dgt_get_hilbert_order", "dgt_set_deferred_overlap",
    "dgt_hilbert_sort_points",
]
STEP_AUTO = 0xFFFFFFFFFFFFFFFF
NOALLOC_MAX_POINTS = 65536
KERNEL_SHAPES = 7   # dgt_set_kernel_shape: 0..6 (include/dgt.h)
PHASES = ["bin", "build", "slow", "test", "repair"]


class Stats(ctypes.Structure):
    _fields_ = [
        ("points", ctypes.c_longlong),
        ("candidates", ctypes.c_longlong),
        ("tests", ctypes.c_longlong),
        ("fp32_undecided", ctypes.c_longlong),
        ("fp64_undecided", ctypes.c_longlong),
        ("exact_points", ctypes.c_longlong),
        ("mismatches", ctypes.c_longlong),
        ("insertions", ctypes.c_longlong),
        ("flagged", ctypes.c_longlong),
        ("repaired", ctypes.c_longlong),
        ("cells", ctypes.c_longlong),
        ("repair_rounds", ctypes.c_int),
        ("max_ring", ctypes.c_int),
        ("error_flags", ctypes.c_int),
        ("launches", ctypes.c_int),
        ("sticky_flags", ctypes.c_int),
        ("reserved", ctypes.c_int),
        ("repair_calls", ctypes.c_longlong),
        ("md_step", ctypes.c_longlong),
        ("heavy_points", ctypes.c_longlong),
        ("flips", ctypes.c_longlong),
        ("flip_spilled", ctypes.c_longlong),
        ("flip_rounds", ctypes.c_int),
        ("rebinned", ctypes.c_int),
    ]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_ if not k.startswith("reserved")}


class Validation(ctypes.Structure):
    _fields_ = [
        ("points", ctypes.c_longlong),
        ("sum_neighbors", ctypes.c_longlong),
        ("bad_rows", ctypes.c_longlong),
        ("asymmetric", ctypes.c_longlong),
        ("not_ccw", ctypes.c_longlong),
        ("winding", ctypes.c_longlong),
        ("not_delaunay", ctypes.c_longlong),
        ("valid", ctypes.c_int),
        ("reserved", ctypes.c_int),
    ]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_ if k != "reserved"}


class TuneResult(ctypes.Structure):
    _fields_ = [
        ("cell_size", ctypes.c_double),
        ("shape", ctypes.c_int),
        ("trials", ctypes.c_int),
        ("best_ms", ctypes.c_float),
        ("default_ms", ctypes.c_float),
        ("from_cache", ctypes.c_int),
        ("work_budget", ctypes.c_int),
        ("deferred_chunks", ctypes.c_int),
        ("reserved", ctypes.c_int),
    ]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_ if not k.startswith("reserved")}


class DgtError(RuntimeError):
    def __init__(self, code: int, where: str):
        self.code = code
        msg = lib().dgt_error_string(code).decode()
        super().__init__(f"{where}: {msg} (code {code})")


_lib = None


def library_path() -> str:
    return _build.LIB


def lib() -> ctypes.CDLL:
    """Load libdgt.so (built in-tree by build.py; built here only if it is missing)."""
    global _lib
    if _lib is not None:
        return _lib
    path = _build.LIB
    if not os.path.exists(path):
        try:
            _build.build()
        except Exception as exc:  # pragma: no cover - build failures surface below
            raise RuntimeError(f"libdgt.so is missing and could not be built: {exc}") from exc
    if not os.path.exists(path):
        raise RuntimeError(f"libdgt.so not found at {path}; run python -m gpudelaunaytriangulation_b200.build")
    L = ctypes.CDLL(path)
    vp = ctypes.c_void_p
    L.dgt_create.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_double, ctypes.c_double, ctypes.c_double,
                             ctypes.POINTER(vp)]
    L.dgt_create_batch.argtypes = [ctypes.c_int, P_I, P_D, ctypes.c_double, ctypes.c_int, ctypes.POINTER(vp)]
    L.dgt_create_batch_general.argtypes = [ctypes.c_int, P_I, P_D, ctypes.c_double, ctypes.c_int,
                                           ctypes.POINTER(vp)]
    L.dgt_destroy.argtypes = [vp]
    L.dgt_destroy.restype = None
    L.dgt_global_triangulation.argtypes = [vp, vp, vp, vp, ctypes.c_int, vp]
    L.dgt_test_and_repair.argtypes = [vp, vp, vp, vp, ctypes.c_int, vp]
    L.dgt_update_list.argtypes = [vp, vp, vp]
    L.dgt_set_cell_size.argtypes = [vp, ctypes.c_double]
    L.dgt_set_box.argtypes = [vp, ctypes.c_double, ctypes.c_double]
    L.dgt_set_box_general.argtypes = [vp, ctypes.c_double, ctypes.c_double, ctypes.c_double, ctypes.c_double]
    L.dgt_get_box.argtypes = [vp, P_D]
    L.dgt_set_safety_mode.argtypes = [vp, ctypes.c_int]
    L.dgt_set_precision.argtypes = [vp, ctypes.c_int]
    L.dgt_set_check_mode.argtypes = [vp, ctypes.c_int]
    L.dgt_resize.argtypes = [vp, ctypes.c_int]
    L.dgt_get_max_size.argtypes = [vp, P_I]
    L.dgt_get_num_points.argtypes = [vp, P_I]
    L.dgt_restride.argtypes = [vp, ctypes.c_int, vp, ctypes.c_int, vp, ctypes.c_int, vp]
    L.dgt_get_stats.argtypes = [vp, ctypes.POINTER(Stats)]
    L.dgt_displace.argtypes = [vp, vp, ctypes.c_double, ctypes.c_ulonglong, ctypes.c_ulonglong, vp]
    L.dgt_error_string.argtypes = [ctypes.c_int]
    L.dgt_error_string.restype = ctypes.c_char_p
    L.dgt_version.restype = ctypes.c_int
    L.dgt_set_timing.argtypes = [vp, ctypes.c_int]
    L.dgt_get_phase_times.argtypes = [vp, P_D]
    L.dgt_md_step.argtypes = [vp, vp, vp, vp, ctypes.c_int, ctypes.c_double, ctypes.c_ulonglong, ctypes.c_int, vp]
    L.dgt_md_graph_create.argtypes = [vp, vp, vp, vp, ctypes.c_int, ctypes.c_double, ctypes.c_ulonglong,
                                      ctypes.c_int, ctypes.c_int, vp, ctypes.POINTER(vp)]
    L.dgt_md_graph_launch.argtypes = [vp, vp]
    L.dgt_md_graph_destroy.argtypes = [vp]
    L.dgt_md_graph_destroy.restype = None
    L.dgt_clear_flags.argtypes = [vp, vp]
    L.dgt_set_kernel_shape.argtypes = [vp, ctypes.c_int]
    L.dgt_set_work_budget.argtypes = [vp, ctypes.c_int]
    L.dgt_set_flip_repair.argtypes = [vp, ctypes.c_int]
    L.dgt_set_graph_flip_rounds.argtypes = [vp, ctypes.c_int]
    L.dgt_validate.argtypes = [vp, vp, vp, vp, ctypes.c_int, ctypes.POINTER(Validation), vp]
    L.dgt_get_cell_order.argtypes = [vp, vp, vp]
    L.dgt_get_hilbert_order.argtypes = [vp, vp, vp, vp]
    L.dgt_hilbert_sort_points.argtypes = [vp, vp, vp, vp]
    L.dgt_set_deferred_overlap.argtypes = [vp, ctypes.c_int]
    L.dgt_get_tuning.argtypes = [vp, P_D, P_I, P_I, P_I]
    L.dgt_autotune.argtypes = [vp, vp, vp, vp, ctypes.c_int, vp, ctypes.POINTER(TuneResult)]
    L.dgt_global_triangulation_noalloc.argtypes = [vp, ctypes.c_int, ctypes.c_double, ctypes.c_double,
                                                   ctypes.c_double, vp, vp, ctypes.c_int, P_I, vp]
    _lib = L
    return L


def check(code: int, where: str) -> int:
    if code != DGT_OK:
        raise DgtError(code, where)
    return code
