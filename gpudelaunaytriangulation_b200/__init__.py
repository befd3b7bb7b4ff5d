"""B200-native periodic Delaunay one-rings (per-point Chen-Gotsman construction and
circumcircle test-and-repair) behind the reference DelaunayGPU API.

The compute path is libdgt.so (CUDA, sm_100a) reached through the C ABI in include/dgt.h.
"""
from .build import LIB as LIBRARY_PATH  # noqa: F401


def __getattr__(name):
    # torch-dependent pieces load lazily so the pure-host parts import without CUDA
    if name in ("DelaunayGPU", "DelaunayBatch", "PeriodicBox"):
        from . import delaunay

        return getattr(delaunay, name)
    raise AttributeError(name)
