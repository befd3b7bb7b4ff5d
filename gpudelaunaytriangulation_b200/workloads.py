"""Seeded synthetic point sets for the five workload families the library is measured on.

Every generator is a pure function of its seed: SplitMix64 (Steele, Lea & Flood 2014) gives
53-bit uniform doubles, Box-Muller turns pairs of them into normals.  Points are float64
``(n, 2)`` arrays in the primary cell ``[0, Lx) x [0, Ly)``.

- uniform periodic sets at unit density (side ``sqrt(n)``), the build/repair workloads;
- MD-like displacement: i.i.d. normal steps, wrapped back into the box;
- a jittered periodic triangular lattice (commensurate rectangular box);
- a wrapped Gaussian mixture with a large density contrast;
- an ensemble of independent sets with log-uniform sizes, each at unit density.
"""
from __future__ import annotations

import math

import numpy as np

_GOLDEN = np.uint64(0x9E3779B97F4A7C15)
_M1 = np.uint64(0xBF58476D1CE4E5B9)
_M2 = np.uint64(0x94D049BB133111EB)


def splitmix64_uniform(seed: int, count: int) -> np.ndarray:
    """``count`` doubles in [0, 1) from the SplitMix64 stream started at ``seed``."""
    with np.errstate(over="ignore"):
        s = np.uint64(seed & 0xFFFFFFFFFFFFFFFF) + np.arange(1, count + 1, dtype=np.uint64) * _GOLDEN
        z = (s ^ (s >> np.uint64(30))) * _M1
        z = (z ^ (z >> np.uint64(27))) * _M2
        z = z ^ (z >> np.uint64(31))
    return (z >> np.uint64(11)).astype(np.float64) * (1.0 / 9007199254740992.0)


def wrap(points: np.ndarray, Lx: float, Ly: float) -> np.ndarray:
    """Put points back into [0, Lx) x [0, Ly) (the periodic box's primary cell)."""
    out = np.array(points, dtype=np.float64, copy=True)
    out[:, 0] = np.mod(out[:, 0], Lx)
    out[:, 1] = np.mod(out[:, 1], Ly)
    # np.mod can return L itself for tiny negative inputs; fold those onto 0
    out[out[:, 0] >= Lx, 0] = 0.0
    out[out[:, 1] >= Ly, 1] = 0.0
    return out


def uniform_points(n: int, L: float | None = None, seed: int = 1, Ly: float | None = None) -> np.ndarray:
    """n i.i.d. uniform points in the periodic box [0, L) x [0, Ly) (default L = sqrt(n))."""
    Lx = math.sqrt(n) if L is None else float(L)
    Ly = Lx if Ly is None else float(Ly)
    u = splitmix64_uniform(seed, 2 * n).reshape(n, 2)
    pts = np.empty((n, 2), np.float64)
    pts[:, 0] = u[:, 0] * Lx
    pts[:, 1] = u[:, 1] * Ly
    return wrap(pts, Lx, Ly)


def normal_pairs(seed: int, n: int) -> np.ndarray:
    """(n, 2) standard normals by Box-Muller from the SplitMix64 stream ``seed``."""
    u = splitmix64_uniform(seed, 2 * n).reshape(n, 2)
    r = np.sqrt(-2.0 * np.log1p(-u[:, 0]))
    t = 2.0 * math.pi * u[:, 1]
    return np.stack([r * np.cos(t), r * np.sin(t)], axis=1)


def displace(points: np.ndarray, sigma: float, Lx: float, Ly: float, seed: int) -> np.ndarray:
    """One MD-like step: every point moves by N(0, sigma^2) per axis, then is wrapped."""
    return wrap(points + sigma * normal_pairs(seed, len(points)), Lx, Ly)


def triangular_lattice(nx: int, ny: int, spacing: float = 1.0, jitter: float = 1e-4, seed: int = 3):
    """Periodic triangular lattice of nx*ny sites (ny even so the box is commensurate),
    each jittered by U[-jitter, jitter]^2.  Returns (points, Lx, Ly)."""
    if ny % 2:
        raise ValueError("ny must be even for a periodic triangular lattice")
    Lx = nx * spacing
    Ly = ny * spacing * math.sqrt(3.0) / 2.0
    j, i = np.meshgrid(np.arange(ny), np.arange(nx), indexing="ij")
    x = (i + 0.5 * (j % 2)) * spacing
    y = j * spacing * math.sqrt(3.0) / 2.0
    pts = np.stack([x.ravel(), y.ravel()], axis=1).astype(np.float64)
    u = splitmix64_uniform(seed, 2 * len(pts)).reshape(-1, 2)
    pts += (2.0 * u - 1.0) * jitter
    return wrap(pts, Lx, Ly), Lx, Ly


def square_lattice(n: int, phase: float = 0.25, seed: int = 4):
    """The reference driver's squareLattice input (triangulation.cpp:39-61): a k x k square
    lattice, k = ceil(sqrt(n)), of spacing sqrt(n) / k in the box of side sqrt(n), each site
    drawn uniformly within +-phase spacings of its centre, sites taken column by column until
    n are placed.  Returns (points, L)."""
    L = math.sqrt(n)
    k = int(math.ceil(math.sqrt(n)))
    s = L / k
    x, y = np.meshgrid(np.arange(k), np.arange(k), indexing="ij")   # x outer, y inner
    centre = np.stack([x.ravel(), y.ravel()], axis=1)[:n].astype(np.float64) + 0.5
    u = splitmix64_uniform(seed, 2 * n).reshape(-1, 2)
    pts = s * (centre + (2.0 * u - 1.0) * phase)
    return wrap(pts, L, L), L


def gaussian_mixture(n: int, components: int = 64, sigma: float = 2.0, L: float | None = None, seed: int = 5):
    """n points from an equal-weight mixture of isotropic Gaussians (std sigma) whose centres are
    uniform in the periodic box of side L (default sqrt(n)), wrapped.  Returns (points, L)."""
    L = math.sqrt(n) if L is None else float(L)
    centres = uniform_points(components, L, seed=seed + 1)
    which = np.floor(splitmix64_uniform(seed + 2, n) * components).astype(np.int64)
    pts = centres[which] + sigma * normal_pairs(seed + 3, n)
    return wrap(pts, L, L), L


def ensemble_sizes(num_sets: int = 256, lo: int = 1000, hi: int = 65536, seed: int = 7) -> np.ndarray:
    """Set sizes drawn log-uniform in [lo, hi]."""
    u = splitmix64_uniform(seed, num_sets)
    return np.floor(np.exp(np.log(lo) + u * (np.log(hi) - np.log(lo)))).astype(np.int64)


def ensemble(num_sets: int = 256, lo: int = 1000, hi: int = 65536, seed: int = 7):
    """Independent uniform sets at unit density.  Returns (points concatenated, sizes, boxes)
    with boxes an (num_sets, 2) array of (Lx, Ly)."""
    sizes = ensemble_sizes(num_sets, lo, hi, seed)
    boxes = np.sqrt(sizes.astype(np.float64))
    pts = [uniform_points(int(n), float(L), seed=seed * 1000003 + s) for s, (n, L) in enumerate(zip(sizes, boxes))]
    return np.concatenate(pts, axis=0), sizes, np.stack([boxes, boxes], axis=1)
