"""Seeded synthetic particle frames with the shapes of the Chain benchmark workloads.

The reference ships one real frame (a DamBreak fluid column, 80,703 particles) and
names no public benchmark suite, so every workload here is a deterministic synthetic
stand-in drawn with ``numpy.random.default_rng(seed)`` (PCG64):

* ``column``      80,703 float32 points: a jittered cubic lattice (spacing 0.0125) filling
                  [0,0.5]x[0,0.5]x[0,1.0] from the bottom, Gaussian jitter sigma=0.001,
                  random particle order.
* ``blobs``       16,777,216 float32 points in [0,100]^3: 80% from 64 isotropic Gaussian
                  blobs (centres uniform, sigma uniform in [0.5, 5], out-of-box samples
                  redrawn), 20% uniform background, random particle order.
* ``trajectory``  4,194,304 float64 points in the periodic box [0,160)^3: a jittered
                  lattice of spacing 1.0 (frame 0) advanced by Gaussian steps of
                  sigma=0.02 per frame and wrapped; one fixed random particle order.
* ``uneven``      256 frames with log-uniform counts in [1e4, 2e6], each drawn from one
                  of {column, blobs, uniform} and an error bound from {1e-2,1e-3,1e-4}.

Every frame is returned as a C-contiguous (N, 3) array; ``eb_for`` gives the absolute
error bound ``frac * range`` with ``range`` the largest per-axis extent (the
``realPSNR``/``equivalent_eb`` convention of the reference's reader.py:269-295).
"""
from __future__ import annotations

import numpy as np

COLUMN_N = 80_703
BLOBS_N = 16_777_216
TRAJECTORY_N = 4_194_304


def data_range(points: np.ndarray) -> float:
    p = np.asarray(points, dtype=np.float64)
    return float(np.max(p.max(axis=0) - p.min(axis=0)))


def eb_for(points: np.ndarray, frac: float) -> float:
    return float(frac) * data_range(points)


def column(n: int = COLUMN_N, seed: int = 0, dtype=np.float32) -> np.ndarray:
    """Dam-break-like fluid column; for n != 80,703 the lattice spacing is rescaled."""
    rng = np.random.default_rng(seed)
    spacing = 0.0125 * (COLUMN_N / n) ** (1.0 / 3.0)
    xs = np.arange(0.0, 0.5 + 1e-9, spacing)
    zs = np.arange(0.0, 1.0 + 1e-9, spacing)
    need = n
    nz = int(np.ceil(need / (xs.size * xs.size)))
    if nz > zs.size:
        zs = np.arange(nz) * spacing
    z, y, x = np.meshgrid(zs[:nz], xs, xs, indexing="ij")
    pts = np.stack([x.ravel(), y.ravel(), z.ravel()], axis=1)[:need]
    pts = pts + rng.normal(0.0, 0.001, size=pts.shape)
    pts = pts[rng.permutation(need)]
    return np.ascontiguousarray(pts.astype(dtype))


def blobs(n: int = BLOBS_N, seed: int = 1, dtype=np.float32, box: float = 100.0,
          nblobs: int = 64, clip: bool = False) -> np.ndarray:
    """Gaussian-blob mixture plus uniform background; ``clip=True`` clips instead of
    redrawing, piling points onto the box faces (an exact-correction stress case)."""
    rng = np.random.default_rng(seed)
    n_clustered = int(round(0.8 * n))
    centres = rng.uniform(0.0, box, size=(nblobs, 3))
    sigmas = rng.uniform(0.5, 5.0, size=nblobs)
    counts = rng.multinomial(n_clustered, np.full(nblobs, 1.0 / nblobs))
    parts = []
    for c, s, k in zip(centres, sigmas, counts):
        pts = rng.normal(c, s, size=(int(k), 3))
        if clip:
            np.clip(pts, 0.0, box, out=pts)
        else:
            bad = np.any((pts < 0.0) | (pts > box), axis=1)
            while bad.any():
                pts[bad] = rng.normal(c, s, size=(int(bad.sum()), 3))
                bad = np.any((pts < 0.0) | (pts > box), axis=1)
        parts.append(pts)
    parts.append(rng.uniform(0.0, box, size=(n - n_clustered, 3)))
    pts = np.concatenate(parts, axis=0)
    pts = pts[rng.permutation(n)]
    return np.ascontiguousarray(pts.astype(dtype))


def uniform(n: int, seed: int, dtype=np.float32, box: float = 100.0) -> np.ndarray:
    rng = np.random.default_rng(seed)
    return np.ascontiguousarray(rng.uniform(0.0, box, size=(n, 3)).astype(dtype))


def trajectory(frame: int = 0, n: int = TRAJECTORY_N, seed: int = 2,
               box: float = 160.0) -> np.ndarray:
    """Frame ``frame`` of the periodic trajectory (float64)."""
    rng = np.random.default_rng(seed)
    side = int(np.ceil(n ** (1.0 / 3.0)))
    while side ** 3 < n:
        side += 1
    idx = np.arange(n)
    pts = np.stack([idx % side, (idx // side) % side, idx // (side * side)], axis=1).astype(np.float64)
    pts += rng.normal(0.0, 0.02, size=pts.shape)
    pts = np.mod(pts, box)
    perm = rng.permutation(n)
    for _ in range(frame):
        pts += rng.normal(0.0, 0.02, size=pts.shape)
        pts = np.mod(pts, box)
    # np.mod can return exactly `box` for tiny negative inputs; keep [0, box).
    pts[pts >= box] = 0.0
    return np.ascontiguousarray(pts[perm])


def uneven_specs(count: int = 256, seed: int = 3, lo: float = 1e4, hi: float = 2e6):
    """(n, kind, eb_frac, frame_seed) for each frame of the uneven batch."""
    rng = np.random.default_rng(seed)
    ns = np.floor(np.exp(rng.uniform(np.log(lo), np.log(hi), size=count))).astype(np.int64)
    kinds = rng.integers(0, 3, size=count)
    fracs = np.array([1e-2, 1e-3, 1e-4])[rng.integers(0, 3, size=count)]
    seeds = rng.integers(0, 2**31 - 1, size=count)
    names = ("column", "blobs", "uniform")
    return [(int(n), names[int(k)], float(f), int(s)) for n, k, f, s in zip(ns, kinds, fracs, seeds)]


def make_frame(n: int, kind: str, seed: int, dtype=np.float32) -> np.ndarray:
    if kind == "column":
        return column(n, seed, dtype)
    if kind == "blobs":
        return blobs(n, seed, dtype)
    if kind == "uniform":
        return uniform(n, seed, dtype)
    raise ValueError(f"unknown frame kind {kind!r}")
