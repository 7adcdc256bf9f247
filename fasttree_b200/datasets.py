"""Seeded synthetic point sets with the shapes of the benchmark configurations.

The reference benchmarks on HDF5 cosmological snapshots that are not available here
(test/benchmark/config.txt); these generators stand in for them with seeded inputs of the
stated sizes and distributions.  All randomness comes from numpy's PCG64 Generator, so a
seed gives the same points on every machine with the same numpy.
"""
from __future__ import annotations

import numpy as np

FIXED_BITS = 40  # "2^40 per side" fixed-point scale of the clustered int64 workloads


def uniform(n: int, seed: int = 1, dtype=np.float64):
    """n points i.i.d. uniform in [0,1)^3 (x, y, z arrays)."""
    rng = np.random.default_rng(seed)
    p = rng.random((3, n))
    return tuple(np.ascontiguousarray(a.astype(dtype)) for a in p)


def _largest_remainder(weights: np.ndarray, total: int) -> np.ndarray:
    share = weights / weights.sum() * total
    base = np.floor(share).astype(np.int64)
    rem = total - int(base.sum())
    if rem > 0:
        order = np.argsort(-(share - base), kind="stable")
        base[order[:rem]] += 1
    return base


def _plummer_offsets(rng, counts: np.ndarray, scale: np.ndarray):
    """Isotropic Plummer-sphere offsets: r = a / sqrt(u^(-2/3) - 1)."""
    m = int(counts.sum())
    a = np.repeat(scale, counts)
    u = rng.random(m)
    u = np.clip(u, 1e-12, 1.0 - 1e-12)
    r = a / np.sqrt(u ** (-2.0 / 3.0) - 1.0)
    cos_t = 2.0 * rng.random(m) - 1.0
    sin_t = np.sqrt(np.maximum(0.0, 1.0 - cos_t * cos_t))
    phi = 2.0 * np.pi * rng.random(m)
    return r * sin_t * np.cos(phi), r * sin_t * np.sin(phi), r * cos_t


def clustered(n: int, n_spheres: int = 20000, seed: int = 2, clustered_frac: float = 0.7):
    """Clustered points in the periodic unit box (float64 in [0,1)).

    clustered_frac of the points sit in n_spheres Plummer spheres with uniform centres,
    log-uniform scale radii in [1e-4, 1e-2] and member counts drawn from dN/dM ~ M^-1.9
    (weights u^(-1/0.9), allocated by largest remainder); the rest are uniform.  Positions
    wrap modulo 1.
    """
    rng = np.random.default_rng(seed)
    n_cl = int(round(clustered_frac * n))
    centres = rng.random((n_spheres, 3))
    scale = 10.0 ** rng.uniform(-4.0, -2.0, n_spheres)
    w = rng.random(n_spheres)
    w = np.clip(w, 1e-12, 1.0) ** (-1.0 / 0.9)
    counts = _largest_remainder(w, n_cl)
    ox, oy, oz = _plummer_offsets(rng, counts, scale)
    cx = np.repeat(centres[:, 0], counts) + ox
    cy = np.repeat(centres[:, 1], counts) + oy
    cz = np.repeat(centres[:, 2], counts) + oz
    ux, uy, uz = rng.random((3, n - n_cl))
    x = np.mod(np.concatenate([cx, ux]), 1.0)
    y = np.mod(np.concatenate([cy, uy]), 1.0)
    z = np.mod(np.concatenate([cz, uz]), 1.0)
    # mod can round up to exactly 1.0 for tiny negative inputs
    for a in (x, y, z):
        a[a >= 1.0] = 0.0
    perm = rng.permutation(n)
    return x[perm], y[perm], z[perm]


def to_fixed(a: np.ndarray, bits: int = FIXED_BITS) -> np.ndarray:
    """Unit-box coordinate -> fixed point with 2^bits cells per side (uint64)."""
    v = np.floor(np.asarray(a, np.float64) * float(1 << bits))
    return np.clip(v, 0, float((1 << bits) - 1)).astype(np.uint64)


def clustered_fixed(n: int, n_spheres: int = 20000, seed: int = 2, bits: int = FIXED_BITS):
    """The clustered set in uint64 fixed point (bits per side; 40 by default, 42 reaches
    the periodic wrap of 42-bit Peano-Hilbert integer coordinates)."""
    x, y, z = clustered(n, n_spheres, seed)
    return to_fixed(x, bits), to_fixed(y, bits), to_fixed(z, bits)


def external_queries(px, py, pz, nq: int, seed: int = 3, sigma: float = 1e-4):
    """Half uniform in [0,1)^3, half jittered copies of particles (Gaussian sigma)."""
    rng = np.random.default_rng(seed)
    nu = nq // 2
    nj = nq - nu
    u = rng.random((3, nu))
    pick = rng.integers(0, len(px), nj)
    j = np.stack([np.asarray(px)[pick], np.asarray(py)[pick], np.asarray(pz)[pick]]).astype(np.float64)
    j = j + rng.normal(0.0, sigma, (3, nj))
    q = np.concatenate([u, j], axis=1)
    dt = np.asarray(px).dtype
    return tuple(np.ascontiguousarray(a.astype(dt)) for a in q)


def batched_set_sizes(n_sets: int = 4096, seed: int = 4, median: float = 8000.0, sigma: float = 1.2,
                      lo: int = 256, hi: int = 500_000) -> np.ndarray:
    rng = np.random.default_rng(seed)
    s = np.exp(np.log(median) + sigma * rng.standard_normal(n_sets))
    return np.clip(np.round(s), lo, hi).astype(np.int64)


def batched_sets(n_sets: int = 4096, seed: int = 4, scale: float = 0.05, sizes=None):
    """Independent Plummer spheres (scale radius 0.05, centred at 0.5) in float32, each
    truncated to the unit box by resampling.  Returns (x, y, z, offsets) with set s at
    [offsets[s], offsets[s+1])."""
    if sizes is None:
        sizes = batched_set_sizes(n_sets, seed)
    rng = np.random.default_rng(seed + 1000)
    total = int(sizes.sum())
    out = np.empty((3, total), np.float32)
    filled = 0
    need = total
    buf = []
    while need > 0:
        m = int(need * 1.05) + 64
        ox, oy, oz = _plummer_offsets(rng, np.array([m]), np.array([scale]))
        p = np.stack([ox, oy, oz]) + 0.5
        ok = np.all((p >= 0.0) & (p < 1.0), axis=0)
        p = p[:, ok].astype(np.float32)
        ok32 = np.all((p >= 0.0) & (p < 1.0), axis=0)
        p = p[:, ok32][:, :need]
        buf.append(p)
        need -= p.shape[1]
    allp = np.concatenate(buf, axis=1)
    out[:, :] = allp[:, :total]
    offsets = np.zeros(len(sizes) + 1, np.int64)
    offsets[1:] = np.cumsum(sizes)
    filled = total
    assert filled == offsets[-1]
    return out[0].copy(), out[1].copy(), out[2].copy(), offsets
