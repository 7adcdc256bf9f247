"""Shared helpers for the GPU parity tests: datasets per coordinate type and comparisons."""
from __future__ import annotations

import numpy as np

from oracle import oracle as O

BOX = 100.0
CONFIGS = [
    # (coord, sfc, periodic)
    (O.F32, O.MORTON, False),
    (O.F64, O.MORTON, False),
    (O.F32, O.PEANO_HILBERT, False),
    (O.F64, O.PEANO_HILBERT, False),
    (O.U32, O.PEANO_HILBERT, False),
    (O.U32, O.PEANO_HILBERT, True),
    (O.U64, O.PEANO_HILBERT, False),
    (O.U64, O.PEANO_HILBERT, True),
]
CONFIG_IDS = ["f32-morton", "f64-morton", "f32-ph", "f64-ph", "u32-ph", "u32-ph-per", "u64-ph", "u64-ph-per"]
NAMES = {O.F32: "f32", O.F64: "f64", O.U32: "u32", O.U64: "u64"}


def int_bits(coord):
    return 42 if coord == O.U64 else 21


def to_coord(a, coord, box=BOX):
    """Physical [0, box) -> the coordinate type (integers: B-bit fixed point, as float_to_int_rep)."""
    a = np.asarray(a, np.float64)
    if coord == O.F32:
        return a.astype(np.float32)
    if coord == O.F64:
        return a.astype(np.float64)
    b = int_bits(coord)
    v = np.floor(np.clip(a / box, 0.0, np.nextafter(1.0, 0.0)) * float(1 << b))
    return v.astype(np.uint32 if coord == O.U32 else np.uint64)


def gen(kind: str, n: int, coord, seed: int):
    """The reference test generators' shapes (test/test_self_knn.cpp:271-368) with numpy RNG."""
    rng = np.random.default_rng(seed)
    if kind == "uniform":
        p = rng.uniform(0.0, BOX, (3, n))
    elif kind == "clustered":
        p = np.empty((3, n))
        n1, n2 = int(n * 0.45), int(n * 0.85)
        p[:, :n1] = rng.normal(0.25 * BOX, 0.04 * BOX, (3, n1))
        p[:, n1:n2] = rng.normal(0.75 * BOX, 0.04 * BOX, (3, n2 - n1))
        p[:, n2:] = rng.uniform(0.0, BOX, (3, n - n2))
        p = np.clip(p, 1e-4, BOX - 1e-4)
    elif kind == "degenerate":
        centres = rng.uniform(0.1 * BOX, 0.9 * BOX, (3, 10))
        p = rng.uniform(0.1 * BOX, 0.9 * BOX, (3, n))
        m = int(n * 0.6)
        p[:, :m] = centres[:, np.arange(m) % 10]
    else:
        raise KeyError(kind)
    return tuple(to_coord(a, coord) for a in p)


def radius(r_phys: float, coord):
    if coord in (O.F32, O.F64):
        return r_phys
    return int(r_phys / BOX * float(1 << int_bits(coord)))


def assert_tree_equal(gpu: dict, ot: "O.Tree", n: int):
    names = ["min_x", "max_x", "min_y", "max_y", "min_z", "max_z", "left_child", "right_child", "parent", "id",
             "is_ghost", "orig_idx"]
    for k in names:
        g = gpu[k]
        o = getattr(ot, k)
        if k in ("left_child", "right_child"):
            o = o[:max(n - 1, 0)]
        else:
            o = o[:2 * n - 1]
        assert g.shape == o.shape, (k, g.shape, o.shape)
        if g.dtype.kind == "f":
            assert np.array_equal(g.view(np.uint32 if g.itemsize == 4 else np.uint64),
                                  o.view(np.uint32 if o.itemsize == 4 else np.uint64)), f"tree array {k} differs"
        else:
            assert np.array_equal(g, o), f"tree array {k} differs (first at {np.argmax(g != o)})"


def tree_height(parent: np.ndarray, n: int) -> int:
    """Height from the parent array (root depth 0), vectorised pointer jumping."""
    if n <= 1:
        return 0
    depth = np.zeros(2 * n - 1, np.int64)
    par = parent.astype(np.int64).copy()
    hop = np.where(par >= 0, 1, 0)
    # pointer doubling
    anc = par.copy()
    dist = hop.copy()
    for _ in range(7):
        valid = anc >= 0
        nxt = np.where(valid, anc[np.where(valid, anc, 0)], -1)
        add = np.where(valid, dist[np.where(valid, anc, 0)], 0)
        dist = dist + add
        anc = nxt
    depth = dist
    return int(depth[n - 1:].max())


def dist_bits(a: np.ndarray) -> np.ndarray:
    return a.view(np.uint64) if a.dtype == np.float64 else a
