"""ctypes wrapper for the CPU oracle (oracle/ft_oracle.cpp).

TEST INFRASTRUCTURE ONLY: the checker that the CUDA library is compared against.  The
library never imports this module; tests/, the smoke check and bench.py's CPU-baseline leg
do.  The restated reference functions and the lines they follow are listed in
ft_oracle.cpp.
"""
from __future__ import annotations

import ctypes
import os
import subprocess
from dataclasses import dataclass

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "_build", "libftoracle.so")

F32, F64, U32, U64 = 0, 1, 2, 3
MORTON, PEANO_HILBERT = 0, 1

NP_COORD = {F32: np.float32, F64: np.float64, U32: np.uint32, U64: np.uint64}


def dist_dtype(coord: int):
    """dist_t of the reference: double for float coordinates, uint64 for integers."""
    return np.float64 if coord in (F32, F64) else np.uint64


def missing_dist(coord: int):
    """type_identity_max<dist_t>() -- the distance written for a missing neighbour."""
    return -np.finfo(np.float64).max if coord in (F32, F64) else np.uint64(0)


MISSING_IDX = np.uint64(0xFFFFFFFFFFFFFFFF)


class _Options(ctypes.Structure):
    _fields_ = [("coord_type", ctypes.c_int32), ("sfc_type", ctypes.c_int32),
                ("periodic", ctypes.c_int32), ("return_orig_indices", ctypes.c_int32)]


class _Tree(ctypes.Structure):
    _fields_ = [(n, ctypes.c_void_p) for n in ("min_x", "max_x", "min_y", "max_y", "min_z", "max_z",
                                                "left_child", "right_child", "parent", "id",
                                                "is_ghost", "orig_idx")] + [("num_leaves", ctypes.c_int64)]


@dataclass(frozen=True)
class Options:
    coord: int = F64
    sfc: int = MORTON
    periodic: bool = False
    return_orig: bool = False

    def c(self) -> _Options:
        return _Options(self.coord, self.sfc, int(self.periodic), int(self.return_orig))


_lib = None


def build_library() -> str:
    subprocess.run(["make", "-s", "-C", _HERE], check=True)
    return _LIB_PATH


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(_LIB_PATH) or os.path.getmtime(_LIB_PATH) < os.path.getmtime(
                os.path.join(_HERE, "ft_oracle.cpp")):
            build_library()
        _lib = ctypes.CDLL(_LIB_PATH)
        for name in ("ora_compute_bbox", "ora_sfc_encode", "ora_build_bvh", "ora_build_tree",
                     "ora_self_knn", "ora_knn", "ora_range", "ora_point_dist", "ora_maxheap_run",
                     "ora_mergeheap_run", "ora_set_threads"):
            getattr(_lib, name).restype = ctypes.c_int
    return _lib


def set_threads(n: int) -> int:
    return lib().ora_set_threads(int(n))


def _p(a):
    return None if a is None else a.ctypes.data_as(ctypes.c_void_p)


def _c(a, dtype):
    return np.ascontiguousarray(a, dtype=dtype)


class Tree:
    """Flat tree with TreeSoA's layout: internal nodes [0, n-2], leaves [n-1, 2n-2]."""

    def __init__(self, n: int, coord: int):
        self.n = int(n)
        self.coord = coord
        tot = max(2 * self.n - 1, 1)
        dt = NP_COORD[coord]
        self.min_x, self.max_x, self.min_y, self.max_y, self.min_z, self.max_z = (
            np.zeros(tot, dt) for _ in range(6))
        self.left_child = np.zeros(max(self.n - 1, 1), np.int32)
        self.right_child = np.zeros(max(self.n - 1, 1), np.int32)
        self.parent = np.full(tot, -1, np.int32)
        self.id = np.zeros(tot, np.uint32)
        self.is_ghost = np.zeros(tot, np.int8)
        self.orig_idx = np.zeros(tot, np.int32)
        self.sorted_hi = np.zeros(max(self.n, 1), np.uint64)
        self.sorted_lo = np.zeros(max(self.n, 1), np.uint64)
        self.bbox = np.zeros(6, dt)

    def c(self) -> _Tree:
        t = _Tree()
        for name in ("min_x", "max_x", "min_y", "max_y", "min_z", "max_z", "left_child",
                     "right_child", "parent", "id", "is_ghost", "orig_idx"):
            setattr(t, name, getattr(self, name).ctypes.data)
        t.num_leaves = self.n
        return t

    @property
    def num_internal(self):
        return max(self.n - 1, 0)

    def leaf_coords(self):
        s = self.num_internal
        return self.min_x[s:s + self.n], self.min_y[s:s + self.n], self.min_z[s:s + self.n]


def compute_bbox(opts: Options, x, y, z):
    dt = NP_COORD[opts.coord]
    x, y, z = _c(x, dt), _c(y, dt), _c(z, dt)
    out = np.zeros(6, dt)
    rc = lib().ora_compute_bbox(ctypes.byref(opts.c()), _p(x), _p(y), _p(z), ctypes.c_int64(len(x)), _p(out))
    assert rc == 0, rc
    return out


def sfc_encode(opts: Options, x, y, z, bbox=None):
    """Keys as (hi, lo) uint64 arrays (hi is zero for 63-bit keys)."""
    dt = NP_COORD[opts.coord]
    x, y, z = _c(x, dt), _c(y, dt), _c(z, dt)
    n = len(x)
    bb = None if bbox is None else _c(bbox, dt)
    hi = np.zeros(max(n, 1), np.uint64)
    lo = np.zeros(max(n, 1), np.uint64)
    rc = lib().ora_sfc_encode(ctypes.byref(opts.c()), _p(x), _p(y), _p(z), ctypes.c_int64(n), _p(bb),
                              _p(hi), _p(lo))
    assert rc == 0, rc
    return hi[:n], lo[:n]


def build_bvh(opts: Options, x, y, z, id=None, ghost=None, bbox=None, keys=None) -> Tree:
    """Build on the CPU.  keys=(hi, lo) arrays are caller keys, sorted in place."""
    dt = NP_COORD[opts.coord]
    x, y, z = _c(x, dt), _c(y, dt), _c(z, dt)
    n = len(x)
    t = Tree(n, opts.coord)
    idp = None if id is None or len(id) == 0 else _c(id, np.uint32)
    gp = None if ghost is None or len(ghost) == 0 else _c(ghost, np.int8)
    bb = None if bbox is None else _c(bbox, dt)
    khi = klo = None
    if keys is not None:
        khi, klo = keys
        assert khi.dtype == np.uint64 and klo.dtype == np.uint64 and khi.flags.c_contiguous
    ct = t.c()
    rc = lib().ora_build_bvh(ctypes.byref(opts.c()), _p(x), _p(y), _p(z), ctypes.c_int64(n), _p(idp),
                             _p(gp), _p(bb), _p(khi), _p(klo), ctypes.byref(ct), _p(t.sorted_hi),
                             _p(t.sorted_lo), _p(t.bbox))
    if rc == 2:
        raise RuntimeError("Particle count n exceeds maximum supported tree size (INT_MAX / 2).")
    assert rc == 0, rc
    return t


def build_tree(opts: Options, keys_hi, keys_lo, sx=None, sy=None, sz=None, sid=None, sghost=None,
               sorig=None) -> Tree:
    dt = NP_COORD[opts.coord]
    n = len(keys_lo)
    t = Tree(n, opts.coord)
    kh = _c(keys_hi if keys_hi is not None else np.zeros(n, np.uint64), np.uint64)
    kl = _c(keys_lo, np.uint64)
    args = [None if a is None else _c(a, dt) for a in (sx, sy, sz)]
    sid = None if sid is None else _c(sid, np.uint32)
    sghost = None if sghost is None else _c(sghost, np.int8)
    sorig = None if sorig is None else _c(sorig, np.int32)
    ct = t.c()
    rc = lib().ora_build_tree(ctypes.byref(opts.c()), ctypes.byref(ct), _p(kh), _p(kl), *[_p(a) for a in args],
                              _p(sid), _p(sghost), _p(sorig))
    assert rc == 0, rc
    return t


def self_knn(opts: Options, tree: Tree, k: int, exclude_self=True, leaf_ids=None):
    num = tree.n if leaf_ids is None else len(leaf_ids)
    lid = None if leaf_ids is None else _c(leaf_ids, np.int32)
    idx = np.zeros(max(num * k, 1), np.uint64)
    dist = np.zeros(max(num * k, 1), dist_dtype(opts.coord))
    ct = tree.c()
    rc = lib().ora_self_knn(ctypes.byref(opts.c()), ctypes.byref(ct), _p(lid), ctypes.c_int64(num),
                            ctypes.c_int(k), ctypes.c_int(int(exclude_self)), _p(idx), _p(dist))
    assert rc == 0, rc
    return idx[:num * k].reshape(num, k), dist[:num * k].reshape(num, k)


def knn(opts: Options, tree: Tree, qx, qy, qz, k: int, max_k: int = 256):
    dt = NP_COORD[opts.coord]
    qx, qy, qz = _c(qx, dt), _c(qy, dt), _c(qz, dt)
    nq = len(qx)
    idx = np.zeros(max(nq * k, 1), np.uint64)
    dist = np.zeros(max(nq * k, 1), dist_dtype(opts.coord))
    ct = tree.c()
    rc = lib().ora_knn(ctypes.byref(opts.c()), ctypes.byref(ct), _p(qx), _p(qy), _p(qz), ctypes.c_int64(nq),
                       ctypes.c_int(k), ctypes.c_int(max_k), _p(idx), _p(dist))
    if rc == 1:
        raise ValueError("k exceeds max_k")
    assert rc == 0, rc
    return idx[:nq * k].reshape(nq, k), dist[:nq * k].reshape(nq, k)


def range_query(opts: Options, tree: Tree, qx, qy, qz, rmin, rmax, max_per_q: int):
    dt = NP_COORD[opts.coord]
    qx, qy, qz, rmin, rmax = (_c(a, dt) for a in (qx, qy, qz, rmin, rmax))
    nq = len(qx)
    res = np.full(max(nq * max_per_q, 1), -1, np.int32)
    cnt = np.zeros(max(nq, 1), np.int32)
    ct = tree.c()
    rc = lib().ora_range(ctypes.byref(opts.c()), ctypes.byref(ct), _p(qx), _p(qy), _p(qz), _p(rmin), _p(rmax),
                         ctypes.c_int64(nq), _p(res), _p(cnt), ctypes.c_int(max_per_q))
    assert rc == 0, rc
    return res[:nq * max_per_q].reshape(nq, max_per_q), cnt[:nq]


def point_dist(opts: Options, p3, box6):
    dt = NP_COORD[opts.coord]
    p3, box6 = _c(p3, dt), _c(box6, dt)
    out = np.zeros(1, dist_dtype(opts.coord))
    rc = lib().ora_point_dist(ctypes.byref(opts.c()), _p(p3), _p(box6), _p(out))
    assert rc == 0
    return out[0]


def maxheap_run(k: int, d, ix, use_prune=True):
    d = _c(d, np.float64)
    ix = _c(ix, np.int32)
    od = np.zeros(max(k, 1), np.float64)
    oi = np.zeros(max(k, 1), np.int32)
    cnt = ctypes.c_int(0)
    lib().ora_maxheap_run(ctypes.c_int(k), _p(d), _p(ix), ctypes.c_int(len(d)), ctypes.c_int(int(use_prune)),
                          _p(od), _p(oi), ctypes.byref(cnt))
    return od[:k], oi[:k], cnt.value


def mergeheap_run(k: int, cap: int, d_rounds, ix_rounds):
    d = _c(d_rounds, np.float64).reshape(-1)
    ix = _c(ix_rounds, np.int32).reshape(-1)
    rounds = len(d) // 32
    od = np.zeros(cap, np.float64)
    oi = np.zeros(cap, np.int32)
    lib().ora_mergeheap_run(ctypes.c_int(k), ctypes.c_int(cap), _p(d), _p(ix), ctypes.c_int(rounds), _p(od), _p(oi))
    return od, oi
