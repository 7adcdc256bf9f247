"""ctypes wrapper for the reference's own code compiled on the CPU (oracle/_ref, see ref.mk).

TEST INFRASTRUCTURE ONLY.  Each configuration of the reference is a separate shared object;
`available()` is false where the reference sources were not present at build time (the
built objects travel with the repository snapshot, the sources do not).  The API mirrors
oracle.py and returns oracle.Tree objects.
"""
from __future__ import annotations

import ctypes
import os

import numpy as np

from . import oracle as O

_HERE = os.path.dirname(os.path.abspath(__file__))
_REF = os.path.join(_HERE, "_ref")

_NAMES = {
    (O.F32, O.MORTON, False, False): "morton_f32",
    (O.F64, O.MORTON, False, False): "morton_f64",
    (O.F32, O.PEANO_HILBERT, False, False): "ph_f32",
    (O.F64, O.PEANO_HILBERT, False, False): "ph_f64",
    (O.U32, O.PEANO_HILBERT, False, False): "ph_u32",
    (O.U32, O.PEANO_HILBERT, True, False): "ph_u32_per",
    (O.U64, O.PEANO_HILBERT, False, False): "ph_u64",
    (O.U64, O.PEANO_HILBERT, True, False): "ph_u64_per",
    (O.F64, O.MORTON, False, True): "morton_f64_orig",
    (O.U64, O.PEANO_HILBERT, True, True): "ph_u64_per_orig",
}
_libs = {}


def _key(opts: O.Options):
    # floating-point coordinates ignore PERIODIC_BC in the reference (src/hlbvh.hpp:1001-1006)
    per = bool(opts.periodic) and opts.coord in (O.U32, O.U64)
    return (opts.coord, opts.sfc, per, bool(opts.return_orig))


def path(opts: O.Options):
    name = _NAMES.get(_key(opts))
    return None if name is None else os.path.join(_REF, f"libftref_{name}.so")


def available(opts: O.Options) -> bool:
    p = path(opts)
    return p is not None and os.path.exists(p)


def lib(opts: O.Options):
    p = path(opts)
    if p not in _libs:
        L = ctypes.CDLL(p)
        for name in ("ref_compute_bbox", "ref_sfc_encode", "ref_build_bvh", "ref_build_tree", "ref_self_knn",
                     "ref_knn", "ref_range", "ref_maxheap_run", "ref_mergeheap_run"):
            getattr(L, name).restype = ctypes.c_int
        c = [ctypes.c_int() for _ in range(4)]
        L.ref_config(*[ctypes.byref(v) for v in c])
        cfg = tuple(v.value for v in c)
        want = _key(opts)
        assert cfg == (want[0], want[1], int(want[2]), int(want[3])), (p, cfg, want)
        _libs[p] = L
    return _libs[p]


_p = O._p
_c = O._c


def compute_bbox(opts, x, y, z):
    dt = O.NP_COORD[opts.coord]
    x, y, z = _c(x, dt), _c(y, dt), _c(z, dt)
    out = np.zeros(6, dt)
    lib(opts).ref_compute_bbox(_p(x), _p(y), _p(z), ctypes.c_int64(len(x)), _p(out))
    return out


def sfc_encode(opts, x, y, z, bbox=None):
    dt = O.NP_COORD[opts.coord]
    x, y, z = _c(x, dt), _c(y, dt), _c(z, dt)
    n = len(x)
    bb = None if bbox is None else _c(bbox, dt)
    hi = np.zeros(max(n, 1), np.uint64)
    lo = np.zeros(max(n, 1), np.uint64)
    lib(opts).ref_sfc_encode(_p(x), _p(y), _p(z), ctypes.c_int64(n), _p(bb), _p(hi), _p(lo))
    return hi[:n], lo[:n]


def build_bvh(opts, x, y, z, id=None, ghost=None, bbox=None) -> O.Tree:
    dt = O.NP_COORD[opts.coord]
    x, y, z = _c(x, dt), _c(y, dt), _c(z, dt)
    n = len(x)
    t = O.Tree(n, opts.coord)
    idp = None if id is None or len(id) == 0 else _c(id, np.uint32)
    gp = None if ghost is None or len(ghost) == 0 else _c(ghost, np.int8)
    bb = None if bbox is None else _c(bbox, dt)
    ct = t.c()
    rc = lib(opts).ref_build_bvh(_p(x), _p(y), _p(z), ctypes.c_int64(n), _p(idp), _p(gp), _p(bb), ctypes.byref(ct),
                                 _p(t.sorted_hi), _p(t.sorted_lo))
    if rc == 2:
        raise RuntimeError("n > INT_MAX / 2")
    return t


def build_tree(opts, keys_hi, keys_lo, sx, sy, sz) -> O.Tree:
    dt = O.NP_COORD[opts.coord]
    n = len(keys_lo)
    t = O.Tree(n, opts.coord)
    kh = _c(keys_hi if keys_hi is not None else np.zeros(n, np.uint64), np.uint64)
    kl = _c(keys_lo, np.uint64)
    sx, sy, sz = _c(sx, dt), _c(sy, dt), _c(sz, dt)
    ct = t.c()
    lib(opts).ref_build_tree(_p(kh), _p(kl), _p(sx), _p(sy), _p(sz), ctypes.c_int64(n), ctypes.byref(ct))
    return t


def self_knn(opts, tree: O.Tree, k: int, exclude_self=True, leaf_ids=None):
    num = tree.n if leaf_ids is None else len(leaf_ids)
    lid = None if leaf_ids is None else _c(leaf_ids, np.int32)
    idx = np.zeros(max(num * k, 1), np.uint64)
    dist = np.zeros(max(num * k, 1), O.dist_dtype(opts.coord))
    ct = tree.c()
    rc = lib(opts).ref_self_knn(ctypes.byref(ct), _p(lid), ctypes.c_int64(num), ctypes.c_int(k),
                                ctypes.c_int(int(exclude_self)), _p(idx), _p(dist))
    assert rc == 0, rc
    return idx[:num * k].reshape(num, k), dist[:num * k].reshape(num, k)


def knn(opts, tree: O.Tree, qx, qy, qz, k: int, max_k: int = 256):
    dt = O.NP_COORD[opts.coord]
    qx, qy, qz = _c(qx, dt), _c(qy, dt), _c(qz, dt)
    nq = len(qx)
    idx = np.zeros(max(nq * k, 1), np.uint64)
    dist = np.zeros(max(nq * k, 1), O.dist_dtype(opts.coord))
    ct = tree.c()
    rc = lib(opts).ref_knn(ctypes.byref(ct), _p(qx), _p(qy), _p(qz), ctypes.c_int64(nq), ctypes.c_int(k),
                           ctypes.c_int(max_k), _p(idx), _p(dist))
    if rc == 1:
        raise ValueError("k exceeds max_k")
    assert rc == 0, rc
    return idx[:nq * k].reshape(nq, k), dist[:nq * k].reshape(nq, k)


def range_query(opts, tree: O.Tree, qx, qy, qz, rmin, rmax, max_per_q: int):
    dt = O.NP_COORD[opts.coord]
    qx, qy, qz, rmin, rmax = (_c(a, dt) for a in (qx, qy, qz, rmin, rmax))
    nq = len(qx)
    res = np.full(max(nq * max_per_q, 1), -1, np.int32)
    cnt = np.zeros(max(nq, 1), np.int32)
    ct = tree.c()
    lib(opts).ref_range(ctypes.byref(ct), _p(qx), _p(qy), _p(qz), _p(rmin), _p(rmax), ctypes.c_int64(nq), _p(res),
                        _p(cnt), ctypes.c_int(max_per_q))
    return res[:nq * max_per_q].reshape(nq, max_per_q), cnt[:nq]


def maxheap_run(opts, k, d, ix, use_prune=True):
    d = _c(d, np.float64)
    ix = _c(ix, np.int32)
    od = np.zeros(max(k, 1), np.float64)
    oi = np.zeros(max(k, 1), np.int32)
    cnt = ctypes.c_int(0)
    rc = lib(opts).ref_maxheap_run(ctypes.c_int(k), _p(d), _p(ix), ctypes.c_int(len(d)), ctypes.c_int(int(use_prune)),
                                   _p(od), _p(oi), ctypes.byref(cnt))
    assert rc == 0
    return od[:k], oi[:k], cnt.value


def mergeheap_run(opts, k, cap, d_rounds, ix_rounds):
    d = _c(d_rounds, np.float64).reshape(-1)
    ix = _c(ix_rounds, np.int32).reshape(-1)
    od = np.zeros(cap, np.float64)
    oi = np.zeros(cap, np.int32)
    lib(opts).ref_mergeheap_run(ctypes.c_int(k), ctypes.c_int(cap), _p(d), _p(ix), ctypes.c_int(len(d) // 32), _p(od),
                                _p(oi))
    return od, oi
