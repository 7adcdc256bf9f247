"""Python mirror of FastTree's C++ API (src/hlbvh.hpp) over the C ABI.

Names and argument meaning follow the reference: particles, BoundingBox, TreeSoA, TreePool,
compute_bbox, sfc_encode, build_tree, build_bvh, knn_query, self_knn_query,
self_knn_query_subset, range_query.  The sycl::queue argument becomes a Context (device +
compile-time options of the reference, now runtime fields) and an optional CUDA stream.
Errors raise ValueError where the reference throws std::invalid_argument and RuntimeError
where it throws std::runtime_error.

Arrays may be torch tensors (CUDA or CPU) or numpy arrays; host arrays are staged by the
library as the reference stages non-USM pointers.  Query outputs of self_knn_query* must be
device tensors (the reference requires USM there and does not wait).
"""
from __future__ import annotations

import ctypes
from dataclasses import dataclass, field
from typing import Optional, Sequence

import numpy as np
import torch

from . import capi
from .capi import F32, F64, U32, U64, MORTON, PEANO_HILBERT, check, lib

_COORD_NAMES = {"f32": F32, "float": F32, "float32": F32, "f64": F64, "double": F64, "float64": F64,
                "u32": U32, "uint32": U32, "u64": U64, "uint64": U64}
_SFC_NAMES = {"morton": MORTON, "ph": PEANO_HILBERT, "peano_hilbert": PEANO_HILBERT, "hilbert": PEANO_HILBERT}
TORCH_COORD = {F32: torch.float32, F64: torch.float64, U32: torch.uint32, U64: torch.uint64}
NP_COORD = {F32: np.float32, F64: np.float64, U32: np.uint32, U64: np.uint64}


def dist_torch_dtype(coord: int):
    """dist_t: double for floating-point coordinates, uint64 for integer coordinates."""
    return torch.float64 if coord in (F32, F64) else torch.uint64


def _stream_handle(stream) -> int:
    if stream is None:
        return torch.cuda.current_stream().cuda_stream
    if isinstance(stream, torch.cuda.Stream):
        return stream.cuda_stream
    return int(stream)


def _ptr(a) -> Optional[int]:
    if a is None:
        return None
    if isinstance(a, torch.Tensor):
        assert a.is_contiguous(), "arrays must be contiguous"
        return a.data_ptr()
    if isinstance(a, np.ndarray):
        assert a.flags.c_contiguous, "arrays must be contiguous"
        return a.ctypes.data
    raise TypeError(f"unsupported array type {type(a)}")


def _rows(a, rows: int, width: int):
    """The first rows x width entries of a flat result buffer (which may be larger), as rows."""
    if rows * width == 0:
        return a
    flat = a.reshape(-1) if isinstance(a, torch.Tensor) else np.asarray(a).reshape(-1)
    return flat[: rows * width].reshape(rows, width)


def _as_coord(a, coord: int):
    """Contiguous array of the coordinate type (keeps device/host placement)."""
    if isinstance(a, torch.Tensor):
        t = a if a.dtype == TORCH_COORD[coord] else a.to(TORCH_COORD[coord])
        return t.contiguous()
    return np.ascontiguousarray(a, dtype=NP_COORD[coord])


class Context:
    """Device plus the reference's compile-time configuration (CMakeLists.txt:63-125)."""

    def __init__(self, coord="f64", sfc="morton", periodic=False, return_orig_indices=False,
                 host_readable_tree=False, device: Optional[int] = None):
        self.coord = _COORD_NAMES[coord] if isinstance(coord, str) else int(coord)
        self.sfc = _SFC_NAMES[sfc] if isinstance(sfc, str) else int(sfc)
        self.periodic = bool(periodic)
        self.return_orig_indices = bool(return_orig_indices)
        self.device = torch.cuda.current_device() if device is None else int(device)
        o = capi.FtOptions(self.coord, self.sfc, int(self.periodic), int(self.return_orig_indices),
                           int(host_readable_tree))
        h = ctypes.c_void_p()
        self._h = None
        _call(lib().ft_context_create(ctypes.byref(o), self.device, ctypes.byref(h)))
        self._h = h

    @property
    def handle(self):
        return self._h

    @property
    def is_float(self):
        return self.coord in (F32, F64)

    def torch_coord(self):
        return TORCH_COORD[self.coord]

    def query_stats(self):
        s = capi.FtQueryStats()
        check(lib().ft_get_query_stats(self._h, ctypes.byref(s)))
        return {"queries": s.queries, "replayed": s.replayed, "visits": s.reserved[0],
                "bound_misses": s.reserved[1], "rerun_visits": s.reserved[2]}

    def set_range_walk(self, walk: int):
        """range_query's walk on trees of height <= 62 (ft_set_range_walk): 0 default (rows by
        a 4-wide walk per query that stops once the row is full, full rows counted by a warp's
        queries together when they lie close, where the 4-wide walk applies), 1 binary walk per
        query, 2 a warp's queries together when their balls overlap, 3 4-wide walk per query,
        4 as 0 with every group counted together."""
        _call(lib().ft_set_range_walk(self._h, int(walk)))

    def profile_builds(self, enable: bool = True):
        """Stage timing of later builds on this context (ft_set_build_profiling)."""
        _call(lib().ft_set_build_profiling(self._h, int(bool(enable))))

    def build_profile(self) -> dict:
        """Stage times (ms) of the last profiled build (ft_get_build_profile; synchronises)."""
        p = capi.FtBuildProfile()
        _call(lib().ft_get_build_profile(self._h, ctypes.byref(p)))
        return p.as_dict()

    def check_device_status(self, stream=None):
        """Synchronises the stream and raises what the kernels recorded (ft_check_device_status)."""
        _call(lib().ft_check_device_status(self._h, _stream_handle(stream)))

    def replayed_queries(self) -> np.ndarray:
        """Output rows the last fast-walk query on this context handed to the reference
        traversal (sorted; empty after a plain-method call).  Synchronises the device."""
        cnt = ctypes.c_size_t(0)
        check(lib().ft_get_replayed_queries(self._h, None, 0, ctypes.byref(cnt)))
        rows = np.empty(cnt.value, dtype=np.int32)
        if cnt.value:
            check(lib().ft_get_replayed_queries(self._h, rows.ctypes.data_as(ctypes.c_void_p), cnt.value,
                                                ctypes.byref(cnt)))
        return np.sort(rows[: cnt.value])

    def close(self):
        if getattr(self, "_h", None):
            lib().ft_context_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


@dataclass
class particles:
    """SoA particle input (src/hlbvh.hpp:26-34)."""
    pos_x: object
    pos_y: object
    pos_z: object
    id: Optional[object] = None
    is_ghost: Optional[object] = None


@dataclass
class BoundingBox:
    min_x: float
    max_x: float
    min_y: float
    max_y: float
    min_z: float
    max_z: float

    def array(self, coord: int) -> np.ndarray:
        return np.array([self.min_x, self.max_x, self.min_y, self.max_y, self.min_z, self.max_z],
                        dtype=NP_COORD[coord])


class _RawCuda:
    """__cuda_array_interface__ view of library-owned device memory."""

    def __init__(self, ptr: int, n: int, dtype: np.dtype):
        self.__cuda_array_interface__ = {"shape": (int(n),), "typestr": np.dtype(dtype).str,
                                         "data": (int(ptr), False), "version": 3, "strides": None}


class TreeSoA:
    """Flat tree (src/hlbvh.hpp:609-673).  Arrays are exposed as zero-copy torch tensors."""

    def __init__(self, ctx: Context, n: int):
        self.ctx = ctx
        p = ctypes.POINTER(capi.FtTree)()
        check(lib().ft_tree_create(ctx.handle, int(n), ctypes.byref(p)))
        self._p = p

    @property
    def c(self):
        return self._p

    @property
    def num_leaves(self) -> int:
        return int(self._p.contents.num_leaves)

    @property
    def num_internal(self) -> int:
        return int(self._p.contents.num_internal)

    @property
    def capacity(self) -> int:
        return int(self._p.contents.capacity)

    def _view(self, name: str, count: int, dtype) -> torch.Tensor:
        ptr = getattr(self._p.contents, name)
        if not ptr or count == 0:
            return torch.empty(0, dtype=torch.from_numpy(np.zeros(0, dtype)).dtype, device=f"cuda:{self.ctx.device}")
        return torch.as_tensor(_RawCuda(ptr, count, dtype), device=f"cuda:{self.ctx.device}")

    def array(self, name: str) -> torch.Tensor:
        n = self.num_leaves
        tot = 2 * n - 1 if n > 0 else 0
        if name in ("min_x", "max_x", "min_y", "max_y", "min_z", "max_z"):
            return self._view(name, tot, NP_COORD[self.ctx.coord])
        if name in ("left_child", "right_child"):
            return self._view(name, max(n - 1, 0), np.int32)
        if name in ("parent", "orig_idx"):
            return self._view(name, tot, np.int32)
        if name == "id":
            return self._view(name, tot, np.uint32)
        if name == "is_ghost":
            return self._view(name, tot, np.int8)
        raise KeyError(name)

    def __getattr__(self, name):
        if name in ("min_x", "max_x", "min_y", "max_y", "min_z", "max_z", "left_child", "right_child",
                    "parent", "id", "is_ghost", "orig_idx"):
            return self.array(name)
        raise AttributeError(name)

    def to_numpy(self) -> dict:
        torch.cuda.synchronize(self.ctx.device)
        return {k: self.array(k).cpu().numpy() for k in ("min_x", "max_x", "min_y", "max_y", "min_z", "max_z",
                                                          "left_child", "right_child", "parent", "id",
                                                          "is_ghost", "orig_idx")}

    def leaf_coords(self):
        s, n = self.num_internal, self.num_leaves
        return self.min_x[s:s + n], self.min_y[s:s + n], self.min_z[s:s + n]

    def height(self) -> int:
        h = ctypes.c_int(0)
        check(lib().ft_tree_height(self.ctx.handle, self._p, ctypes.byref(h)))
        return h.value

    def export_size(self) -> int:
        """Bytes of the serialised tree (ft_tree_export)."""
        size = ctypes.c_size_t(0)
        _call(lib().ft_tree_export(self.ctx.handle, self._p, None, ctypes.byref(size), _stream_handle(None)))
        return size.value

    def export(self, out: Optional[torch.Tensor] = None, stream=None) -> torch.Tensor:
        """The tree in the library's serialised form (ft_tree_export) as a uint8 tensor (host
        memory unless `out`, of sufficient size, is given, e.g. a device tensor)."""
        if out is None:
            out = torch.empty(self.export_size(), dtype=torch.uint8)
        cap = ctypes.c_size_t(out.numel())
        _call(lib().ft_tree_export(self.ctx.handle, self._p, _ptr(out), ctypes.byref(cap), _stream_handle(stream)))
        return out[:cap.value]

    def save(self, path: str):
        """Writes the serialised tree to a file."""
        with open(path, "wb") as f:
            f.write(self.export().numpy().tobytes())

    def free(self):
        if getattr(self, "_p", None):
            lib().ft_tree_destroy(self.ctx.handle, self._p)
            self._p = None

    def __del__(self):
        try:
            self.free()
        except Exception:
            pass


class TreePool:
    """Persistent tree that reallocates only when n exceeds capacity (src/hlbvh.hpp:682-715)."""

    def __init__(self, ctx: Context):
        self.ctx = ctx
        self.tree: Optional[TreeSoA] = None

    def ensure(self, n: int) -> TreeSoA:
        if self.tree is None:
            self.tree = TreeSoA(self.ctx, 0)
        check(lib().ft_tree_ensure(self.ctx.handle, self.tree.c, int(n)))
        return self.tree

    @property
    def capacity(self):
        return 0 if self.tree is None else self.tree.capacity

    def free_all(self):
        if self.tree is not None:
            self.tree.free()
            self.tree = None


def _raise_for(e: capi.FastTreeError):
    if e.status == capi.FT_ERR_INVALID_ARGUMENT:
        raise ValueError(str(e)) from e
    if e.status in (capi.FT_ERR_RUNTIME, capi.FT_ERR_TIMEOUT):
        raise RuntimeError(str(e)) from e
    if e.status == capi.FT_ERR_OUT_OF_MEMORY:
        raise MemoryError(str(e)) from e
    raise e


def _call(status):
    try:
        check(status)
    except capi.FastTreeError as e:
        _raise_for(e)


def compute_bbox(ctx: Context, pos_x, pos_y, pos_z, n: Optional[int] = None, stream=None) -> np.ndarray:
    """compute_bbox (src/hlbvh.hpp:462-572): {min_x, max_x, min_y, max_y, min_z, max_z}."""
    x, y, z = (_as_coord(a, ctx.coord) for a in (pos_x, pos_y, pos_z))
    n = len(x) if n is None else int(n)
    out = np.zeros(6, NP_COORD[ctx.coord])
    _call(lib().ft_compute_bbox(ctx.handle, _ptr(x), _ptr(y), _ptr(z), n, out.ctypes.data, _stream_handle(stream)))
    return out


def ref_key_dtype(ctx: Context):
    """numpy dtype of one reference sfc_key: uint64 (Morton), 3 x uint32 or 3 x uint64."""
    if ctx.sfc == MORTON:
        return np.dtype(np.uint64), 1
    return (np.dtype(np.uint64), 3) if ctx.coord == U64 else (np.dtype(np.uint32), 3)


def sfc_encode(ctx: Context, pos_x, pos_y, pos_z, bbox=None, keys=None, stream=None):
    """sfc_encode (src/hlbvh.hpp:357-423); keys in the reference's sfc_key layout, shape (n, words)."""
    x, y, z = (_as_coord(a, ctx.coord) for a in (pos_x, pos_y, pos_z))
    n = len(x)
    dt, words = ref_key_dtype(ctx)
    if keys is None:
        keys = np.zeros((n, words), dt)
    bb = None
    if bbox is not None:
        bb = bbox.array(ctx.coord) if isinstance(bbox, BoundingBox) else np.ascontiguousarray(bbox, NP_COORD[ctx.coord])
    _call(lib().ft_sfc_encode(ctx.handle, _ptr(x), _ptr(y), _ptr(z), n, _ptr(keys),
                              None if bb is None else bb.ctypes.data, _stream_handle(stream)))
    return keys


def build_bvh(ctx: Context, p, tree: TreeSoA, bbox=None, key=None, scratch=None, stream=None) -> TreeSoA:
    """build_bvh (src/hlbvh.hpp:2165-2302).  key: caller keys (reference layout), sorted in place.
    `scratch` is accepted for signature parity; scratch is owned by the tree."""
    if not isinstance(p, particles):
        p = particles(*p)
    x, y, z = (_as_coord(a, ctx.coord) for a in (p.pos_x, p.pos_y, p.pos_z))
    n = len(x)
    ids = None
    if p.id is not None and len(p.id) > 0:
        if isinstance(p.id, torch.Tensor):
            assert p.id.element_size() == 4, "id must hold 32-bit values"
            ids = p.id.contiguous()
        else:
            ids = np.ascontiguousarray(p.id, np.uint32)
    gh = None
    if p.is_ghost is not None and len(p.is_ghost) > 0:
        gh = p.is_ghost.to(torch.int8).contiguous() if isinstance(p.is_ghost, torch.Tensor) else \
            np.ascontiguousarray(p.is_ghost, np.int8)
    bb = None
    if bbox is not None:
        bb = bbox.array(ctx.coord) if isinstance(bbox, BoundingBox) else np.ascontiguousarray(bbox, NP_COORD[ctx.coord])
    if tree.capacity < n:
        raise ValueError("tree capacity is smaller than the particle count")
    _call(lib().ft_build_bvh(ctx.handle, _ptr(x), _ptr(y), _ptr(z), n, _ptr(ids), _ptr(gh),
                             None if bb is None else bb.ctypes.data, _ptr(key), tree.c, _stream_handle(stream)))
    return tree


def import_tree(ctx: Context, data, tree: Optional[TreeSoA] = None, stream=None) -> TreeSoA:
    """A tree from its serialised form (ft_tree_import): bytes, a numpy array or a uint8 tensor
    (host or device).  A new TreeSoA of the stored size unless `tree` is given."""
    if isinstance(data, (bytes, bytearray, memoryview)):
        data = np.frombuffer(data, np.uint8)
    if isinstance(data, np.ndarray):
        data = np.ascontiguousarray(data, np.uint8)
    if tree is None:
        head = data[:48].cpu().numpy() if isinstance(data, torch.Tensor) else data[:48]
        n = int(np.frombuffer(np.ascontiguousarray(head).tobytes()[40:48], np.uint64)[0]) if len(head) >= 48 else 0
        tree = TreeSoA(ctx, max(n, 1))
    _call(lib().ft_tree_import(ctx.handle, _ptr(data), int(data.numel() if isinstance(data, torch.Tensor)
                                                               else data.size), tree.c, _stream_handle(stream)))
    return tree


def load_tree(ctx: Context, path: str, tree: Optional[TreeSoA] = None) -> TreeSoA:
    """A tree saved by TreeSoA.save."""
    with open(path, "rb") as f:
        return import_tree(ctx, f.read(), tree)


def refit_bvh(ctx: Context, p, tree: TreeSoA, leaf_order: bool = False, stream=None) -> TreeSoA:
    """Refit-only update for moved points (ft_refit_bvh): new positions of the same points,
    in the build's input order (or leaf order); keys and topology are kept.  Blocking."""
    if not isinstance(p, particles):
        p = particles(*p)
    x, y, z = (_as_coord(a, ctx.coord) for a in (p.pos_x, p.pos_y, p.pos_z))
    _call(lib().ft_refit_bvh(ctx.handle, _ptr(x), _ptr(y), _ptr(z), len(x), int(bool(leaf_order)), tree.c,
                             _stream_handle(stream)))
    return tree


def build_tree(ctx: Context, tree: TreeSoA, sorted_keys, sorted_x=None, sorted_y=None, sorted_z=None,
               sorted_id=None, sorted_is_ghost=None, sorted_orig_idx=None, stream=None) -> TreeSoA:
    """build_tree (src/hlbvh.hpp:773-982) from caller-sorted keys (reference layout)."""
    args = [None if a is None else _as_coord(a, ctx.coord) for a in (sorted_x, sorted_y, sorted_z)]
    sid = None if sorted_id is None else np.ascontiguousarray(sorted_id, np.uint32)
    sg = None if sorted_is_ghost is None else np.ascontiguousarray(sorted_is_ghost, np.int8)
    so = None if sorted_orig_idx is None else np.ascontiguousarray(sorted_orig_idx, np.int32)
    _call(lib().ft_build_tree(ctx.handle, tree.c, _ptr(sorted_keys), *[_ptr(a) for a in args], _ptr(sid), _ptr(sg),
                              _ptr(so), _stream_handle(stream)))
    return tree


METHODS = {"default": 0, "fast": 1, "plain": 2, "persistent": 3}  # ft_query_options.method (FT_METHOD_*)


def _method(method) -> int:
    """"fast" (the default: the fast walk with exact replay), "plain" (the reference traversal
    alone), "persistent" (batched build + query in one persistent launch; elsewhere "fast") or
    the C value (FT_METHOD_DEFAULT 0, FT_METHOD_FAST 1, FT_METHOD_PLAIN 2, FT_METHOD_PERSISTENT 3)."""
    if isinstance(method, str):
        if method not in METHODS:
            raise ValueError(f"method must be one of {sorted(METHODS)}")
        return METHODS[method]
    m = int(method)
    if m not in (0, 1, 2, 3):
        raise ValueError("method must be 0 (default), 1 (fast), 2 (plain) or 3 (persistent)")
    return m


def _qopts(max_k: int, method="fast", half_window: int = 0, variant: int = 0):
    o = capi.FtQueryOptions(int(max_k), _method(method))
    o.reserved[0] = int(half_window)  # fast walk: SFC seeding half-window (0 = k)
    o.reserved[1] = int(variant)      # fast walk: 0 default, 1 per-lane, 2 compact, 3 warp-shared, 4 4-wide, 5 group
    return o


def _alloc_knn_out(ctx: Context, rows: int, k: int):
    dev = f"cuda:{ctx.device}"
    return (torch.empty(rows * k, dtype=torch.uint64, device=dev),
            torch.empty(rows * k, dtype=dist_torch_dtype(ctx.coord), device=dev))


def self_knn_query(ctx: Context, tree: TreeSoA, k: int, results=None, result_dists=None, exclude_self=True,
                   max_k: int = 32, method="fast", stream=None, half_window: int = 0, variant: int = 0):
    """self_knn_query<MAXK> (src/hlbvh.hpp:1929-1954).  Asynchronous; returns (idx, dist) of shape
    (num_leaves, k).  method "fast" (default) and "plain" (the reference traversal) return the
    same rows bit for bit."""
    n = tree.num_leaves
    if results is None:
        results, result_dists = _alloc_knn_out(ctx, n, k)
    _call(lib().ft_self_knn(ctx.handle, tree.c, None, n, int(k), int(bool(exclude_self)), _ptr(results),
                            _ptr(result_dists), ctypes.byref(_qopts(max_k, method, half_window, variant)),
                            _stream_handle(stream)))
    return _rows(results, n, k), _rows(result_dists, n, k)


def self_knn_query_bounded(ctx: Context, tree: TreeSoA, k: int, bound, results=None, result_dists=None,
                           exclude_self=True, leaf_ids=None, max_k: int = 32, stream=None, half_window: int = 0,
                           variant: int = 0):
    """self_knn_query with a per-query pruning bound (device tensor of dist_t, in the units of
    the returned distances).  Output equals self_knn_query's for any bound; see
    ft_self_knn_bounded."""
    num = tree.num_leaves if leaf_ids is None else len(leaf_ids)
    if results is None:
        results, result_dists = _alloc_knn_out(ctx, num, k)
    _call(lib().ft_self_knn_bounded(ctx.handle, tree.c, _ptr(leaf_ids), num, int(k), int(bool(exclude_self)),
                                    _ptr(bound), _ptr(results), _ptr(result_dists),
                                    ctypes.byref(_qopts(max_k, 1, half_window, variant)), _stream_handle(stream)))
    return _rows(results, num, k), _rows(result_dists, num, k)


def self_knn_query_subset(ctx: Context, tree: TreeSoA, leaf_ids, k: int, results=None, result_dists=None,
                          exclude_self=True, max_k: int = 256, method="fast", stream=None, variant: int = 0):
    """self_knn_query_subset<MAXK> (src/hlbvh.hpp:1956-1983); leaf_ids is a device int32 tensor."""
    num = len(leaf_ids)
    if results is None:
        results, result_dists = _alloc_knn_out(ctx, num, k)
    _call(lib().ft_self_knn(ctx.handle, tree.c, _ptr(leaf_ids), num, int(k), int(bool(exclude_self)),
                            _ptr(results), _ptr(result_dists), ctypes.byref(_qopts(max_k, method, variant=variant)),
                            _stream_handle(stream)))
    return _rows(results, num, k), _rows(result_dists, num, k)


def knn_query(ctx: Context, tree: TreeSoA, qx, qy, qz, k: int, results=None, result_dists=None, max_k: int = 256,
              method="fast", stream=None, variant: int = 0):
    """knn_query<MAXK> (src/hlbvh.hpp:1405-1472).  Blocking."""
    x, y, z = (_as_coord(a, ctx.coord) for a in (qx, qy, qz))
    nq = len(x)
    if results is None:
        results, result_dists = _alloc_knn_out(ctx, nq, k)
    _call(lib().ft_knn(ctx.handle, tree.c, _ptr(x), _ptr(y), _ptr(z), nq, int(k), _ptr(results), _ptr(result_dists),
                       ctypes.byref(_qopts(max_k, method, variant=variant)), _stream_handle(stream)))
    return _rows(results, nq, k), _rows(result_dists, nq, k)


def tune_self_knn(ctx: Context, tree: TreeSoA, k: int, exclude_self=True, stream=None) -> dict:
    """Autotunes the fast walk for this tree's shape at k (ft_tune_self_knn); later default
    calls take the choice.  Returns the choice and the sample's times."""
    r = capi.FtTuneResult()
    _call(lib().ft_tune_self_knn(ctx.handle, tree.c, int(k), int(bool(exclude_self)), ctypes.byref(r),
                                 _stream_handle(stream)))
    return r.as_dict()


def tune_build(ctx: Context, p, tree: TreeSoA, stream=None) -> dict:
    """Autotunes the build's sort tile on these points (ft_tune_build); the tree is left built."""
    n = len(p.pos_x)
    args = [_as_coord(a, ctx.coord) for a in (p.pos_x, p.pos_y, p.pos_z)]
    r = capi.FtTuneResult()
    _call(lib().ft_tune_build(ctx.handle, *[_ptr(a) for a in args], n, tree.c, ctypes.byref(r),
                              _stream_handle(stream)))
    return r.as_dict()


def tune_reset(ctx: Context):
    _call(lib().ft_tune_reset(ctx.handle))


def range_query(ctx: Context, tree: TreeSoA, qx, qy, qz, r_min, r_max, max_results_per_query: int, results=None,
                result_counts=None, stream=None):
    """range_query (src/hlbvh.hpp:2006-2136).  Blocking; returns (results, counts)."""
    x, y, z, r0, r1 = (_as_coord(a, ctx.coord) for a in (qx, qy, qz, r_min, r_max))
    nq = len(x)
    dev = f"cuda:{ctx.device}"
    if results is None:
        results = torch.full((nq * max_results_per_query,), -1, dtype=torch.int32, device=dev)
    if result_counts is None:
        result_counts = torch.zeros(nq, dtype=torch.int32, device=dev)
    _call(lib().ft_range(ctx.handle, tree.c, _ptr(x), _ptr(y), _ptr(z), _ptr(r0), _ptr(r1), nq, _ptr(results),
                         _ptr(result_counts), int(max_results_per_query), _stream_handle(stream)))
    return _rows(results, nq, max_results_per_query), result_counts


class _BatchSetTree(TreeSoA):
    """One set of a BatchedSets as a TreeSoA (arrays inside the batch; valid until its next build)."""

    def __init__(self, ctx: Context, batch: "BatchedSets", c: capi.FtTree):
        self.ctx = ctx
        self._batch = batch  # keeps the batch's storage alive
        self._c = c
        self._p = ctypes.pointer(c)

    def free(self):
        self._p = None


class BatchedSets:
    """Many independent point sets of uneven size built and queried together (ft_batch_*; no
    counterpart in the reference, whose callers loop build_bvh + self_knn_query over sets).

    Set s holds points [set_offsets[s], set_offsets[s+1]) of the concatenated coordinates; its
    tree and neighbour rows are those of its own build_bvh / self_knn_query calls.  Every array
    is device memory; build and queries are asynchronous and never synchronise the host."""

    def __init__(self, ctx: Context, max_points: int, max_sets: int):
        self.ctx = ctx
        h = ctypes.c_void_p()
        self._h = None
        _call(lib().ft_batch_create(ctx.handle, int(max_points), int(max_sets), ctypes.byref(h)))
        self._h = h
        self._keep = ()
        self.num_sets = 0
        self.num_points = 0

    def _device(self, a, dtype):
        dev = f"cuda:{self.ctx.device}"
        if isinstance(a, torch.Tensor):
            t = a if a.dtype == dtype else a.to(dtype)
            return t.to(dev).contiguous()
        return torch.as_tensor(np.ascontiguousarray(a), device=dev).to(dtype).contiguous()

    def _inputs(self, set_offsets, pos_x, pos_y, pos_z, id, is_ghost):
        off = self._device(set_offsets, torch.int64)
        xyz = [self._device(a, TORCH_COORD[self.ctx.coord]) for a in (pos_x, pos_y, pos_z)]
        ids = None
        if id is not None:  # 32-bit ids, passed through bit for bit
            ids = (id if isinstance(id, torch.Tensor) and id.element_size() == 4 else
                   torch.as_tensor(np.ascontiguousarray(id, np.uint32).view(np.int32)))
            ids = ids.to(f"cuda:{self.ctx.device}").contiguous()
        gh = None if is_ghost is None else self._device(is_ghost, torch.int8)
        return off, xyz, ids, gh

    def set_build_method(self, method="default"):
        """How build() builds the sets: "persistent" (each set whole in one thread block) or
        "default" (the launch sequence); ft_batch_set_build_method."""
        _call(lib().ft_batch_set_build_method(self.ctx.handle, self._h, _method(method)))

    def build(self, set_offsets, pos_x, pos_y, pos_z, id=None, is_ghost=None, stream=None):
        off, xyz, ids, gh = self._inputs(set_offsets, pos_x, pos_y, pos_z, id, is_ghost)
        S, N = off.numel() - 1, xyz[0].numel()
        _call(lib().ft_batch_build(self.ctx.handle, self._h, _ptr(off), S, N, *[_ptr(a) for a in xyz], _ptr(ids),
                                   _ptr(gh), _stream_handle(stream)))
        self._keep = (off, xyz, ids, gh)
        self.num_sets, self.num_points = S, N
        return self

    def self_knn(self, k: int, exclude_self=True, max_k: int = 32, method="fast", results=None,
                 result_dists=None, stream=None, half_window: int = 0, variant: int = 0):
        """self_knn_query<MAXK> of every set; rows in set order, indices local to each set."""
        N = self.num_points
        if results is None:
            results, result_dists = _alloc_knn_out(self.ctx, N, k)
        _call(lib().ft_batch_self_knn(self.ctx.handle, self._h, int(k), int(bool(exclude_self)), _ptr(results),
                                      _ptr(result_dists), ctypes.byref(_qopts(max_k, method, half_window, variant)),
                                      _stream_handle(stream)))
        return _rows(results, N, k), _rows(result_dists, N, k)

    def build_knn(self, set_offsets, pos_x, pos_y, pos_z, k: int, results, result_dists, exclude_self=True,
                  max_k: int = 32, method="default", id=None, is_ghost=None, stream=None):
        """build + self_knn as one CUDA graph (captured on the first call with these arrays, replayed
        afterwards): "default" / "persistent", one persistent launch (k <= 64); "fast" / "plain",
        the launch sequence.  The arrays must stay alive and in place between calls: pass device
        tensors of the right dtype, which are used as they are."""
        off, xyz, ids, gh = self._inputs(set_offsets, pos_x, pos_y, pos_z, id, is_ghost)
        S, N = off.numel() - 1, xyz[0].numel()
        _call(lib().ft_batch_build_knn(self.ctx.handle, self._h, _ptr(off), S, N, *[_ptr(a) for a in xyz],
                                       _ptr(ids), _ptr(gh), int(k), int(bool(exclude_self)), _ptr(results),
                                       _ptr(result_dists), ctypes.byref(_qopts(max_k, method)),
                                       _stream_handle(stream)))
        self._keep = (off, xyz, ids, gh, results, result_dists)
        self.num_sets, self.num_points = S, N
        return _rows(results, N, k), _rows(result_dists, N, k)

    def tune(self, k: int, exclude_self=True, stream=None) -> dict:
        """Autotunes the batched walk for the last build's shape at k (ft_tune_batch_self_knn)."""
        r = capi.FtTuneResult()
        _call(lib().ft_tune_batch_self_knn(self.ctx.handle, self._h, int(k), int(bool(exclude_self)),
                                           ctypes.byref(r), _stream_handle(stream)))
        return r.as_dict()

    def bound_features(self, k: int, stream=None) -> torch.Tensor:
        """(num_points, 12) float32 learned-bound features of every leaf, each on its own set."""
        out = torch.empty((max(self.num_points, 1), 12), dtype=torch.float32, device=f"cuda:{self.ctx.device}")
        _call(lib().ft_batch_bound_features(self.ctx.handle, self._h, int(k), _ptr(out), _stream_handle(stream)))
        return out[: self.num_points]

    def self_knn_learned(self, model, k: int, inflation: float = 1.3, exclude_self=True, max_k: int = 32,
                         results=None, result_dists=None, stream=None):
        """self_knn of every set with the learned radius bound (ft_batch_self_knn_learned): the
        same rows as self_knn; `model` is a learned.BoundModel of this context."""
        N = self.num_points
        if results is None:
            results, result_dists = _alloc_knn_out(self.ctx, N, k)
        _call(lib().ft_batch_self_knn_learned(self.ctx.handle, self._h, model._h, int(k), int(bool(exclude_self)),
                                              ctypes.c_float(inflation), _ptr(results), _ptr(result_dists),
                                              ctypes.byref(_qopts(max_k, "fast")), _stream_handle(stream)))
        return _rows(results, N, k), _rows(result_dists, N, k)

    def build_knn_learned(self, model, set_offsets, pos_x, pos_y, pos_z, k: int, results, result_dists,
                          inflation: float = 1.3, exclude_self=True, max_k: int = 32, id=None, is_ghost=None,
                          stream=None):
        """build + self_knn_learned as one CUDA graph (ft_batch_build_knn_learned); the arrays
        must stay alive and in place between calls, as for build_knn."""
        off, xyz, ids, gh = self._inputs(set_offsets, pos_x, pos_y, pos_z, id, is_ghost)
        S, N = off.numel() - 1, xyz[0].numel()
        _call(lib().ft_batch_build_knn_learned(self.ctx.handle, self._h, model._h, ctypes.c_float(inflation),
                                               _ptr(off), S, N, *[_ptr(a) for a in xyz], _ptr(ids), _ptr(gh), int(k),
                                               int(bool(exclude_self)), _ptr(results), _ptr(result_dists),
                                               ctypes.byref(_qopts(max_k, "fast")), _stream_handle(stream)))
        self._keep = (off, xyz, ids, gh, results, result_dists, model)
        self.num_sets, self.num_points = S, N
        return _rows(results, N, k), _rows(result_dists, N, k)

    def tree(self, s: int, stream=None) -> TreeSoA:
        c = capi.FtTree()
        _call(lib().ft_batch_tree(self.ctx.handle, self._h, int(s), ctypes.byref(c), _stream_handle(stream)))
        return _BatchSetTree(self.ctx, self, c)

    def set_info(self, stream=None):
        """(boxes (S, 6) in the coordinate type, tree heights (S,) uint8) of the last build."""
        S = self.num_sets
        box = np.zeros((S, 6), NP_COORD[self.ctx.coord])
        h = np.zeros(S, np.uint8)
        _call(lib().ft_batch_set_info(self.ctx.handle, self._h, box.ctypes.data, h.ctypes.data,
                                      _stream_handle(stream)))
        return box, h

    def query_stats(self):
        st = capi.FtQueryStats()
        _call(lib().ft_batch_query_stats(self.ctx.handle, self._h, ctypes.byref(st)))
        return {"queries": st.queries, "replayed": st.replayed, "visits": st.reserved[0],
                "bound_misses": st.reserved[1], "rerun_visits": st.reserved[2]}

    def check(self, stream=None):
        """Reports errors the kernels recorded (bad set offsets, bounded waits); synchronises."""
        _call(lib().ft_check_device_status(self.ctx.handle, _stream_handle(stream)))

    def free(self):
        if getattr(self, "_h", None):
            lib().ft_batch_destroy(self.ctx.handle, self._h)
            self._h = None

    def __del__(self):
        try:
            self.free()
        except Exception:
            pass
