"""ctypes declarations of the C ABI in include/fasttree_b200.h.

Loading fails loudly when libfasttree_b200.so is missing: there is no CPU fallback.
"""
from __future__ import annotations

import ctypes
import os

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libfasttree_b200.so")

FT_OK, FT_ERR_INVALID_ARGUMENT, FT_ERR_RUNTIME, FT_ERR_CUDA, FT_ERR_OUT_OF_MEMORY, FT_ERR_TIMEOUT = range(6)
FT_METHOD_DEFAULT, FT_METHOD_FAST, FT_METHOD_PLAIN = 0, 1, 2
F32, F64, U32, U64 = 0, 1, 2, 3
MORTON, PEANO_HILBERT = 0, 1

# Every entry point declared in include/fasttree_b200.h.
EXPORTED = (
    "ft_context_create", "ft_context_destroy", "ft_last_error", "ft_version", "ft_get_query_stats",
    "ft_check_device_status",
    "ft_tree_create", "ft_tree_ensure", "ft_tree_destroy", "ft_compute_bbox", "ft_sfc_encode",
    "ft_build_bvh", "ft_build_tree", "ft_refit_bvh", "ft_tree_export", "ft_tree_import", "ft_self_knn", "ft_knn", "ft_range", "ft_tree_height",
    "ft_self_knn_noalloc", "ft_self_knn_bounded",
    "ft_batch_create", "ft_batch_destroy", "ft_batch_build", "ft_batch_self_knn", "ft_batch_build_knn",
    "ft_batch_tree", "ft_batch_set_info", "ft_batch_query_stats", "ft_batch_self_knn_learned",
    "ft_batch_build_knn_learned", "ft_batch_bound_features", "ft_get_replayed_queries",
    "ft_tune_self_knn", "ft_tune_batch_self_knn", "ft_tune_build", "ft_tune_reset", "ft_set_build_profiling", "ft_set_range_walk", "ft_batch_set_build_method",
    "ft_get_build_profile",
    "ft_bound_model_create", "ft_bound_model_destroy", "ft_bound_model_get_params", "ft_bound_model_set_params",
    "ft_bound_model_set_norm", "ft_bound_features", "ft_bound_targets", "ft_bound_model_gradient",
    "ft_bound_model_fit", "ft_bound_model_predict", "ft_self_knn_learned", "ft_bound_features_points",
    "ft_knn_learned",
)


class FtOptions(ctypes.Structure):
    _fields_ = [("coord_type", ctypes.c_int32), ("sfc_type", ctypes.c_int32), ("periodic", ctypes.c_int32),
                ("return_orig_indices", ctypes.c_int32), ("host_readable_tree", ctypes.c_int32),
                ("reserved", ctypes.c_int32 * 3)]


class FtTree(ctypes.Structure):
    _fields_ = [(n, ctypes.c_void_p) for n in ("min_x", "max_x", "min_y", "max_y", "min_z", "max_z",
                                                "left_child", "right_child", "parent", "id", "is_ghost",
                                                "orig_idx")] + [
        ("num_leaves", ctypes.c_size_t), ("num_internal", ctypes.c_size_t), ("capacity", ctypes.c_size_t),
        ("impl", ctypes.c_void_p)]


class FtQueryOptions(ctypes.Structure):
    _fields_ = [("max_k", ctypes.c_int32), ("method", ctypes.c_int32), ("reserved", ctypes.c_int32 * 6)]


class FtQueryStats(ctypes.Structure):
    _fields_ = [("queries", ctypes.c_int64), ("replayed", ctypes.c_int64), ("reserved", ctypes.c_int64 * 6)]


class FtTuneResult(ctypes.Structure):
    _fields_ = [("walk_variant", ctypes.c_int32), ("half_window", ctypes.c_int32), ("block_threads", ctypes.c_int32),
                ("sort_items", ctypes.c_int32), ("candidates", ctypes.c_int32), ("best_ms", ctypes.c_float),
                ("default_ms", ctypes.c_float), ("reserved", ctypes.c_int32 * 9)]

    def as_dict(self):
        return {f: getattr(self, f) for f, _ in self._fields_ if f != "reserved"}


class FtBuildProfile(ctypes.Structure):
    _fields_ = [(f, ctypes.c_float) for f in ("bbox_ms", "encode_ms", "sort_ms", "gather_ms", "topology_ms",
                                              "refit_ms", "records_ms", "total_ms")] + [
        ("reserved", ctypes.c_int32 * 8)]

    def as_dict(self):
        return {f: getattr(self, f) for f, _ in self._fields_ if f != "reserved"}


class FastTreeError(RuntimeError):
    def __init__(self, status: int, msg: str):
        super().__init__(f"[status {status}] {msg}")
        self.status = status


_lib = None

_vp, _sz, _i, _st = ctypes.c_void_p, ctypes.c_size_t, ctypes.c_int, ctypes.c_void_p
_SIGS = {
    "ft_context_create": [ctypes.POINTER(FtOptions), _i, ctypes.POINTER(_vp)],
    "ft_context_destroy": [_vp],
    "ft_get_query_stats": [_vp, ctypes.POINTER(FtQueryStats)],
    "ft_get_replayed_queries": [_vp, _vp, _sz, ctypes.POINTER(ctypes.c_size_t)],
    "ft_check_device_status": [_vp, _st],
    "ft_tree_create": [_vp, _sz, ctypes.POINTER(ctypes.POINTER(FtTree))],
    "ft_tree_ensure": [_vp, ctypes.POINTER(FtTree), _sz],
    "ft_tree_destroy": [_vp, ctypes.POINTER(FtTree)],
    "ft_tree_height": [_vp, ctypes.POINTER(FtTree), ctypes.POINTER(_i)],
    "ft_compute_bbox": [_vp, _vp, _vp, _vp, _sz, _vp, _st],
    "ft_sfc_encode": [_vp, _vp, _vp, _vp, _sz, _vp, _vp, _st],
    "ft_build_bvh": [_vp, _vp, _vp, _vp, _sz, _vp, _vp, _vp, _vp, ctypes.POINTER(FtTree), _st],
    "ft_refit_bvh": [_vp, _vp, _vp, _vp, _sz, _i, ctypes.POINTER(FtTree), _st],
    "ft_tree_export": [_vp, ctypes.POINTER(FtTree), _vp, ctypes.POINTER(ctypes.c_size_t), _st],
    "ft_tree_import": [_vp, _vp, _sz, ctypes.POINTER(FtTree), _st],
    "ft_build_tree": [_vp, ctypes.POINTER(FtTree), _vp, _vp, _vp, _vp, _vp, _vp, _vp, _st],
    "ft_self_knn": [_vp, ctypes.POINTER(FtTree), _vp, _sz, _i, _i, _vp, _vp, ctypes.POINTER(FtQueryOptions), _st],
    "ft_self_knn_noalloc": [_vp, ctypes.POINTER(FtTree), _vp, _sz, _i, _i, _vp, _vp, _st],
    "ft_self_knn_bounded": [_vp, ctypes.POINTER(FtTree), _vp, _sz, _i, _i, _vp, _vp, _vp,
                            ctypes.POINTER(FtQueryOptions), _st],
    "ft_knn": [_vp, ctypes.POINTER(FtTree), _vp, _vp, _vp, _sz, _i, _vp, _vp, ctypes.POINTER(FtQueryOptions), _st],
    "ft_range": [_vp, ctypes.POINTER(FtTree), _vp, _vp, _vp, _vp, _vp, _sz, _vp, _vp, _i, _st],
    "ft_batch_create": [_vp, _sz, _sz, ctypes.POINTER(_vp)],
    "ft_batch_destroy": [_vp, _vp],
    "ft_batch_build": [_vp, _vp, _vp, _sz, _sz, _vp, _vp, _vp, _vp, _vp, _st],
    "ft_batch_self_knn": [_vp, _vp, _i, _i, _vp, _vp, ctypes.POINTER(FtQueryOptions), _st],
    "ft_batch_build_knn": [_vp, _vp, _vp, _sz, _sz, _vp, _vp, _vp, _vp, _vp, _i, _i, _vp, _vp,
                           ctypes.POINTER(FtQueryOptions), _st],
    "ft_batch_tree": [_vp, _vp, _sz, ctypes.POINTER(FtTree), _st],
    "ft_batch_bound_features": [_vp, _vp, _i, _vp, _st],
    "ft_tune_self_knn": [_vp, ctypes.POINTER(FtTree), _i, _i, ctypes.POINTER(FtTuneResult), _st],
    "ft_tune_batch_self_knn": [_vp, _vp, _i, _i, ctypes.POINTER(FtTuneResult), _st],
    "ft_tune_build": [_vp, _vp, _vp, _vp, _sz, ctypes.POINTER(FtTree), ctypes.POINTER(FtTuneResult), _st],
    "ft_tune_reset": [_vp],
    "ft_set_build_profiling": [_vp, _i],
    "ft_set_range_walk": [_vp, _i],
    "ft_batch_set_build_method": [_vp, _vp, _i],
    "ft_get_build_profile": [_vp, ctypes.POINTER(FtBuildProfile)],
    "ft_batch_self_knn_learned": [_vp, _vp, _vp, _i, _i, ctypes.c_float, _vp, _vp, ctypes.POINTER(FtQueryOptions),
                                  _st],
    "ft_batch_build_knn_learned": [_vp, _vp, _vp, ctypes.c_float, _vp, _sz, _sz, _vp, _vp, _vp, _vp, _vp, _i, _i,
                                   _vp, _vp, ctypes.POINTER(FtQueryOptions), _st],
    "ft_batch_set_info": [_vp, _vp, _vp, _vp, _st],
    "ft_batch_query_stats": [_vp, _vp, ctypes.POINTER(FtQueryStats)],
    "ft_bound_model_create": [_vp, ctypes.c_uint64, ctypes.POINTER(_vp)],
    "ft_bound_model_destroy": [_vp, _vp],
    "ft_bound_model_get_params": [_vp, _vp, _vp],
    "ft_bound_model_set_params": [_vp, _vp, _vp],
    "ft_bound_model_set_norm": [_vp, _vp, _vp, _vp, ctypes.c_float, ctypes.c_float],
    "ft_bound_features": [_vp, ctypes.POINTER(FtTree), _vp, _sz, _i, _vp, _st],
    "ft_bound_targets": [_vp, _vp, _vp, _sz, _i, _vp, _st],
    "ft_bound_model_gradient": [_vp, _vp, _vp, _vp, _sz, _vp, _vp, _st],
    "ft_bound_model_fit": [_vp, _vp, _vp, _vp, _sz, _i, _i, ctypes.c_float, ctypes.c_uint64, _vp, _st],
    "ft_bound_model_predict": [_vp, _vp, _vp, _sz, ctypes.c_float, _vp, _vp, _st],
    "ft_self_knn_learned": [_vp, ctypes.POINTER(FtTree), _vp, _vp, _sz, _i, _i, ctypes.c_float, _vp, _vp,
                            ctypes.POINTER(FtQueryOptions), _st],
    "ft_bound_features_points": [_vp, ctypes.POINTER(FtTree), _vp, _vp, _vp, _sz, _i, _vp, _st],
    "ft_knn_learned": [_vp, ctypes.POINTER(FtTree), _vp, _vp, _vp, _vp, _sz, _i, ctypes.c_float, _vp, _vp,
                       ctypes.POINTER(FtQueryOptions), _st],
}


def lib():
    """The loaded C library (raises if it has not been built)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(f"{LIB_PATH} is missing: build it with `python -m fasttree_b200._build_ext` "
                              "(or __graft_entry__.build()); there is no CPU fallback")
        L = ctypes.CDLL(LIB_PATH)
        for name, args in _SIGS.items():
            f = getattr(L, name)
            f.argtypes = args
            f.restype = ctypes.c_int
        L.ft_last_error.restype = ctypes.c_char_p
        L.ft_last_error.argtypes = []
        L.ft_version.restype = ctypes.c_int
        _lib = L
    return _lib


def check(status: int):
    if status != FT_OK:
        raise FastTreeError(status, lib().ft_last_error().decode(errors="replace"))
