"""fasttree_b200 -- B200-native (sm_100a) HLBVH build and neighbour queries with FastTree's API.

The compute path is libfasttree_b200.so (hand-written CUDA kernels behind the C ABI in
include/fasttree_b200.h); this package binds it with ctypes and uses torch only for device
buffers and streams.  Importing the package does not need a GPU; calling into it does, and
there is no CPU fallback.
"""
from .capi import F32, F64, U32, U64, MORTON, PEANO_HILBERT, FastTreeError  # noqa: F401
from .hlbvh import (BatchedSets, BoundingBox, Context, TreePool, TreeSoA, build_bvh, build_tree,  # noqa: F401
                    compute_bbox, dist_torch_dtype, import_tree, knn_query, load_tree, particles, range_query,
                    refit_bvh, self_knn_query, self_knn_query_bounded, self_knn_query_subset, sfc_encode,
                    tune_build, tune_reset, tune_self_knn)

__version__ = "0.1.0"
