// fasttree/hlbvh.hpp -- drop-in C++ API for FastTree's HLBVH build and neighbour queries on
// a B200, implemented over the C ABI of libfasttree_b200.so (include/fasttree_b200.h).
//
// Same names, template parameters and argument meaning as the reference's src/hlbvh.hpp:
// particles<T> (26-34), BoundingBox<T> (78-110), TreeSoA (609-673), TreePool (682-715),
// BvhScratch (720-745), compute_bbox (462-578), sfc_encode (357-450), build_tree (773-982),
// build_bvh (2165-2302), knn_query<MAXK> (1405-1472), self_knn_query<MAXK> (1929-1954),
// self_knn_query_subset<MAXK> (1956-1983), range_query (2006-2136).  The sycl::queue
// argument becomes a fasttree::queue (device + CUDA stream).  The reference's compile-time
// configuration macros select the same types:
//   SFC_TYPE_MORTON | SFC_TYPE_PEANO_HILBERT, FASTTREE_INTEGER_COORDS with
//   POSITIONS_IN_32BIT | POSITIONS_IN_64BIT, COORDS_TYPE_DOUBLE, PERIODIC_BC,
//   RETURN_ORIG_INDICES.
// Errors: std::invalid_argument and std::runtime_error where the reference throws them;
// other library failures throw std::runtime_error with the library's message.
// Synchronisation: build_bvh, build_tree, compute_bbox, sfc_encode, knn_query and
// range_query block; self_knn_query* are asynchronous on the queue's stream, as in the
// reference.  TreeSoA arrays are host-readable (managed memory), as USM shared memory is.
#pragma once

#include <cstddef>
#include <cstdint>
#include <limits>
#include <stdexcept>
#include <string>
#include <type_traits>
#include <vector>

#include <cuda_runtime.h>

#include "../fasttree_b200.h"

#if !defined(SFC_TYPE_PEANO_HILBERT) && !defined(SFC_TYPE_MORTON)
#error "Undefined SFC_TYPE - either SFC_TYPE_PEANO_HILBERT or SFC_TYPE_MORTON must be defined"
#endif

namespace fasttree {

// ---- configuration -------------------------------------------------------------------
#if defined(FASTTREE_INTEGER_COORDS)
#if defined(POSITIONS_IN_64BIT)
using coord_t                        = uint64_t;
constexpr int32_t kCoordType         = FT_COORD_U64;
constexpr int     BITS_PER_DIMENSION = 42;
#else
using coord_t                        = uint32_t;
constexpr int32_t kCoordType         = FT_COORD_U32;
constexpr int     BITS_PER_DIMENSION = 21;
#endif
using dist_t = uint64_t;
#elif defined(COORDS_TYPE_DOUBLE)
using coord_t                        = double;
constexpr int32_t kCoordType         = FT_COORD_F64;
constexpr int     BITS_PER_DIMENSION = 21;
using dist_t                         = double;
#else
using coord_t                        = float;
constexpr int32_t kCoordType         = FT_COORD_F32;
constexpr int     BITS_PER_DIMENSION = 21;
using dist_t                         = double;
#endif
using heap_dist_t = dist_t;

#if defined(SFC_TYPE_MORTON)
using sfc_key                 = uint64_t;
constexpr int32_t kSfcType    = FT_SFC_MORTON;
#else
constexpr int32_t kSfcType    = FT_SFC_PEANO_HILBERT;
#if defined(POSITIONS_IN_64BIT)
struct sfc_key {
    uint64_t hs = 0, is = 0, ls = 0;
    bool     operator<(const sfc_key &o) const { return hs != o.hs ? hs < o.hs : is != o.is ? is < o.is : ls < o.ls; }
    bool     operator==(const sfc_key &o) const { return hs == o.hs && is == o.is && ls == o.ls; }
    bool     operator!=(const sfc_key &o) const { return !(*this == o); }
};
#else
struct sfc_key {
    uint32_t hs = 0, is = 0, ls = 0;
    bool     operator<(const sfc_key &o) const { return hs != o.hs ? hs < o.hs : is != o.is ? is < o.is : ls < o.ls; }
    bool     operator==(const sfc_key &o) const { return hs == o.hs && is == o.is && ls == o.ls; }
    bool     operator!=(const sfc_key &o) const { return !(*this == o); }
};
#endif
#endif
static constexpr int KEY_TOTAL_BITS = 3 * BITS_PER_DIMENSION;

#if defined(PERIODIC_BC)
constexpr int32_t kPeriodic = 1;
#else
constexpr int32_t kPeriodic = 0;
#endif
#if defined(RETURN_ORIG_INDICES)
constexpr int32_t kReturnOrig = 1;
#else
constexpr int32_t kReturnOrig = 0;
#endif

// ---- errors ------------------------------------------------------------------------------
inline void check(ft_status s) {
    if (s == FT_OK) return;
    std::string msg = ft_last_error();
    if (s == FT_ERR_INVALID_ARGUMENT) throw std::invalid_argument(msg);
    throw std::runtime_error(msg);
}

// ---- queue: device + stream + library context (replaces sycl::queue) -------------------
class queue {
  public:
    explicit queue(int device = 0, ft_stream_t stream = nullptr) : stream_(stream) {
        ft_options o{};
        o.coord_type          = kCoordType;
        o.sfc_type            = kSfcType;
        o.periodic            = kPeriodic;
        o.return_orig_indices = kReturnOrig;
        o.host_readable_tree  = 1;
        check(ft_context_create(&o, device, &ctx_));
    }
    ~queue() {
        if (ctx_) ft_context_destroy(ctx_);
    }
    queue(const queue &)            = delete;
    queue &operator=(const queue &) = delete;
    ft_context *context() const { return ctx_; }
    ft_stream_t stream() const { return stream_; }
    void        wait() {
        check(ft_check_device_status(ctx_, stream_));
        cudaStreamSynchronize(reinterpret_cast<cudaStream_t>(stream_));
    }

  private:
    ft_context *ctx_ = nullptr;
    ft_stream_t stream_;
};

// ---- USM-style allocations (sycl::malloc_shared / malloc_device / free) ---------------------
template <typename T> inline T *malloc_shared(size_t n, queue &) {
    void *p = nullptr;
    if (cudaMallocManaged(&p, (n ? n : 1) * sizeof(T)) != cudaSuccess) throw std::runtime_error("malloc_shared failed");
    return static_cast<T *>(p);
}
template <typename T> inline T *malloc_device(size_t n, queue &) {
    void *p = nullptr;
    if (cudaMalloc(&p, (n ? n : 1) * sizeof(T)) != cudaSuccess) throw std::runtime_error("malloc_device failed");
    return static_cast<T *>(p);
}
inline void free(void *p, queue &) {
    if (p) cudaFree(p);
}

// ---- data types ----------------------------------------------------------------------------
template <typename T> struct particles {
    std::vector<T>        pos_x, pos_y, pos_z;
    std::vector<uint32_t> id;
    std::vector<int8_t>   is_ghost;
};

template <typename T> inline T type_identity_min() {
    if constexpr (std::is_floating_point_v<T>) return std::numeric_limits<T>::max();
    else return std::numeric_limits<T>::max();
}
template <typename T> inline T type_identity_max() {
    if constexpr (std::is_floating_point_v<T>) return -std::numeric_limits<T>::max();
    else return T(0);
}

template <typename FloatT> struct BoundingBox {
    FloatT min_x, max_x, min_y, max_y, min_z, max_z;
    BoundingBox(FloatT a, FloatT b, FloatT c, FloatT d, FloatT e, FloatT f)
        : min_x(a), max_x(b), min_y(c), max_y(d), min_z(e), max_z(f) {}
    BoundingBox()
        : min_x(type_identity_min<FloatT>()), max_x(type_identity_max<FloatT>()), min_y(type_identity_min<FloatT>()),
          max_y(type_identity_max<FloatT>()), min_z(type_identity_min<FloatT>()), max_z(type_identity_max<FloatT>()) {}
};

// Flat tree; arrays point into the library's managed allocation (host-readable).
struct TreeSoA {
    coord_t  *min_x = nullptr, *max_x = nullptr, *min_y = nullptr, *max_y = nullptr, *min_z = nullptr,
            *max_z   = nullptr;
    int      *left_child = nullptr, *right_child = nullptr, *parent = nullptr;
    uint32_t *id        = nullptr;
    int8_t   *is_ghost  = nullptr;
    int      *orig_idx  = nullptr;
    size_t    num_leaves = 0, num_internal = 0;
    ft_tree  *handle     = nullptr;
    ft_context *ctx      = nullptr;

    TreeSoA(queue &q, size_t n) : ctx(q.context()) {
        check(ft_tree_create(ctx, n, &handle));
        sync();
    }
    TreeSoA(const TreeSoA &)            = delete;
    TreeSoA &operator=(const TreeSoA &) = delete;
    ~TreeSoA() { release(); }
    void free(queue &) { release(); }
    void release() {
        if (handle) ft_tree_destroy(ctx, handle);
        handle = nullptr;
        min_x = max_x = min_y = max_y = min_z = max_z = nullptr;
        left_child = right_child = parent = nullptr;
        id                                = nullptr;
        is_ghost                          = nullptr;
        orig_idx                          = nullptr;
        num_leaves = num_internal = 0;
    }
    // refresh the member pointers/sizes from the library's tree
    void sync() {
        if (!handle) return;
        min_x        = static_cast<coord_t *>(handle->min_x);
        max_x        = static_cast<coord_t *>(handle->max_x);
        min_y        = static_cast<coord_t *>(handle->min_y);
        max_y        = static_cast<coord_t *>(handle->max_y);
        min_z        = static_cast<coord_t *>(handle->min_z);
        max_z        = static_cast<coord_t *>(handle->max_z);
        left_child   = handle->left_child;
        right_child  = handle->right_child;
        parent       = handle->parent;
        id           = handle->id;
        is_ghost     = handle->is_ghost;
        orig_idx     = handle->orig_idx;
        num_leaves   = handle->num_leaves;
        num_internal = handle->num_internal;
    }
};

// TreePool (src/hlbvh.hpp:682-715): reallocates only when n exceeds capacity.
struct TreePool {
    TreeSoA *tree     = nullptr;
    size_t   capacity = 0;
    TreeSoA &ensure(queue &q, size_t n_total) {
        if (!tree) tree = new TreeSoA(q, 0);
        check(ft_tree_ensure(q.context(), tree->handle, n_total));
        tree->sync();
        capacity = tree->handle->capacity;
        return *tree;
    }
    void free_all(queue &) {
        delete tree;
        tree     = nullptr;
        capacity = 0;
    }
};

// BvhScratch (src/hlbvh.hpp:720-745): build scratch lives with each tree here; kept for
// signature compatibility.
struct BvhScratch {
    size_t capacity = 0;
    void   ensure(size_t n, queue &) { capacity = n > capacity ? n : capacity; }
    void   free_all(queue &) { capacity = 0; }
};

// ---- build -------------------------------------------------------------------------------
template <typename FloatT>
inline BoundingBox<FloatT> compute_bbox(queue &q, const FloatT *x, const FloatT *y, const FloatT *z, size_t n) {
    FloatT o[6];
    check(ft_compute_bbox(q.context(), x, y, z, n, o, q.stream()));
    return BoundingBox<FloatT>(o[0], o[1], o[2], o[3], o[4], o[5]);
}
template <typename FloatT> inline BoundingBox<FloatT> compute_bbox(queue &q, const particles<FloatT> &p, size_t n) {
    return compute_bbox(q, p.pos_x.data(), p.pos_y.data(), p.pos_z.data(), n);
}

template <typename FloatT>
inline void sfc_encode(queue &q, const FloatT *x, const FloatT *y, const FloatT *z, size_t n, sfc_key *keys,
                       const BoundingBox<FloatT> &bbox) {
    FloatT b[6] = {bbox.min_x, bbox.max_x, bbox.min_y, bbox.max_y, bbox.min_z, bbox.max_z};
    check(ft_sfc_encode(q.context(), x, y, z, n, keys, b, q.stream()));
}
template <typename FloatT>
inline void sfc_encode(queue &q, const particles<FloatT> &p, sfc_key *keys, const BoundingBox<FloatT> &bbox) {
    sfc_encode(q, p.pos_x.data(), p.pos_y.data(), p.pos_z.data(), p.pos_x.size(), keys, bbox);
}

inline void build_tree(queue &q, TreeSoA &tree, const sfc_key *sorted_keys, const coord_t *sx = nullptr,
                       const coord_t *sy = nullptr, const coord_t *sz = nullptr, const uint32_t *sid = nullptr,
                       const int8_t *sghost = nullptr, const int *sorig = nullptr) {
    check(ft_build_tree(q.context(), tree.handle, sorted_keys, sx, sy, sz, sid, sghost, sorig, q.stream()));
    tree.sync();
}

inline void build_bvh(queue &q, const particles<coord_t> &p, TreeSoA &tree, BvhScratch &,
                      BoundingBox<coord_t> *bbox = nullptr, sfc_key *key = nullptr) {
    size_t  n = p.pos_x.size();
    coord_t b[6];
    if (bbox) {
        b[0] = bbox->min_x;
        b[1] = bbox->max_x;
        b[2] = bbox->min_y;
        b[3] = bbox->max_y;
        b[4] = bbox->min_z;
        b[5] = bbox->max_z;
    }
    check(ft_build_bvh(q.context(), p.pos_x.data(), p.pos_y.data(), p.pos_z.data(), n,
                       p.id.empty() ? nullptr : p.id.data(), p.is_ghost.empty() ? nullptr : p.is_ghost.data(),
                       bbox ? b : nullptr, key, tree.handle, q.stream()));
    tree.sync();
}
inline void build_bvh(queue &q, const particles<coord_t> &p, TreeSoA &tree, BoundingBox<coord_t> *bbox = nullptr,
                      sfc_key *key = nullptr) {
    BvhScratch s;
    build_bvh(q, p, tree, s, bbox, key);
}

// Refit-only update for moved points (no reference counterpart; ft_refit_bvh): the same
// points at new positions, in build_bvh's input order; keys and topology are kept.
inline void refit_bvh(queue &q, const particles<coord_t> &p, TreeSoA &tree) {
    check(ft_refit_bvh(q.context(), p.pos_x.data(), p.pos_y.data(), p.pos_z.data(), p.pos_x.size(), 0,
                       tree.handle, q.stream()));
    tree.sync();
}

// Tree serialisation (ft_tree_export / ft_tree_import): the raw SoA arrays and keys behind
// a fixed header, e.g. to ship a tree between ranks as test/test_mpi.cpp ships its arrays.
inline std::vector<unsigned char> save_tree(queue &q, const TreeSoA &tree) {
    size_t bytes = 0;
    check(ft_tree_export(q.context(), tree.handle, nullptr, &bytes, q.stream()));
    std::vector<unsigned char> out(bytes);
    check(ft_tree_export(q.context(), tree.handle, out.data(), &bytes, q.stream()));
    return out;
}
inline void load_tree(queue &q, const std::vector<unsigned char> &data, TreeSoA &tree) {
    check(ft_tree_import(q.context(), data.data(), data.size(), tree.handle, q.stream()));
    tree.sync();
}

// ---- queries -----------------------------------------------------------------------------
// The kNN queries take the fast walk (SFC-window seeding, exact replay of tied queries):
// its output is bit-identical to the reference traversal's.  Define
// FASTTREE_B200_PLAIN_TRAVERSAL to run the reference traversal itself.
#if defined(FASTTREE_B200_PLAIN_TRAVERSAL)
inline constexpr int kQueryMethod = FT_METHOD_PLAIN;
#else
inline constexpr int kQueryMethod = FT_METHOD_DEFAULT;
#endif

template <int _MAX_K_ = 256>
inline void knn_query(queue &q, const TreeSoA &tree, const coord_t *qx, const coord_t *qy, const coord_t *qz, int k,
                      int num_queries, size_t *results, dist_t *result_dists) {
    ft_query_options o{};
    o.max_k  = _MAX_K_;
    o.method = kQueryMethod;
    check(ft_knn(q.context(), tree.handle, qx, qy, qz, (size_t)num_queries, k, reinterpret_cast<uint64_t *>(results),
                 result_dists, &o, q.stream()));
}

template <int _MAX_K_ = 32>
inline void self_knn_query(queue &q, const TreeSoA &tree, int k, size_t *results, dist_t *result_dists,
                           bool exclude_self = true) {
    ft_query_options o{};
    o.max_k  = _MAX_K_;
    o.method = kQueryMethod;
    check(ft_self_knn(q.context(), tree.handle, nullptr, tree.num_leaves, k, exclude_self ? 1 : 0,
                      reinterpret_cast<uint64_t *>(results), result_dists, &o, q.stream()));
}

template <int _MAX_K_ = 256>
inline void self_knn_query_subset(queue &q, const TreeSoA &tree, const int *leaf_ids, int num_ids, int k,
                                  size_t *results, dist_t *result_dists, bool exclude_self = true) {
    if (num_ids == 0) return;
    ft_query_options o{};
    o.max_k  = _MAX_K_;
    o.method = kQueryMethod;
    check(ft_self_knn(q.context(), tree.handle, leaf_ids, (size_t)num_ids, k, exclude_self ? 1 : 0,
                      reinterpret_cast<uint64_t *>(results), result_dists, &o, q.stream()));
}

inline void range_query(queue &q, const TreeSoA &tree, const coord_t *qx, const coord_t *qy, const coord_t *qz,
                        const coord_t *r_min, const coord_t *r_max, int num_queries, int *results, int *result_counts,
                        int max_results_per_query) {
    check(ft_range(q.context(), tree.handle, qx, qy, qz, r_min, r_max, (size_t)num_queries, results, result_counts,
                   max_results_per_query, q.stream()));
}

} // namespace fasttree
