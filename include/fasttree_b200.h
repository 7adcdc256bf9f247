/* fasttree_b200.h -- C ABI of the B200 (sm_100a) HLBVH build and neighbour-query library.
 *
 * One entry point per operation of FastTree's C++ API (sparxastronomy/fasttree,
 * src/hlbvh.hpp).  The reference is a header-only C++/SYCL library; its callers bind the
 * C++ templates directly.  The functions below are what a non-C++ caller (or the C++
 * wrapper in include/fasttree/hlbvh.hpp) binds instead: plain pointers and sizes, a
 * cudaStream_t in place of the sycl::queue, status codes in place of exceptions.
 *
 * Compile-time choices of the reference (coordinate type, SFC type, PERIODIC_BC,
 * RETURN_ORIG_INDICES; CMakeLists.txt:63-125) are runtime fields of ft_options.
 *
 * Pointers: any argument documented as "host or device" may be a host pointer; it is
 * staged through device memory (the reference's ensure_device_readable /
 * ensure_device_writable rule, src/hlbvh.hpp:125-200).  Arguments documented as "device"
 * must be device-accessible (cudaMalloc, cudaMallocManaged or mapped memory).
 */
#ifndef FASTTREE_B200_H
#define FASTTREE_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct CUstream_st *ft_stream_t; /* == cudaStream_t; NULL = legacy default stream */

typedef enum ft_status {
    FT_OK                   = 0,
    FT_ERR_INVALID_ARGUMENT = 1, /* reference: std::invalid_argument (e.g. k > MAXK)       */
    FT_ERR_RUNTIME          = 2, /* reference: std::runtime_error (n > INT_MAX/2, ...)      */
    FT_ERR_CUDA             = 3, /* a CUDA runtime call failed; see ft_last_error()         */
    FT_ERR_OUT_OF_MEMORY    = 4,
    FT_ERR_TIMEOUT          = 5  /* a bounded device-side wait gave up (status word set)   */
} ft_status;

typedef enum ft_coord_type { /* coord_t (src/hlbvh.hpp:202-209)                                   */
    FT_COORD_F32 = 0,        /* COORDS_TYPE_FLOAT                                                 */
    FT_COORD_F64 = 1,        /* COORDS_TYPE_DOUBLE                                                */
    FT_COORD_U32 = 2,        /* FASTTREE_INTEGER_COORDS + POSITIONS_IN_32BIT (21 bits per axis)   */
    FT_COORD_U64 = 3         /* FASTTREE_INTEGER_COORDS + POSITIONS_IN_64BIT (42 bits per axis)   */
} ft_coord_type;

typedef enum ft_sfc_type {
    FT_SFC_MORTON        = 0, /* SFC_TYPE_MORTON (floating-point coordinates only) */
    FT_SFC_PEANO_HILBERT = 1  /* SFC_TYPE_PEANO_HILBERT                            */
} ft_sfc_type;

typedef struct ft_options {
    int32_t coord_type;          /* ft_coord_type                                          */
    int32_t sfc_type;            /* ft_sfc_type                                            */
    int32_t periodic;            /* PERIODIC_BC: toroidal distance (integer coords only)   */
    int32_t return_orig_indices; /* RETURN_ORIG_INDICES: queries return input indices      */
    int32_t host_readable_tree;  /* 1: tree arrays in managed memory (the reference's USM
                                    shared allocation, src/hlbvh.hpp:632-650); 0: device  */
    int32_t reserved[3];
} ft_options;

typedef struct ft_context ft_context;

/* Flat tree with TreeSoA's members and index layout (src/hlbvh.hpp:609-673): internal
 * nodes [0, n-2] (root 0), leaves [n-1, 2n-2]; leaf boxes have min == max. Coordinate
 * arrays hold ft_options.coord_type values. */
typedef struct ft_tree {
    void     *min_x, *max_x, *min_y, *max_y, *min_z, *max_z; /* 2n-1 each                  */
    int32_t  *left_child, *right_child;                      /* n-1 each                    */
    int32_t  *parent;                                        /* 2n-1, root -1               */
    uint32_t *id;                                            /* 2n-1 (leaf slots used)      */
    int8_t   *is_ghost;                                      /* 2n-1 (leaf slots used)      */
    int32_t  *orig_idx;                                      /* 2n-1 (leaf slots used)      */
    size_t    num_leaves;
    size_t    num_internal;
    size_t    capacity;  /* leaf capacity of the allocation (TreePool::capacity)           */
    void     *impl;      /* library-owned acceleration data; do not touch                  */
} ft_tree;

/* Query method (ft_query_options.method).  Both methods return the same rows bit for bit;
 * the fast walk hands every query whose rows it cannot prove equal to the reference
 * traversal's (ties, a stack that could overflow, the reference's stack guard) to that
 * traversal, so the plain method is both fallback and check. */
#define FT_METHOD_DEFAULT 0 /* the fast walk with exact replay (a zeroed ft_query_options)  */
#define FT_METHOD_FAST    1 /* the same, named                                             */
#define FT_METHOD_PLAIN   2 /* the reference traversal and heap alone                       */
#define FT_METHOD_PERSISTENT 3 /* ft_batch_build_knn: one persistent launch builds every set
                                  and walks its queries (k <= 64; else its build, then the fast
                                  walk) -- also what FT_METHOD_DEFAULT does there, while
                                  FT_METHOD_FAST selects the launch sequence; other calls
                                  treat it as FT_METHOD_FAST                                  */

/* Per-query-call options (the reference's template parameters and dispatch choices). */
typedef struct ft_query_options {
    int32_t max_k;        /* _MAX_K_ template argument; 0 = the reference's default         */
    int32_t method;       /* FT_METHOD_DEFAULT / FT_METHOD_FAST / FT_METHOD_PLAIN           */
    int32_t reserved[6];  /* [0] SFC seeding half-window (0 = k), [1] walk variant (0 = the
                             tuned default), others 0                                      */
} ft_query_options;

/* Statistics of the last query on a context (fallback rate, visits). */
typedef struct ft_query_stats {
    int64_t queries;
    int64_t replayed;      /* queries rerun by the plain traversal (ties, the stack guard)   */
    int64_t reserved[6];   /* [0] node visits of the fast walk (lane-node evaluations, every
                              launch); [1] queries whose pruning bound proved too small, rerun
                              by the fast walk without the bound; [2] the visits of that rerun */
} ft_query_stats;

/* ---------------------------------------------------------------------------------- */
/* Context                                                                             */
/* ---------------------------------------------------------------------------------- */
ft_status   ft_context_create(const ft_options *opts, int device, ft_context **out);
ft_status   ft_context_destroy(ft_context *ctx);
const char *ft_last_error(void); /* thread-local message of the last failing call */
int         ft_version(void);
ft_status   ft_get_query_stats(ft_context *ctx, ft_query_stats *out);
/* Output rows (query numbers) that the last fast-walk query on this context handed to the
 * reference traversal (ties that could change the order, a full stack, the reference's
 * stack guard, a bound that proved too small), in no particular order: *count_out receives
 * how many, and up to `capacity` of them go to rows_out (host; NULL with capacity 0 to ask
 * for the count).  Covers ft_self_knn / ft_self_knn_bounded / ft_self_knn_learned /
 * ft_knn / ft_knn_learned with device outputs; 0 after a plain-method call.  Synchronises
 * the device.  No counterpart in the reference (its callers cannot see which path ran). */
ft_status   ft_get_replayed_queries(ft_context *ctx, int32_t *rows_out, size_t capacity, size_t *count_out);
/* Synchronises stream and reports (then clears) the context's device status word: kernels
 * record bad leaf ids or an exceeded traversal bound there instead of trapping.  Blocking
 * calls check it themselves; call this after asynchronous self-kNN queries. */
ft_status   ft_check_device_status(ft_context *ctx, ft_stream_t stream);

/* ---------------------------------------------------------------------------------- */
/* Trees: TreeSoA(q, n) / TreeSoA::free (src/hlbvh.hpp:632-672) and                    */
/* TreePool::ensure (src/hlbvh.hpp:682-705): reallocation only when n exceeds capacity. */
/* ---------------------------------------------------------------------------------- */
ft_status ft_tree_create(ft_context *ctx, size_t n, ft_tree **out);
ft_status ft_tree_ensure(ft_context *ctx, ft_tree *tree, size_t n);
ft_status ft_tree_destroy(ft_context *ctx, ft_tree *tree);

/* ---------------------------------------------------------------------------------- */
/* Build                                                                               */
/* ---------------------------------------------------------------------------------- */

/* compute_bbox (src/hlbvh.hpp:462-572).  x/y/z: host or device, n coords each.
 * out6 (host): {min_x, max_x, min_y, max_y, min_z, max_z} in the coordinate type.
 * Blocking.  n == 0 returns the identity box. */
ft_status ft_compute_bbox(ft_context *ctx, const void *x, const void *y, const void *z, size_t n,
                          void *out6, ft_stream_t stream);

/* sfc_encode (src/hlbvh.hpp:357-423).  keys: host or device, n keys in the reference's
 * sfc_key layout: uint64 for Morton; {hs,is,ls} uint32 triples (12 B) for Peano-Hilbert
 * with 32-bit positions (F32/F64/U32); {hs,is,ls} uint64 triples (24 B) for U64.
 * bbox6: host, ignored for integer coordinates.  Blocking. */
ft_status ft_sfc_encode(ft_context *ctx, const void *x, const void *y, const void *z, size_t n,
                        void *keys, const void *bbox6, ft_stream_t stream);

/* build_bvh (src/hlbvh.hpp:2165-2302).  x/y/z: host or device; id, is_ghost: host or
 * device or NULL (then iota / 0, as the reference fills them).  bbox6: host or NULL
 * (computed).  keys: NULL or the caller's keys in sfc_key layout (host or device), which
 * are sorted in place as in the reference.  tree: from ft_tree_create/ensure; resized to
 * n.  Blocking (the reference waits internally). */
ft_status ft_build_bvh(ft_context *ctx, const void *x, const void *y, const void *z, size_t n,
                       const uint32_t *id, const int8_t *is_ghost, const void *bbox6, void *keys,
                       ft_tree *tree, ft_stream_t stream);

/* build_tree (src/hlbvh.hpp:773-982) from caller-sorted keys (sfc_key layout) and
 * optional sorted leaf attributes (each host or device or NULL).  tree->num_leaves keys. */
ft_status ft_build_tree(ft_context *ctx, ft_tree *tree, const void *sorted_keys,
                        const void *sorted_x, const void *sorted_y, const void *sorted_z,
                        const uint32_t *sorted_id, const int8_t *sorted_is_ghost,
                        const int32_t *sorted_orig_idx, ft_stream_t stream);

/* Refit-only update of a built tree for moved points (no reference counterpart: the
 * reference rebuilds, test/benchmark/rebuild_scaling.cpp).  x/y/z hold the new positions of
 * the same n points, in the build's input order (leaf_order = 0: leaf i takes the point
 * orig_idx[n-1+i]) or in leaf order (leaf_order = 1).  Keys, leaf order and topology are
 * kept; every box, node record and height is recomputed, so the tree equals the one
 * ft_build_tree makes from the build's sorted keys with the new positions as its leaf
 * arrays.  Queries stay exact; they prune best while the points stay near their cells.
 * Host or device arrays.  Blocking. */
ft_status ft_refit_bvh(ft_context *ctx, const void *x, const void *y, const void *z, size_t n, int leaf_order,
                       ft_tree *tree, ft_stream_t stream);

/* Tree serialisation: the raw SoA arrays the reference ships between ranks
 * (test/test_mpi.cpp:71-101), plus the sorted keys, behind a 128-byte header (magic
 * "FTB2TREE", format version, coordinate / SFC / periodic options, leaf count, build box).
 * Layout, all little-endian, each array starting on a 16-byte boundary: min_x, max_x, min_y,
 * max_y, min_z, max_z ((2n-1) coordinates each), left_child, right_child ((n-1) int32),
 * parent, id, is_ghost (int8), orig_idx ((2n-1) each), key low words (n uint64), key high
 * words (n uint64, 64-bit coordinates only).
 * ft_tree_export: buf == NULL stores the size in *bytes; otherwise *bytes is buf's size.
 * ft_tree_import: the context's options must match the header's and the tree's capacity must
 * hold the leaves; topology, internal boxes and the query records are recomputed from the
 * keys and leaves, so the tree equals the exported one.  buf may be host or device memory.
 * Blocking. */
ft_status ft_tree_export(ft_context *ctx, const ft_tree *tree, void *buf, size_t *bytes, ft_stream_t stream);
ft_status ft_tree_import(ft_context *ctx, const void *buf, size_t bytes, ft_tree *tree, ft_stream_t stream);

/* ---------------------------------------------------------------------------------- */
/* Queries.  Output rows are k wide: idx (size_t, SIZE_MAX when missing) and dist        */
/* (double for float coords, uint64 for integer coords; -DBL_MAX / 0 when missing).     */
/* ---------------------------------------------------------------------------------- */

/* self_knn_query<MAXK> (leaf_ids == NULL, num = tree->num_leaves; src/hlbvh.hpp:1929-1954)
 * and self_knn_query_subset<MAXK> (src/hlbvh.hpp:1956-1983).  leaf_ids: device.  idx_out,
 * dist_out: both device, or both host memory (the reference requires USM here; host
 * buffers are filled chunk by chunk through device staging, each chunk's copy-out
 * overlapping the next chunk's walk -- pinned memory overlaps fully).  Asynchronous on
 * stream, like the reference.  k > max_k -> INVALID_ARGUMENT.  Default max_k: 32 for the
 * full query, 256 for the subset. */
ft_status ft_self_knn(ft_context *ctx, const ft_tree *tree, const int32_t *leaf_ids, size_t num,
                      int k, int exclude_self, uint64_t *idx_out, void *dist_out,
                      const ft_query_options *qopts, ft_stream_t stream);

/* Self-kNN (full, leaf_ids == NULL, or subset) that allocates no device memory itself, for
 * callers that cannot let a library allocate: codes that give the whole GPU to their own
 * memory pool at start-up, or steps that must not be stalled by the device-wide
 * synchronisation of cudaMalloc / cudaFree.  No counterpart in the reference.
 * Same results as ft_self_knn (fast walk with exact replay; the reference traversal when
 * k > 64).  The replay list lives in a fixed array that every
 * GPU loading this library holds until exit: at most 1048576 (2^20) queries per call, more
 * is FT_ERR_INVALID_ARGUMENT.  The first call on a device looks up that array's address;
 * make it before any stream capture.  All calls share the array: calls that overlap on the
 * GPU race and must be serialised by the caller.  leaf_ids, idx_out, dist_out: device.
 * The walk keeps a per-thread stack in local memory, and the first launch on a device may
 * make the driver enlarge its local-memory reservation: make one call before giving the
 * rest of the GPU's memory to a pool.
 * Asynchronous on stream; errors from the kernels surface in ft_check_device_status. */
ft_status ft_self_knn_noalloc(ft_context *ctx, const ft_tree *tree, const int32_t *leaf_ids, size_t num,
                              int k, int exclude_self, uint64_t *idx_out, void *dist_out, ft_stream_t stream);

/* Self-kNN with a per-query pruning bound: the hook of the learned radius bound.  No
 * counterpart in the reference.  bound: device, one value per query in dist_out's units
 * (the squared distance the query returns).  The fast walk prunes every node beyond the
 * bound; a query that ends with its k-th distance above its bound, or with fewer than k
 * points, is rerun by the reference traversal, so the output equals ft_self_knn's for any
 * bound (a good bound only saves work).  k <= 64 uses the bound; other
 * calls take the reference traversal.  Asynchronous. */
ft_status ft_self_knn_bounded(ft_context *ctx, const ft_tree *tree, const int32_t *leaf_ids, size_t num,
                              int k, int exclude_self, const void *bound, uint64_t *idx_out, void *dist_out,
                              const ft_query_options *qopts, ft_stream_t stream);

/* knn_query<MAXK> (src/hlbvh.hpp:1405-1472).  qx/qy/qz, idx_out, dist_out: host or device.
 * Default max_k 256.  Blocking. */
ft_status ft_knn(ft_context *ctx, const ft_tree *tree, const void *qx, const void *qy,
                 const void *qz, size_t num_queries, int k, uint64_t *idx_out, void *dist_out,
                 const ft_query_options *qopts, ft_stream_t stream);

/* range_query (src/hlbvh.hpp:2006-2136).  All arrays host or device.  results: num_queries
 * x max_results_per_query ints (sorted leaf ranks, or input indices with
 * return_orig_indices); counts: the full count (may exceed the row width).  Blocking. */
ft_status ft_range(ft_context *ctx, const ft_tree *tree, const void *qx, const void *qy,
                   const void *qz, const void *r_min, const void *r_max, size_t num_queries,
                   int32_t *results, int32_t *counts, int max_results_per_query,
                   ft_stream_t stream);

/* How ft_range walks trees of height <= 62 on this context: 0 (default), where the box
 * distance is monotone over nested boxes, each query writes its row with a walk over the
 * 4-wide records and stops once the row is full, then the full rows of a warp's 32 queries
 * (neighbours in SFC order) are counted together when their points lie close against the
 * radius (nodes inside every query's shell counted whole, nodes beyond every ball skipped,
 * the leaves between tested per query), else per query; elsewhere one walk per query over the
 * binary records; 1, one walk per query over the binary records; 2, the 32 queries of a warp
 * walk the union of their nodes together, each stack entry with the mask of the queries that
 * need it, when their balls overlap (else one walk each); 3, one 4-wide walk per query where
 * it applies; 4, as 0 with every group counted together whatever its spread.  Same rows and
 * counts either way.  (Taller trees keep the reference's walk with its stack guard.) */
ft_status ft_set_range_walk(ft_context *ctx, int walk);

/* Height of the built tree (root to deepest leaf).  The traversal stack of the reference
 * drops both children of a node popped with 62 entries below it (src/hlbvh.hpp:1152, 1618),
 * which only trees of height >= 63 can reach; on those the fast walk tests each query for
 * it and hands the queries it may affect to the reference traversal. */
ft_status ft_tree_height(ft_context *ctx, const ft_tree *tree, int *height_out);

/* ---------------------------------------------------------------------------------- */
/* Learned radius bound.  No counterpart in the reference.  A 12 -> 64 -> 64 -> 1 GELU MLP  */
/* (bfloat16 weights and activations, fp32 accumulation) predicts each self query's       */
/* log2 k-th-neighbour distance from 12 tree features; the prediction times an inflation   */
/* becomes the query's bound in ft_self_knn_bounded, so results stay identical to         */
/* ft_self_knn's.  The network is trained on the GPU (forward, backward and Adam kernels)  */
/* on targets taken from exact self-kNN results.  k <= 64.                                 */
/* ---------------------------------------------------------------------------------- */
#define FT_BOUND_FEATURES     12   /* features per query (float)                         */
#define FT_BOUND_MODEL_PARAMS 5057 /* W1[64][12] b1[64] W2[64][64] b2[64] w3[64] b3        */

typedef struct ft_bound_model ft_bound_model;

/* New network with seeded U(-1/sqrt(fan_in), 1/sqrt(fan_in)) weights and identity
 * standardisation. */
ft_status ft_bound_model_create(ft_context *ctx, uint64_t seed, ft_bound_model **out);
ft_status ft_bound_model_destroy(ft_context *ctx, ft_bound_model *model);
/* fp32 master weights in the layout above (host arrays of FT_BOUND_MODEL_PARAMS floats);
 * set also resets the Adam state. */
ft_status ft_bound_model_get_params(ft_context *ctx, ft_bound_model *model, float *params_out);
ft_status ft_bound_model_set_params(ft_context *ctx, ft_bound_model *model, const float *params);
/* Input standardisation (host: 12 means, 12 standard deviations) and the target's mean and
 * standard deviation (the network predicts the standardised target). */
ft_status ft_bound_model_set_norm(ft_context *ctx, ft_bound_model *model, const float *feature_mean,
                                  const float *feature_std, float target_mean, float target_std);

/* The 12 features of self queries (leaf_ids NULL: every leaf) of a tree built by
 * ft_build_bvh / ft_build_tree.  features_out: device, num x 12 floats.  Asynchronous. */
ft_status ft_bound_features(ft_context *ctx, const ft_tree *tree, const int32_t *leaf_ids, size_t num, int k,
                            float *features_out, ft_stream_t stream);
/* Training targets from self-kNN results (device idx / dist, num x k): 0.5 log2 of each
 * row's k-th distance, NaN for rows with fewer than k neighbours.  Asynchronous. */
ft_status ft_bound_targets(ft_context *ctx, const uint64_t *idx, const void *dist, size_t num, int k,
                           float *targets_out, ft_stream_t stream);
/* Gradient (host, FT_BOUND_MODEL_PARAMS floats) and loss (host, 1 float) of the mean squared
 * error over all n samples, without an update.  features / targets: device.  Blocking. */
ft_status ft_bound_model_gradient(ft_context *ctx, ft_bound_model *model, const float *features,
                                  const float *targets, size_t n, float *grad_out, float *loss_out,
                                  ft_stream_t stream);
/* `steps` Adam steps (lr; beta 0.9 / 0.999) on minibatches of `batch` rows drawn from [0, n)
 * with a seeded hash.  loss_out: NULL or host, one loss per step (then blocking).  Targets
 * must be finite. */
ft_status ft_bound_model_fit(ft_context *ctx, ft_bound_model *model, const float *features, const float *targets,
                             size_t n, int steps, int batch, float lr, uint64_t seed, float *loss_out,
                             ft_stream_t stream);
/* Predicted log2 k-th distance (pred_out: NULL or device floats) and bound = (inflation x
 * 2^pred)^2 in distance units (bound_out: NULL or device dist values).  Asynchronous. */
ft_status ft_bound_model_predict(ft_context *ctx, ft_bound_model *model, const float *features, size_t n,
                                 float inflation, float *pred_out, void *bound_out, ft_stream_t stream);
/* The 12 features of external query points (knn_query): each point is placed at the SFC
 * rank of its key among the tree's sorted keys (trees from ft_build_bvh without caller
 * keys); the leaf there stands for the point and the window is seen from the point.
 * qx/qy/qz, features_out: device.  Asynchronous. */
ft_status ft_bound_features_points(ft_context *ctx, const ft_tree *tree, const void *qx, const void *qy,
                                   const void *qz, size_t num_queries, int k, float *features_out, ft_stream_t stream);
/* knn_query<MAXK> of external points with the learned bound: features -> bound -> the fast
 * walk; queries whose bound proves too small, or with ties, are rerun by knn_query's own heap
 * tier, so the output equals ft_knn's.  Arrays as ft_knn (host or device).  Blocking. */
ft_status ft_knn_learned(ft_context *ctx, const ft_tree *tree, ft_bound_model *model, const void *qx,
                         const void *qy, const void *qz, size_t num_queries, int k, float inflation,
                         uint64_t *idx_out, void *dist_out, const ft_query_options *qopts, ft_stream_t stream);
/* Features -> bound -> ft_self_knn_bounded in one call (scratch kept in the context).
 * Same output as ft_self_knn.  Asynchronous. */
ft_status ft_self_knn_learned(ft_context *ctx, const ft_tree *tree, ft_bound_model *model, const int32_t *leaf_ids,
                              size_t num, int k, int exclude_self, float inflation, uint64_t *idx_out,
                              void *dist_out, const ft_query_options *qopts, ft_stream_t stream);

/* ---------------------------------------------------------------------------------- */
/* Batched point sets.  No counterpart in the reference: its callers loop over sets and   */
/* call build_bvh (src/hlbvh.hpp:2165-2302) and self_knn_query<MAXK> (1929-1954) once per */
/* set.  Here num_sets independent sets of uneven size lie back to back in x/y/z (set s =  */
/* points [set_offsets[s], set_offsets[s+1])) and go through one launch sequence; every    */
/* set's tree and neighbour rows equal those of its own reference calls (own bounding box  */
/* and keys, own leaf ranks, indices local to the set).                                  */
/*                                                                                         */
/* Keys must fit 63 bits: F32 / F64 coordinates (Morton or Peano-Hilbert) or U32 with      */
/* Peano-Hilbert keys; a U64 context is rejected.  Every array argument is device memory.  */
/* Build and query allocate nothing and never synchronise the host, so they may be        */
/* captured in a CUDA graph; bad offsets (set_offsets[0] != 0, set_offsets[num_sets] !=   */
/* num_points, or a decreasing pair) surface in ft_check_device_status.                   */
/* ---------------------------------------------------------------------------------- */
typedef struct ft_batch ft_batch;

/* Storage for up to max_points points in up to max_sets (<= 2^24) sets. */
ft_status ft_batch_create(ft_context *ctx, size_t max_points, size_t max_sets, ft_batch **out);
ft_status ft_batch_destroy(ft_context *ctx, ft_batch *batch);

/* build_bvh of every set.  set_offsets: num_sets + 1 int64.  id / is_ghost: NULL or
 * num_points entries (NULL: the index within the set / 0, as the reference fills them).
 * Asynchronous. */
ft_status ft_batch_build(ft_context *ctx, ft_batch *batch, const int64_t *set_offsets, size_t num_sets,
                         size_t num_points, const void *x, const void *y, const void *z, const uint32_t *id,
                         const int8_t *is_ghost, ft_stream_t stream);

/* How ft_batch_build builds the sets: FT_METHOD_PERSISTENT, each set whole in one thread
 * block (the persistent launch's builds, without its queries; the trees are the same);
 * otherwise the launch sequence over all points.  Batches of 64-bit integer positions
 * (126-bit keys) always take the per-set builds. */
ft_status ft_batch_set_build_method(ft_context *ctx, ft_batch *batch, int method);

/* self_knn_query<MAXK> of every set: row j (set s = the set holding j) is leaf j - off[s] of
 * set s; indices are that set's leaf ranks (or input indices within the set with
 * return_orig_indices).  idx_out / dist_out: num_points x k.  Default max_k 32; the fast walk
 * with exact replay unless method is FT_METHOD_PLAIN.  Asynchronous. */
ft_status ft_batch_self_knn(ft_context *ctx, ft_batch *batch, int k, int exclude_self, uint64_t *idx_out,
                            void *dist_out, const ft_query_options *qopts, ft_stream_t stream);

/* ft_batch_build + ft_batch_self_knn as one CUDA graph, captured on the first call with
 * these arguments and replayed by later calls with the same arguments (array contents may
 * change between calls).  With method FT_METHOD_DEFAULT or FT_METHOD_PERSISTENT (and k <= 64)
 * the graph holds one persistent kernel: each block builds whole sets (largest first, the
 * same trees as ft_batch_build), then its warps take chunks of queries of the finished sets;
 * tied queries are replayed by a second launch.  FT_METHOD_FAST / FT_METHOD_PLAIN select the
 * launch sequence (ft_batch_build, then ft_batch_self_knn).  Same rows either way.
 * Asynchronous. */
ft_status ft_batch_build_knn(ft_context *ctx, ft_batch *batch, const int64_t *set_offsets, size_t num_sets,
                             size_t num_points, const void *x, const void *y, const void *z, const uint32_t *id,
                             const int8_t *is_ghost, int k, int exclude_self, uint64_t *idx_out, void *dist_out,
                             const ft_query_options *qopts, ft_stream_t stream);

/* The learned bound's 12 features (ft_bound_features) of every leaf of every set of the last
 * build, each computed on its own set's tree: features_out is device memory, num_points x 12
 * floats.  Asynchronous. */
ft_status ft_batch_bound_features(ft_context *ctx, ft_batch *batch, int k, float *features_out, ft_stream_t stream);

/* ft_batch_self_knn with the learned radius bound (k <= 64): the 12 features of every leaf
 * of every set (each set's own tree, parents and keys), the network's bound for each, the
 * fast walk with that bound, a second launch of the walk without the bound for the queries
 * whose bound proved too small, then the replay of tied queries.  Same rows as
 * ft_batch_self_knn.  The first call on a batch allocates its feature and bound scratch
 * (13 floats per point of max_points); later calls allocate nothing.  The model must live as
 * long as the call runs.  Asynchronous. */
ft_status ft_batch_self_knn_learned(ft_context *ctx, ft_batch *batch, ft_bound_model *model, int k, int exclude_self,
                                    float inflation, uint64_t *idx_out, void *dist_out, const ft_query_options *qopts,
                                    ft_stream_t stream);

/* ft_batch_build + ft_batch_self_knn_learned as one CUDA graph (captured on the first call
 * with these arguments, replayed by later calls; the scratch is allocated before the
 * capture).  The graph reads the model's weights when it runs, so a retrained model is
 * used as it stands; destroying the model while the batch may still replay the graph is
 * an error of the caller.  Asynchronous. */
ft_status ft_batch_build_knn_learned(ft_context *ctx, ft_batch *batch, ft_bound_model *model, float inflation,
                                     const int64_t *set_offsets, size_t num_sets, size_t num_points, const void *x,
                                     const void *y, const void *z, const uint32_t *id, const int8_t *is_ghost, int k,
                                     int exclude_self, uint64_t *idx_out, void *dist_out,
                                     const ft_query_options *qopts, ft_stream_t stream);

/* View of one built set as an ft_tree (arrays inside the batch; valid until the next build
 * of the batch).  Usable with every query entry point; not with builds, ensure or destroy.
 * Blocking. */
ft_status ft_batch_tree(ft_context *ctx, ft_batch *batch, size_t set, ft_tree *out, ft_stream_t stream);

/* Per-set bounding boxes (host, 6 coordinates per set, or NULL) and tree heights (host,
 * one byte per set, or NULL) of the last build.  Blocking. */
ft_status ft_batch_set_info(ft_context *ctx, ft_batch *batch, void *bbox_out, uint8_t *height_out,
                            ft_stream_t stream);

/* Replay count and visits of the last ft_batch_self_knn / ft_batch_build_knn (synchronises). */
ft_status ft_batch_query_stats(ft_context *ctx, ft_batch *batch, ft_query_stats *out);

/* ---------------------------------------------------------------------------------- */
/* Autotuner.  The reference picks one kernel shape per device: the sub-group width from  */
/* get_native_sub_group_width and its MAXK dispatchers (src/hlbvh.hpp:1828-1927).  Here    */
/* every candidate returns the same rows bit for bit, so the tuner times the candidates on  */
/* the caller's own data and keeps the fastest per shape (kind, k, size class floor(log2    */
/* n)) in the context; later calls with default options (ft_query_options zeroed past       */
/* method) take it.  Each tuner checks on the device that every candidate's rows (the leaf  */
/* order, for the build) equal the default's and fails with FT_ERR_RUNTIME otherwise.       */
/* Blocking; they allocate scratch of their own.                                            */
/* ---------------------------------------------------------------------------------- */
typedef struct ft_tune_result {
    int32_t walk_variant;  /* fast walk: 2 compact binary, 4 4-wide per-lane, 5 group walk  */
    int32_t half_window;   /* SFC seeding half-window                                      */
    int32_t block_threads; /* 64 (two warps, 32-entry heap template) or 32 (one warp)      */
    int32_t sort_items;    /* build: keys per thread of a onesweep tile                    */
    int32_t candidates;    /* configurations timed                                         */
    float   best_ms;       /* the sample's time with the choice                            */
    float   default_ms;    /* and with the defaults                                        */
    int32_t reserved[9];
} ft_tune_result;

/* Self-kNN on `tree` at k (1..64): walk variant x half-window x block shape, timed on up to
 * 2^18 of its queries (four stretches of consecutive leaves). */
ft_status ft_tune_self_knn(ft_context *ctx, const ft_tree *tree, int k, int exclude_self, ft_tune_result *out,
                           ft_stream_t stream);
/* The batched self-kNN of the batch's last build at k (1..64), timed on the whole batch. */
ft_status ft_tune_batch_self_knn(ft_context *ctx, ft_batch *batch, int k, int exclude_self, ft_tune_result *out,
                                 ft_stream_t stream);
/* build_bvh of these points (host or device, as ft_build_bvh): the sort's tile size, timed
 * over whole builds into `tree` (left holding the last candidate's build, equal to any). */
ft_status ft_tune_build(ft_context *ctx, const void *x, const void *y, const void *z, size_t n, ft_tree *tree,
                        ft_tune_result *out, ft_stream_t stream);
/* Forgets every choice the tuners made on this context. */
ft_status ft_tune_reset(ft_context *ctx);

/* ---------------------------------------------------------------------------------- */
/* Build stage timing (the reference reports per-stage build times in its profiling notes):  */
/* with profiling on, ft_build_bvh records CUDA events on its stream between its stages;   */
/* ft_get_build_profile returns the last profiled build's stage times (synchronises).       */
/* ---------------------------------------------------------------------------------- */
typedef struct ft_build_profile {
    float   bbox_ms;      /* compute_bbox                                                  */
    float   encode_ms;    /* SFC keys + permutation                                        */
    float   sort_ms;      /* key + permutation sort                                        */
    float   gather_ms;    /* leaf gather                                                   */
    float   topology_ms;  /* Karras topology                                               */
    float   refit_ms;     /* bottom-up refit (boxes, node records, heights)                */
    float   records_ms;   /* 4-wide records of the fast walk                               */
    float   total_ms;
    int32_t reserved[8];
} ft_build_profile;
ft_status ft_set_build_profiling(ft_context *ctx, int enable);
ft_status ft_get_build_profile(ft_context *ctx, ft_build_profile *out);

#ifdef __cplusplus
}
#endif

#endif /* FASTTREE_B200_H */
