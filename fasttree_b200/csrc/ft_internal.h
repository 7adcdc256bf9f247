// ft_internal.h -- host-side structures shared by the build, query and C-ABI units.
#pragma once

#include <cuda_runtime.h>
#include <stddef.h>
#include <stdint.h>

#include <map>
#include <string>
#include <type_traits>

#include "../../include/fasttree_b200.h"

namespace ft {

// Error carried from deep inside the library to the C ABI.
struct Error {
    ft_status   status;
    std::string msg;
};

[[noreturn]] void fail(ft_status s, const std::string &msg);
void              check_cuda(cudaError_t e, const char *what);
#define FT_CUDA(call) ::ft::check_cuda((call), #call)

// Device status word bits (written by kernels instead of trapping).
enum : uint32_t { STATUS_SPIN_LIMIT = 1u, STATUS_TRAVERSAL_LIMIT = 2u, STATUS_BAD_INPUT = 4u };

// Library-owned per-tree acceleration data and build scratch (the persistent part plays
// the role of the reference's BvhScratch, src/hlbvh.hpp:720-745).
struct TreeImpl {
    size_t    cap          = 0; // leaf capacity
    int       coord        = 0;
    void     *recs         = nullptr; // NodeRec<T>[cap-1]
    uint8_t  *height       = nullptr; // subtree height of internal nodes
    int32_t  *counters     = nullptr; // refit arrival counters
    int32_t  *leafcount    = nullptr; // leaves under each internal node (Karras range size)
    void     *wide         = nullptr; // WideRec<T>[cap-1]: grandchildren of each internal node
    uint64_t *key_lo       = nullptr; // sorted keys (low word)
    uint64_t *key_hi       = nullptr; // sorted keys (high word, 126-bit keys only)
    uint64_t *tmp_lo       = nullptr; // sort ping-pong
    uint64_t *tmp_hi       = nullptr;
    uint32_t *perm         = nullptr; // sorted permutation (original index per leaf rank)
    uint32_t *tmp_perm     = nullptr;
    void     *bbox         = nullptr; // 6 coords on the device
    void     *bbox_partial = nullptr; // per-block partial boxes
    uint32_t *hist         = nullptr; // [digit position][256] counts, then offsets
    uint32_t *lookback     = nullptr; // onesweep tile status
    size_t    lookback_words = 0;
    uint32_t *tile_counter = nullptr; // per-pass tile ticket
    uint32_t *status       = nullptr; // device status word
    bool      managed      = false;
    int       height_root  = -1;    // host copy after a build
    bool      clean42      = false; // 64-bit integer tree with every coordinate below 2^42
    bool      clean42_ok   = false; // the tree may use that form (built by build_bvh)
    bool      in_period    = true;  // integer coordinates all below 2^bits (42 for 64-bit, 21
                                    // for 32-bit): the periodic distance is then monotone over
                                    // nested boxes, which the fast walks rely on
    bool      view         = false; // one set of a batch: arrays owned by the batch, no builds
    bool      own_keys     = false; // key_lo / key_hi hold keys this library encoded (build_bvh
                                    // without caller keys), with the box in bbox
};

// Batched trees: S independent trees stored back to back.  Set s owns leaves (queries)
// [off[s], off[s+1]); its nodes start at node_off[s] in the node arrays and its internal
// records / child arrays at rec_off[s].  Inside a set, indices follow TreeSoA's layout.
// All arrays live on the device.
struct BatchDev {
    const long long *off      = nullptr; // S + 1 leaf offsets (null: a single tree)
    const long long *node_off = nullptr;
    const long long *rec_off  = nullptr;
    const uint8_t   *height   = nullptr; // root height of each set's tree
    int              S        = 0;
};

// Distance mode of query kernels on this tree (see met_dispatch in ft_common.cuh).
// The fast walks return the reference's rows only when the box distance never exceeds the
// distance to any point inside the box.  Every metric has that property except the periodic
// integer one on coordinates at or above the period (2^42 / 2^21), whose unmasked box bounds
// break it; such trees keep the reference traversal.
inline bool fast_walk_applies(const ft_options &o, const TreeImpl &t) {
    return !o.periodic || o.coord_type == FT_COORD_F32 || o.coord_type == FT_COORD_F64 || t.in_period;
}

template <class T> inline int metric_mode(const ft_options &o, const ft_tree &t) {
    if (std::is_floating_point<T>::value || !o.periodic) return 0;
    return (sizeof(T) == 8 && ((const TreeImpl *)t.impl)->clean42) ? 2 : 1;
}

// The autotuner's choice for one shape (0: the built-in default of that parameter).
struct TuneChoice {
    int variant = 0; // fast walk variant (walk_variant's numbering)
    int half    = 0; // SFC seeding half-window
    int kc      = 0; // heap template of the walk: 32 (two-warp blocks) or 64 (one-warp blocks)
    int items   = 0; // keys per thread of a onesweep tile (build)
};
enum TuneKind { TUNE_SELF_KNN = 0, TUNE_BATCH = 1, TUNE_BUILD = 2 };
// Shape key: kind, k (or key words for the build) and the size class floor(log2 n).
inline unsigned long long tune_key(int kind, int k, size_t n) {
    int l = 0;
    while (n > 1) {
        n >>= 1;
        ++l;
    }
    return ((unsigned long long)kind << 48) | ((unsigned long long)(unsigned)k << 16) | (unsigned long long)l;
}

// Stage timing of build_bvh (ft_set_build_profiling): events recorded on the build's stream
// between its stages.
enum BuildStage { BS_START, BS_BBOX, BS_ENCODE, BS_SORT, BS_GATHER, BS_TOPOLOGY, BS_REFIT, BS_RECORDS, BS_COUNT };
struct BuildProfile {
    bool        on       = false;
    bool        recorded = false; // the last build recorded every stage
    cudaEvent_t ev[BS_COUNT] = {};
};

struct Context {
    ft_options     opts{};
    int            device = 0;
    int            num_sms = 148;
    ft_query_stats stats{};
    uint32_t      *status = nullptr; // [0] status word of query kernels, [1] replay count,
                                     // [2..3] visits, [4] bound misses (8 words)
    int32_t       *replay_ranks = nullptr; // queries the fast traversal hands to the exact one
    int32_t       *replay_rows  = nullptr;
    int32_t       *seed_ranks   = nullptr; // SFC rank of each external query (fast knn)
    size_t         replay_cap   = 0;
    int32_t       *miss_ranks   = nullptr; // queries whose pruning bound proved too small
    int32_t       *miss_rows    = nullptr;
    size_t         miss_cap     = 0;
    bool           last_fast    = false; // the last self-kNN call used the fast traversal
    bool           last_rows    = false; // replay_rows holds the last fast call's replayed rows
    TreeImpl       qsort;                   // sort scratch of external queries (fast knn)
    void          *stage_idx[2]  = {nullptr, nullptr}; // device staging of host-output self-kNN
    void          *stage_dist[2] = {nullptr, nullptr};
    size_t         stage_cap     = 0;       // rows x k per staging buffer
    int32_t       *iota          = nullptr; // leaf ranks 0 .. iota_cap-1
    size_t         iota_cap      = 0;
    cudaStream_t   copy_stream   = nullptr;
    cudaEvent_t    ev_walked[2]  = {nullptr, nullptr};
    cudaEvent_t    ev_copied[2]  = {nullptr, nullptr};
    std::map<unsigned long long, TuneChoice> tuned; // autotuner choices by shape (tune_key)
    BuildProfile   bprof;
    int            range_walk = 0; // range_query, trees of height <= 62: 0 default, 1 binary, 2 warp-shared, 3 4-wide, 4 group counts forced
    float         *learned_feats = nullptr; // learned-bound scratch: features and bounds
    void          *learned_bound = nullptr;
    size_t         learned_cap   = 0;
};

// ---- fast self-kNN (ft_fast.cu) ----
// Returns false when the fast traversal does not apply (k > 64, a periodic tree with
// coordinates beyond the period).
// half_window / variant / kc <= 0: the autotuner's choice for the shape when there is one,
// else the defaults.
bool fast_self_knn(Context &ctx, const ft_tree &tree, const int32_t *leaf_ids, size_t num, int k, bool exclude_self,
                   uint64_t *idx, void *dist, const void *bound, int half_window, int variant, cudaStream_t st,
                   int kc = 0);
void ensure_replay(Context &ctx, size_t num);
// Fast self-kNN whose scratch is a fixed static device array (no allocation); false when
// the fast walk does not apply.  At most noalloc_max_queries() queries per call.
bool   fast_self_knn_noalloc(Context &ctx, const ft_tree &tree, const int32_t *leaf_ids, size_t num, int k,
                             bool exclude_self, uint64_t *idx, void *dist, cudaStream_t st);
size_t noalloc_max_queries();
// Reruns the listed self queries (ranks[i] -> row rows[i], *count_dev of them) with the
// reference traversal (ft_query.cu).
void replay_exact(Context &ctx, const ft_tree &tree, const int32_t *ranks, const int32_t *rows, uint32_t *count_dev,
                  int k, bool exclude_self, uint64_t *idx, void *dist, cudaStream_t st, const BatchDev &bt = {});
// Self-kNN over every leaf of a batch of trees (`all` spans the concatenated arrays):
// the fast walk with its replay (replay lists rr / rw, counters = 4 device words) or, with
// fast == false or k > 64, the reference traversal.  No allocation, no host synchronisation.
// With a per-query bound (device, dist units) the queries whose bound proves too small go
// through the miss list (mw, counters[4]) to a second launch of the walk without the bound.
void batch_self_knn(Context &ctx, const ft_tree &all, const BatchDev &bt, size_t num, int k, bool exclude_self,
                    uint64_t *idx, void *dist, bool fast, int half_window, int variant, int32_t *rr, int32_t *rw,
                    uint32_t *counters, cudaStream_t st, const void *bound = nullptr, int32_t *mw = nullptr,
                    int kc = 0);
// The persistent batched launch (ft_fast.cu): one kernel whose blocks first build whole sets
// (largest first, one set per block, ft_cta_build.cuh), each published when done, then take
// chunks of queries of the published sets and walk them (the fast walk; tied queries go to
// the replay list).  With query == false only the builds run.  The scheduling words (ctl,
// ready, chunk_next) must be zeroed / set to -1 on the stream before the launch.
struct PersistLaunch {
    const long long *off = nullptr, *node_off = nullptr, *rec_off = nullptr; // prepared offsets
    int              S   = 0;
    const void      *x = nullptr, *y = nullptr, *z = nullptr;
    const uint32_t  *id    = nullptr;
    const int8_t    *ghost = nullptr;
    ft_tree          all{};        // the batch's node arrays
    TreeImpl        *scr = nullptr; // records, heights, counters, leaf counts and key buffers
    void            *bbox       = nullptr; // 6 coordinates per set
    uint8_t         *set_height = nullptr;
    const int32_t   *order = nullptr; // build order of the sets (largest first)
    int32_t         *ready = nullptr; // sets in the order their builds finished (-1: not yet)
    int32_t         *chunk_next = nullptr;
    uint32_t        *ctl        = nullptr; // [0] build tickets, [1] ready slots, [2] query cursor
    bool             query      = true;
    int              k          = 0;
    bool             excl       = true;
    uint64_t        *idx        = nullptr;
    void            *dist       = nullptr;
    int32_t         *rr = nullptr, *rw = nullptr;
    uint32_t        *counters   = nullptr; // [0] replay count, [2..3] visits
};
void batch_persistent(Context &ctx, const PersistLaunch &p, cudaStream_t st);
// The reference traversal over every leaf of a batch (ft_query.cu).
void batch_self_knn_exact(Context &ctx, const ft_tree &all, const BatchDev &bt, size_t num, int k, bool exclude_self,
                          uint64_t *idx, void *dist, cudaStream_t st);

// Fast kNN of external query points (knn_query): the same walk seeded from the SFC window
// around each query's key rank; tied queries replayed by the reference's heap tier.  False
// when it does not apply (k > 64, k equal to the merge heap's capacity).
void free_query_sort(Context &ctx);
// Order of external query points along the tree's SFC (sorted by each point's key rank), so
// that neighbouring threads take neighbouring queries; null when the tree's keys are not
// this library's own encoding.  Valid until the next call on the context.
const uint32_t *sfc_query_order(Context &ctx, const ft_tree &tree, const void *qx, const void *qy, const void *qz,
                                size_t nq, cudaStream_t st);
void recompute_from_keys(Context &ctx, ft_tree &tree, cudaStream_t st);
void refit_bvh(Context &ctx, ft_tree &tree, const void *x, const void *y, const void *z, size_t n, bool leaf_order,
               cudaStream_t st);
bool fast_knn(Context &ctx, const ft_tree &tree, const void *qx, const void *qy, const void *qz, size_t nq, int k,
              int max_k, uint64_t *idx, void *dist, int half_window, cudaStream_t st, const void *bound = nullptr,
              int walk = 0);
// SFC rank of each external query point in ctx.seed_ranks (-1 without this library's keys).
void query_seed_ranks(Context &ctx, const ft_tree &tree, const void *qx, const void *qy, const void *qz, size_t nq,
                      cudaStream_t st);
// Reruns listed external queries (rows, *count_dev of them) with knn_query's heap tier.
void replay_external(Context &ctx, const ft_tree &tree, const void *qx, const void *qy, const void *qz,
                     const int32_t *rows, uint32_t *count_dev, int k, int max_k, uint64_t *idx, void *dist,
                     cudaStream_t st);

// Reads and clears a device status word (synchronises the stream); throws on a set bit.
void check_device_status(uint32_t *status, cudaStream_t st);

// ---- autotuner (ft_tune.cu) ----
// Each times its candidates on the caller's data, checks that every candidate returns the
// default's rows (leaf order for the build), and keeps the fastest in ctx.tuned.
void tune_self_knn(Context &ctx, const ft_tree &tree, int k, bool exclude_self, ft_tune_result *out, cudaStream_t st);
void tune_batch_self_knn(Context &ctx, const ft_tree &all, const BatchDev &bt, size_t num, int k, bool exclude_self,
                         int32_t *rr, int32_t *rw, uint32_t *counters, ft_tune_result *out, cudaStream_t st);
void tune_build(Context &ctx, ft_tree &tree, const void *x, const void *y, const void *z, size_t n,
                ft_tune_result *out, cudaStream_t st);

// Records build stage i on st when build profiling is on.
inline void stage_mark(Context *ctx, int i, cudaStream_t st) {
    if (ctx && ctx->bprof.on) cudaEventRecord(ctx->bprof.ev[i], st);
}

// ---- build (ft_build.cu) ----
// sort_items: keys per thread of the sort's tiles (0: the autotuner's choice for the shape,
// else the default).
void build_bvh(Context &ctx, ft_tree &tree, const void *x, const void *y, const void *z, size_t n,
               const uint32_t *id, const int8_t *ghost, const void *bbox_host, void *caller_keys_dev,
               cudaStream_t st, int sort_items = 0);
// Tile sizes the build's sort offers for one- or two-word keys (the default first).
const int *sort_item_choices(int words, int *count);
int        key_words_of(const ft_options &o);
void build_tree_from_keys(Context &ctx, ft_tree &tree, const void *keys_ref_dev, const void *sx,
                          const void *sy, const void *sz, const uint32_t *sid, const int8_t *sghost,
                          const int32_t *sorig, cudaStream_t st);
void compute_bbox(Context &ctx, TreeImpl *scratch, const void *x, const void *y, const void *z, size_t n,
                  void *bbox_dev, cudaStream_t st);
void sfc_encode_ref_layout(Context &ctx, TreeImpl &scratch, const void *x, const void *y, const void *z,
                           size_t n, const void *bbox_dev, void *keys_ref_dev, cudaStream_t st);
size_t ref_key_bytes(const ft_options &o);
// Onesweep sort of (key_lo[, key_hi], perm) in s over a fixed digit list (8-bit digits,
// d < 8: low word, 8 <= d < 16: high word); no host synchronisation.
void   sort_pairs_fixed(TreeImpl &s, size_t n, int words, int ndigits, const int *digits, cudaStream_t st);
size_t sort_lookback_words(size_t n, int words);
void   ensure_scratch(TreeImpl &impl, const ft_options &o, size_t n);
void   free_scratch(TreeImpl &impl);

// ---- queries (ft_query.cu) ----
// bound: optional per-query pruning bound (device, dist units); it selects the fast walk.
void self_knn(Context &ctx, const ft_tree &tree, const int32_t *leaf_ids, size_t num, int k,
              bool exclude_self, uint64_t *idx, void *dist, const ft_query_options &q, cudaStream_t st,
              const void *bound = nullptr);
// Self-kNN into host memory with the copy-out overlapped (chunks walked into two device
// buffers in turn; copies on a second stream).
void self_knn_to_host(Context &ctx, const ft_tree &tree, const int32_t *leaf_ids, size_t num, int k,
                      bool exclude_self, uint64_t *h_idx, void *h_dist, const ft_query_options &q, cudaStream_t st);
// bound: optional per-query pruning bound (device, dist units); it selects the fast walk.
void knn(Context &ctx, const ft_tree &tree, const void *qx, const void *qy, const void *qz, size_t nq,
         int k, int max_k, uint64_t *idx, void *dist, const ft_query_options &q, cudaStream_t st,
         const void *bound = nullptr);
void range(Context &ctx, const ft_tree &tree, const void *qx, const void *qy, const void *qz,
           const void *rmin, const void *rmax, size_t nq, int32_t *results, int32_t *counts,
           int max_per_q, cudaStream_t st);

size_t coord_bytes(int coord);
inline size_t wide_bytes(int coord) { return coord_bytes(coord) == 8 ? 208 : 112; } // sizeof(WideRec<T>)

// ---- batched sets (ft_batch.cu) ----
struct BatchImpl;
BatchImpl *batch_create(Context &ctx, size_t max_points, size_t max_sets);
void       batch_free(BatchImpl *b);
// ft_batch_build's method: FT_METHOD_PERSISTENT builds every set in one block (the
// persistent launch without its queries), otherwise the launch sequence (126-bit keys always
// take the per-set builds).
void batch_set_build_method(BatchImpl &b, int method);
// set_offsets: device, S + 1 entries.  Asynchronous; no allocation, no host synchronisation.
void batch_build(Context &ctx, BatchImpl &b, const long long *set_offsets, size_t S, size_t N, const void *x,
                 const void *y, const void *z, const uint32_t *id, const int8_t *ghost, cudaStream_t st);
struct BoundModel;
// model: null, or the learned radius bound (its scratch must exist: batch_query_learned or a
// graph with the model makes it).
void batch_query(Context &ctx, BatchImpl &b, int k, bool exclude_self, uint64_t *idx, void *dist,
                 const ft_query_options &q, cudaStream_t st, BoundModel *model = nullptr, float inflation = 0.0f);
// The learned bound's 12 features of every leaf of every set (device, N x 12 floats).
void batch_features(Context &ctx, BatchImpl &b, int k, float *out, cudaStream_t st);
void batch_query_learned(Context &ctx, BatchImpl &b, BoundModel &model, int k, bool exclude_self, float inflation,
                         uint64_t *idx, void *dist, const ft_query_options &q, cudaStream_t st);
void batch_build_query_graph(Context &ctx, BatchImpl &b, const long long *set_offsets, size_t S, size_t N,
                             const void *x, const void *y, const void *z, const uint32_t *id, const int8_t *ghost,
                             int k, bool exclude_self, uint64_t *idx, void *dist, const ft_query_options &q,
                             cudaStream_t st, BoundModel *model = nullptr, float inflation = 0.0f);
void batch_tree_view(Context &ctx, BatchImpl &b, size_t set, ft_tree &out, cudaStream_t st);
void batch_set_info(Context &ctx, BatchImpl &b, void *bbox_out, uint8_t *height_out, cudaStream_t st);
void batch_stats(BatchImpl &b, ft_query_stats &out);
void batch_tune(Context &ctx, BatchImpl &b, int k, bool exclude_self, ft_tune_result *out, cudaStream_t st);

// ---- learned radius bound (ft_learned.cu) ----
struct BoundModel;
BoundModel *bound_model_create(Context &ctx, unsigned long long seed);
void        bound_model_free(BoundModel *b);
void        bound_model_get_params(BoundModel &b, float *host);
void        bound_model_set_params(BoundModel &b, const float *host, cudaStream_t st);
void        bound_model_set_norm(BoundModel &b, const float *mean12, const float *std12, float t_mean, float t_std);
void        bound_features(Context &ctx, const ft_tree &tr, const int32_t *leaf_ids, size_t num, int k, float *out,
                           cudaStream_t st);
void        bound_targets(Context &ctx, const uint64_t *idx, const void *dist, size_t num, int k, float *out,
                          cudaStream_t st);
void        bound_model_gradient(BoundModel &b, const float *feats, const float *targets, int n, float *grad_host,
                                 float *loss_host, cudaStream_t st);
void        bound_model_fit(BoundModel &b, const float *feats, const float *targets, int n, int steps, int batch,
                            float lr, unsigned long long seed, float *loss_host, cudaStream_t st);
void        bound_model_predict(Context &ctx, BoundModel &b, const float *feats, size_t n, float inflation,
                                float *pred, void *bound, cudaStream_t st);
// Features of every leaf of a batch of sets (BatchDev over the concatenated arrays of `all`).
void        bound_features_batch(Context &ctx, const ft_tree &all, const BatchDev &bt, size_t num, int k, float *out,
                                 cudaStream_t st);
void        bound_features_points(Context &ctx, const ft_tree &tr, const void *qx, const void *qy, const void *qz,
                                  size_t nq, int k, float *out, cudaStream_t st);
void        knn_learned(Context &ctx, const ft_tree &tr, BoundModel &b, const void *qx, const void *qy,
                        const void *qz, size_t nq, int k, int max_k, float inflation, uint64_t *idx, void *dist,
                        const ft_query_options &q, cudaStream_t st);
void        self_knn_learned(Context &ctx, const ft_tree &tr, BoundModel &b, const int32_t *leaf_ids, size_t num,
                             int k, bool exclude_self, float inflation, uint64_t *idx, void *dist,
                             const ft_query_options &q, cudaStream_t st);

} // namespace ft
