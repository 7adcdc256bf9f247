// ft_batch.cu -- thousands of independent point sets of uneven size built and queried
// together.  No counterpart in the reference: every set behaves exactly like its own
// build_bvh (src/hlbvh.hpp:2165-2290) + self_knn_query (1929-1954) call on that set's
// points -- its own bounding box and keys, its own leaf ranks and tree, indices local to
// the set -- but all sets go through one sequence of launches.
//
// Launch sequence (no host synchronisation and no allocation, so it can be captured in a
// CUDA graph and replayed):
//  1. prep      one block: validates the set offsets and scans them into node / record
//               offsets (set s owns nodes [node_off[s], +2n_s-1) and internal records
//               [rec_off[s], +n_s-1)).
//  2. bbox      chunks of 4096 points, each chunk folds every set
//               segment it overlaps and merges it into the set's box with order-preserving
//               integer atomics (min / max are exact, so the order does not matter).
//  3. encode    per point: the set's quantisation parameters -> 63-bit SFC key; perm = i.
//  4. sort      LSD onesweep over the 8 key digits, then over the set id of each element's
//               point: a stable sort by (set, key, input index), which inside each set is
//               the single-tree order (keys, ties by input index).
//  5. gather    per sorted position: leaf slot of its set, local id / orig index, and the
//               key again (recomputed from the point) for the topology.
//  6. karras    per internal node of every set (Karras 2012 on the set's key range).
//  7. refit     per leaf of every set; then each set's root height.
//  8. queries   the fast self-kNN walk with each lane on its own set's tree, and the exact
//               replay; or the reference traversal per set.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>
#include <memory>
#include <string>
#include <vector>

#include "ft_build_dev.cuh"
#include "ft_common.cuh"
#include "ft_cta_build.cuh"
#include "ft_internal.h"

namespace ft {

static constexpr int kPrepThreads = 1024;
static constexpr int kChunk       = kBboxThreads * 16; // points per bbox chunk

// =========================================================================================
// 1. prep: offsets check + node / record offsets.  Invalid offsets (off[0] != 0, off[S] != N
// or a decreasing pair) set STATUS_BAD_INPUT and are replaced by a safe layout (every point
// in the last set), so that no later launch leaves its buffers.
// =========================================================================================
__global__ void __launch_bounds__(kPrepThreads)
    batch_prep_kernel(const long long *__restrict__ in_off, int S, long long N, long long *off, long long *node_off,
                      long long *rec_off, uint32_t *status) {
    __shared__ int       s_bad;
    __shared__ long long s_warp[kPrepThreads / 32];
    __shared__ long long s_carry;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    if (tid == 0) {
        s_bad   = (in_off[0] != 0 || in_off[S] != N) ? 1 : 0;
        s_carry = 0;
    }
    __syncthreads();
    for (int s = tid; s < S; s += kPrepThreads)
        if (in_off[s + 1] < in_off[s]) s_bad = 1;
    __syncthreads();
    const bool bad = s_bad != 0;
    if (bad && tid == 0) atomicOr(status, STATUS_BAD_INPUT);
    // off[s] and the number of non-empty sets before s (block scan in chunks of 1024)
    for (int base = 0; base <= S; base += kPrepThreads) {
        const int s  = base + tid;
        long long o  = 0;
        int       ne = 0;
        if (s <= S) {
            o  = bad ? (s == S ? N : 0) : in_off[s];
            ne = (s < S && (bad ? (s == S - 1 && N > 0) : in_off[s + 1] > in_off[s])) ? 1 : 0;
        }
        long long incl = ne;
#pragma unroll
        for (int d = 1; d < 32; d <<= 1) {
            long long v = __shfl_up_sync(0xffffffffu, incl, d);
            if (lane >= d) incl += v;
        }
        if (lane == 31) s_warp[warp] = incl;
        __syncthreads();
        long long pre = s_carry;
        for (int w = 0; w < warp; ++w) pre += s_warp[w];
        const long long before = pre + incl - ne; // non-empty sets before s
        if (s <= S) {
            off[s]      = o;
            node_off[s] = 2 * o - before;
            rec_off[s]  = o - before;
        }
        __syncthreads();
        if (tid == kPrepThreads - 1) s_carry = pre + incl;
        __syncthreads();
    }
}

// =========================================================================================
// 2. per-set boxes (the keys of float coordinates depend on them)
// =========================================================================================
template <class T>
__global__ void __launch_bounds__(kBboxThreads)
    batch_bbox_kernel(const long long *__restrict__ off, int S, long long N, const T *__restrict__ x,
                      const T *__restrict__ y, const T *__restrict__ z, typename Ord<T>::type *bmin,
                      typename Ord<T>::type *bmax) {
    for (long long c0 = blockIdx.x * (long long)kChunk; c0 < N; c0 += (long long)gridDim.x * kChunk) {
        const long long c1 = min(c0 + (long long)kChunk, N);
        for (int s = find_set(off, S, c0);; ++s) {
            const long long a = max(off[s], c0), b = min(off[s + 1], c1);
            if (b > a) { // uniform over the block
                T m[6];
                bb_identity(m);
                for (long long i = a + threadIdx.x; i < b; i += blockDim.x) {
                    T v[6] = {x[i], x[i], y[i], y[i], z[i], z[i]};
                    bb_fold(m, v);
                }
                bb_block_reduce(m);
                if (threadIdx.x == 0) {
#pragma unroll
                    for (int d = 0; d < 3; ++d) {
                        atomicMin(bmin + 3 * (size_t)s + d, Ord<T>::bits(m[2 * d]));
                        atomicMax(bmax + 3 * (size_t)s + d, Ord<T>::bits(m[2 * d + 1]));
                    }
                }
                __syncthreads();
            }
            if (off[s + 1] >= c1 || s + 1 >= S) break;
        }
    }
}

// Box of each set in the coordinate type and, for float coordinates, its quantisation
// parameters {lo, inv} per axis.
template <class T>
__global__ void batch_params_kernel(int S, const typename Ord<T>::type *bmin, const typename Ord<T>::type *bmax,
                                    T *bbox, T *par) {
    for (int s = blockIdx.x * blockDim.x + threadIdx.x; s < S; s += gridDim.x * blockDim.x) {
#pragma unroll
        for (int d = 0; d < 3; ++d) {
            const T lo = Ord<T>::value(bmin[3 * (size_t)s + d]), hi = Ord<T>::value(bmax[3 * (size_t)s + d]);
            bbox[6 * (size_t)s + 2 * d]     = lo;
            bbox[6 * (size_t)s + 2 * d + 1] = hi;
            if constexpr (Coord<T>::is_float)
                sfc_axis_params(lo, hi, par[6 * (size_t)s + 2 * d], par[6 * (size_t)s + 2 * d + 1]);
        }
    }
}

// =========================================================================================
// 3. keys
// =========================================================================================
template <class T, int SFC>
__global__ void __launch_bounds__(256)
    batch_encode_kernel(const long long *__restrict__ off, int S, long long N, const T *__restrict__ x,
                        const T *__restrict__ y, const T *__restrict__ z, const T *__restrict__ par,
                        unsigned long long *klo, uint32_t *perm) {
    __shared__ uint8_t s_rot[48 * 8], s_sub[48 * 8];
    for (int i = threadIdx.x; i < 48 * 8; i += blockDim.x) {
        s_rot[i] = c_rot[i];
        s_sub[i] = c_sub[i];
    }
    __syncthreads();
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < N; i += (long long)gridDim.x * blockDim.x) {
        const T *p = Coord<T>::is_float ? par + 6 * (size_t)find_set(off, S, i) : nullptr;
        unsigned long long hi, lo;
        encode_point<T, SFC>(x[i], y[i], z[i], p, s_rot, s_sub, hi, lo);
        klo[i]  = lo;
        perm[i] = (uint32_t)i;
    }
}

// 4b. set id of each sorted element's point: the key of the final sort passes.
__global__ void batch_set_key_kernel(const long long *__restrict__ off, int S, long long N,
                                     const uint32_t *__restrict__ perm, unsigned long long *klo) {
    for (long long j = blockIdx.x * (long long)blockDim.x + threadIdx.x; j < N; j += (long long)gridDim.x * blockDim.x)
        klo[j] = (unsigned long long)find_set(off, S, (long long)perm[j]);
}

// =========================================================================================
// 5. gather: sorted position j (set s, leaf rank j - off[s]) <- point perm[j]
// =========================================================================================
template <class T, int SFC>
__global__ void __launch_bounds__(256)
    batch_gather_kernel(const long long *__restrict__ off, const long long *__restrict__ node_off, int S, long long N,
                        const T *__restrict__ x, const T *__restrict__ y, const T *__restrict__ z,
                        const T *__restrict__ par, const uint32_t *__restrict__ perm, const uint32_t *__restrict__ id,
                        const int8_t *__restrict__ ghost, T *mnx, T *mxx, T *mny, T *mxy, T *mnz, T *mxz,
                        uint32_t *id_out, int8_t *ghost_out, int32_t *orig_out, unsigned long long *klo) {
    __shared__ uint8_t s_rot[48 * 8], s_sub[48 * 8];
    for (int i = threadIdx.x; i < 48 * 8; i += blockDim.x) {
        s_rot[i] = c_rot[i];
        s_sub[i] = c_sub[i];
    }
    __syncthreads();
    for (long long j = blockIdx.x * (long long)blockDim.x + threadIdx.x; j < N; j += (long long)gridDim.x * blockDim.x) {
        const int       s    = find_set(off, S, j);
        const long long o    = off[s];
        const long long n    = off[s + 1] - o;
        const long long src  = perm[j];
        const long long leaf = node_off[s] + (n - 1) + (j - o);
        const T         a = x[src], b = y[src], c = z[src];
        mnx[leaf] = a;
        mxx[leaf] = a;
        mny[leaf] = b;
        mxy[leaf] = b;
        mnz[leaf] = c;
        mxz[leaf] = c;
        id_out[leaf]    = id ? id[src] : (uint32_t)(src - o);
        ghost_out[leaf] = ghost ? ghost[src] : (int8_t)0;
        orig_out[leaf]  = (int32_t)(src - o);
        unsigned long long hi, lo;
        encode_point<T, SFC>(a, b, c, Coord<T>::is_float ? par + 6 * (size_t)s : nullptr, s_rot, s_sub, hi, lo);
        klo[j] = lo;
    }
}

// =========================================================================================
// 6. topology: global internal index g -> set s (rec_off), node g - rec_off[s] of that set
// =========================================================================================
template <int KIND>
__global__ void __launch_bounds__(256)
    batch_karras_kernel(const long long *__restrict__ off, const long long *__restrict__ node_off,
                        const long long *__restrict__ rec_off, int S, long long N,
                        const unsigned long long *__restrict__ klo, int32_t *left, int32_t *right, int32_t *parent,
                        int32_t *leaves) {
    const long long total = rec_off[S];
    for (long long g = blockIdx.x * (long long)blockDim.x + threadIdx.x; g < N && g < total;
         g += (long long)gridDim.x * blockDim.x) {
        const int       s  = find_set(rec_off, S, g);
        const long long ro = rec_off[s];
        const int       n  = (int)(off[s + 1] - off[s]);
        karras_node<KIND>(klo + off[s], nullptr, n, (int)(g - ro), left + ro, right + ro, parent + node_off[s],
                          leaves + ro);
    }
}

// =========================================================================================
// 7. refit of every set with >= 2 leaves (climbs from its leaves), then the root height of
//    each set
// =========================================================================================
// The same refit with every lane kept busy (as refit_stream_kernel for one tree): warps take
// leaves in chunks from a device counter (*work, zero at launch) and a lane whose climb ended
// takes the next leaf, finding its set by binary search over the offsets.
template <class T>
__global__ void __launch_bounds__(256)
    batch_refit_stream_kernel(const long long *__restrict__ off, const long long *__restrict__ node_off,
                              const long long *__restrict__ rec_off, int S, long long N,
                              const int32_t *__restrict__ left, const int32_t *__restrict__ right,
                              const int32_t *__restrict__ parent, T *mnx, T *mxx, T *mny, T *mxy, T *mnz, T *mxz,
                              NodeRec<T> *recs, uint8_t *height, int32_t *counters,
                              const int32_t *__restrict__ leaves, int32_t *work) {
    const unsigned FULL   = 0xffffffffu;
    const int      lane   = threadIdx.x & 31;
    constexpr int  kChunk = 256;
    const int      total  = (int)N; // at most 2^30 (batch_create)
    int            next = 0, end = 0;
    bool           more = true;
    int            curr = -1, steps = 0, n = 0;
    long long      no = 0, ro = 0;
    for (;;) {
        unsigned idle = __ballot_sync(FULL, curr < 0);
        while (idle && more) {
            if (next >= end) {
                int b = 0;
                if (lane == 0) b = atomicAdd(work, kChunk);
                b = __shfl_sync(FULL, b, 0);
                if (b >= total) {
                    more = false;
                    break;
                }
                next = b;
                end  = min(b + kChunk, total);
            }
            const int take = min(__popc(idle), end - next);
            const int rank = __popc(idle & ((1u << lane) - 1u));
            if (curr < 0 && rank < take) {
                const long long g = next + rank;
                const int       s = find_set(off, S, g);
                n                 = (int)(off[s + 1] - off[s]);
                no                = node_off[s];
                ro                = rec_off[s];
                curr              = n >= 2 ? (int)(g - off[s]) + n - 1 : -1; // one-leaf sets have no refit
                steps             = 0;
            }
            next += take;
            idle = __ballot_sync(FULL, curr < 0);
        }
        if (!__any_sync(FULL, curr >= 0)) break;
        if (curr >= 0) {
            T *const soa[6] = {mnx + no, mxx + no, mny + no, mxy + no, mnz + no, mxz + no};
            curr = ++steps < n ? refit_step<T>(curr, n, left + ro, right + ro, parent + no, soa, recs + ro,
                                               height + ro, counters + ro, leaves + ro)
                               : -1;
        }
    }
}

template <class T>
__global__ void __launch_bounds__(256)
    batch_collapse_kernel(const long long *__restrict__ off, const long long *__restrict__ node_off,
                          const long long *__restrict__ rec_off, int S, long long N, const int32_t *__restrict__ left,
                          const int32_t *__restrict__ right, const T *mnx, const T *mxx, const T *mny, const T *mxy,
                          const T *mnz, const T *mxz, WideRec<T> *wide) {
    const long long total = rec_off[S];
    for (long long g = blockIdx.x * (long long)blockDim.x + threadIdx.x; g < N && g < total;
         g += (long long)gridDim.x * blockDim.x) {
        const int       s  = find_set(rec_off, S, g);
        const long long ro = rec_off[s], no = node_off[s];
        const int       n  = (int)(off[s + 1] - off[s]);
        const T *const  soa[6] = {mnx + no, mxx + no, mny + no, mxy + no, mnz + no, mxz + no};
        collapse_node<T>((int)(g - ro), n, left + ro, right + ro, soa, wide + ro);
    }
}

__global__ void batch_heights_kernel(const long long *__restrict__ off, const long long *__restrict__ rec_off, int S,
                                     const uint8_t *__restrict__ height, uint8_t *set_height) {
    for (int s = blockIdx.x * blockDim.x + threadIdx.x; s < S; s += gridDim.x * blockDim.x)
        set_height[s] = (off[s + 1] - off[s] >= 2) ? height[rec_off[s]] : (uint8_t)0;
}

// Build order of the persistent launch: sets by decreasing size class (floor(log2 n)), so the
// longest builds start first.  One block; the order inside a class is whatever the atomics
// give (it schedules work and changes no result).
__global__ void __launch_bounds__(1024) batch_order_kernel(const long long *__restrict__ off, int S, int32_t *order) {
    __shared__ uint32_t s_cnt[64];
    for (int i = threadIdx.x; i < 64; i += blockDim.x) s_cnt[i] = 0;
    __syncthreads();
    auto cls = [&](int s) {
        const long long n = off[s + 1] - off[s];
        return n > 0 ? 64 - __clzll((unsigned long long)n) : 0;
    };
    for (int s = threadIdx.x; s < S; s += blockDim.x) atomicAdd(&s_cnt[cls(s)], 1u);
    __syncthreads();
    if (threadIdx.x == 0) {
        uint32_t run = 0;
        for (int c = 63; c >= 0; --c) {
            const uint32_t v = s_cnt[c];
            s_cnt[c]         = run;
            run += v;
        }
    }
    __syncthreads();
    for (int s = threadIdx.x; s < S; s += blockDim.x) order[atomicAdd(&s_cnt[cls(s)], 1u)] = s;
}

// =========================================================================================
// Host side
// =========================================================================================
struct GraphKey {
    const void *in_off = nullptr, *x = nullptr, *y = nullptr, *z = nullptr, *id = nullptr, *ghost = nullptr;
    void       *idx = nullptr, *dist = nullptr;
    size_t      S = 0, N = 0;
    int         k = 0, excl = 0, method = 0, half = 0, variant = 0;
    const void *model     = nullptr; // learned bound (its weights are read when the graph runs)
    float       inflation = 0.0f;
    bool operator==(const GraphKey &o) const {
        return in_off == o.in_off && x == o.x && y == o.y && z == o.z && id == o.id && ghost == o.ghost &&
               idx == o.idx && dist == o.dist && S == o.S && N == o.N && k == o.k && excl == o.excl &&
               method == o.method && half == o.half && variant == o.variant && model == o.model &&
               inflation == o.inflation;
    }
};

struct BatchImpl {
    size_t    max_points = 0, max_sets = 0;
    ft_tree   all{};  // concatenated node arrays of every set
    TreeImpl  scr{};  // records, heights, refit counters and sort scratch of the whole batch
    long long *off = nullptr, *node_off = nullptr, *rec_off = nullptr; // max_sets + 1 each
    uint8_t   *set_height = nullptr;
    void      *bmin = nullptr, *bmax = nullptr; // ordered-integer boxes, 3 words per set each
    void      *bbox = nullptr, *par = nullptr;  // 6 coordinates per set each
    int32_t   *rr = nullptr, *rw = nullptr;     // replay list of the fast walk
    int32_t   *mw = nullptr;                    // rows whose learned bound proved too small
    int32_t   *order = nullptr, *ready = nullptr, *chunk_next = nullptr; // persistent launch: max_sets each
    uint32_t  *ctl = nullptr;                   // persistent launch: build tickets, ready slots, cursor
    uint32_t  *counters = nullptr;              // [0] replay count, [2..3] visits, [4] bound misses
    float     *feats = nullptr;                 // learned bound: features and bounds of every leaf,
    void      *bound = nullptr;                 // allocated by the first learned query
    size_t     learned_cap = 0;
    size_t     S = 0, N = 0;
    bool       built = false;
    std::vector<std::unique_ptr<TreeImpl>> views;
    cudaStream_t    cap_stream = nullptr;
    cudaGraphExec_t exec       = nullptr;
    GraphKey        key{};
    bool            per_set_build = false; // ft_batch_build through the persistent launch's per-set builds
};

template <class T> static T *dalloc(size_t count) {
    void *p = nullptr;
    if (count == 0) count = 1;
    cudaError_t e = cudaMalloc(&p, count * sizeof(T));
    if (e != cudaSuccess) {
        cudaGetLastError();
        fail(FT_ERR_OUT_OF_MEMORY, "cudaMalloc of batch storage failed");
    }
    return (T *)p;
}

void batch_free(BatchImpl *b) {
    if (!b) return;
    if (b->exec) cudaGraphExecDestroy(b->exec);
    if (b->cap_stream) cudaStreamDestroy(b->cap_stream);
    void *ptrs[] = {b->all.min_x, b->all.max_x, b->all.min_y,  b->all.max_y,    b->all.min_z,  b->all.max_z,
                    b->all.left_child, b->all.right_child, b->all.parent, b->all.id, b->all.is_ghost,
                    b->all.orig_idx, b->off, b->node_off, b->rec_off, b->set_height, b->bmin, b->bmax, b->bbox,
                    b->par, b->rr, b->rw, b->mw, b->counters, b->feats, b->bound, b->order, b->ready,
                    b->chunk_next, b->ctl};
    for (void *p : ptrs)
        if (p) cudaFree(p);
    free_scratch(b->scr);
    delete b;
}

BatchImpl *batch_create(Context &ctx, size_t max_points, size_t max_sets) {
    const ft_options &o = ctx.opts;
    if (max_sets < 1 || max_sets > (size_t(1) << 24)) fail(FT_ERR_INVALID_ARGUMENT, "max_sets must be in [1, 2^24]");
    if (max_points > (size_t(1) << 30)) fail(FT_ERR_INVALID_ARGUMENT, "max_points must be at most 2^30");
    std::unique_ptr<BatchImpl, void (*)(BatchImpl *)> b(new BatchImpl(), batch_free);
    b->max_points = max_points;
    b->max_sets   = max_sets;
    const size_t cb = coord_bytes(o.coord_type), P = std::max<size_t>(max_points, 1), nodes = 2 * P;
    ft_tree     &t  = b->all;
    t.min_x = dalloc<unsigned char>(nodes * cb);
    t.max_x = dalloc<unsigned char>(nodes * cb);
    t.min_y = dalloc<unsigned char>(nodes * cb);
    t.max_y = dalloc<unsigned char>(nodes * cb);
    t.min_z = dalloc<unsigned char>(nodes * cb);
    t.max_z = dalloc<unsigned char>(nodes * cb);
    t.left_child  = dalloc<int32_t>(P);
    t.right_child = dalloc<int32_t>(P);
    t.parent      = dalloc<int32_t>(nodes);
    t.id          = dalloc<uint32_t>(nodes);
    t.is_ghost    = dalloc<int8_t>(nodes);
    t.orig_idx    = dalloc<int32_t>(nodes);
    t.capacity    = 0;
    t.impl        = &b->scr;
    TreeImpl &s   = b->scr;
    s.coord       = o.coord_type;
    s.cap         = P;
    s.recs        = dalloc<unsigned char>(P * 16 * cb);
    s.height      = dalloc<uint8_t>(P);
    s.counters    = dalloc<int32_t>(P);
    s.leafcount   = dalloc<int32_t>(P);
    s.wide        = dalloc<unsigned char>(P * wide_bytes(o.coord_type));
    s.key_lo      = (uint64_t *)dalloc<unsigned long long>(P);
    s.tmp_lo      = (uint64_t *)dalloc<unsigned long long>(P);
    if (o.coord_type == U64) { // 126-bit keys (built by the persistent launch only)
        s.key_hi = (uint64_t *)dalloc<unsigned long long>(P);
        s.tmp_hi = (uint64_t *)dalloc<unsigned long long>(P);
    }
    s.perm        = dalloc<uint32_t>(P);
    s.tmp_perm    = dalloc<uint32_t>(P);
    s.hist        = dalloc<uint32_t>(16 * 256 + 16);
    s.lookback_words = sort_lookback_words(P, 1);
    s.lookback       = dalloc<uint32_t>(s.lookback_words);
    s.tile_counter   = dalloc<uint32_t>(16);
    s.status         = dalloc<uint32_t>(4);
    FT_CUDA(cudaMemset(s.status, 0, 16));
    s.height_root = -1;
    s.clean42     = false;
    b->off        = dalloc<long long>(max_sets + 1);
    b->node_off   = dalloc<long long>(max_sets + 1);
    b->rec_off    = dalloc<long long>(max_sets + 1);
    b->set_height = dalloc<uint8_t>(max_sets);
    b->bmin       = dalloc<unsigned long long>(3 * max_sets);
    b->bmax       = dalloc<unsigned long long>(3 * max_sets);
    b->bbox       = dalloc<unsigned long long>(6 * max_sets);
    b->par        = dalloc<unsigned long long>(6 * max_sets);
    b->rr         = dalloc<int32_t>(P);
    b->rw         = dalloc<int32_t>(P);
    b->mw         = dalloc<int32_t>(P);
    b->counters   = dalloc<uint32_t>(8);
    b->order      = dalloc<int32_t>(max_sets);
    b->ready      = dalloc<int32_t>(max_sets);
    b->chunk_next = dalloc<int32_t>(max_sets);
    b->ctl        = dalloc<uint32_t>(4);
    FT_CUDA(cudaMemset(b->counters, 0, 32));
    return b.release();
}

static int grid_of(size_t n, int threads, int max_blocks) {
    size_t g = (n + threads - 1) / threads;
    return (int)std::max<size_t>(1, std::min<size_t>(g, (size_t)max_blocks));
}

static BatchDev batch_dev(const BatchImpl &b) {
    BatchDev d;
    d.off      = b.off;
    d.node_off = b.node_off;
    d.rec_off  = b.rec_off;
    d.height   = b.set_height;
    d.S        = (int)b.S;
    return d;
}

template <class T>
static void batch_build_typed(Context &ctx, BatchImpl &b, const long long *in_off, const T *x, const T *y,
                              const T *z, const uint32_t *id, const int8_t *ghost, cudaStream_t st) {
    const ft_options &o  = ctx.opts;
    TreeImpl         &s  = b.scr;
    ft_tree          &t  = b.all;
    const int         S  = (int)b.S;
    const long long   N  = (long long)b.N;
    const int         sm = ctx.num_sms;
    using O              = typename Ord<T>::type;
    T *par               = (T *)b.par;

    batch_prep_kernel<<<1, kPrepThreads, 0, st>>>(in_off, S, N, b.off, b.node_off, b.rec_off, ctx.status);
    FT_CUDA(cudaGetLastError());
    if (N == 0) {
        FT_CUDA(cudaMemsetAsync(b.set_height, 0, (size_t)S, st));
        return;
    }
    {
        FT_CUDA(cudaMemsetAsync(b.bmin, 0xFF, 3 * (size_t)S * sizeof(O), st));
        FT_CUDA(cudaMemsetAsync(b.bmax, 0x00, 3 * (size_t)S * sizeof(O), st));
        batch_bbox_kernel<T><<<grid_of((size_t)N, kChunk, sm * 8), kBboxThreads, 0, st>>>(b.off, S, N, x, y, z,
                                                                                          (O *)b.bmin, (O *)b.bmax);
        batch_params_kernel<T><<<grid_of((size_t)S, 256, sm * 4), 256, 0, st>>>(S, (const O *)b.bmin,
                                                                                (const O *)b.bmax, (T *)b.bbox, par);
        FT_CUDA(cudaGetLastError());
    }
    const int gN = grid_of((size_t)N, 256, sm * 16);
    if (o.sfc_type == MORTON)
        batch_encode_kernel<T, MORTON><<<gN, 256, 0, st>>>(b.off, S, N, x, y, z, par,
                                                           (unsigned long long *)s.key_lo, s.perm);
    else
        batch_encode_kernel<T, PEANO_HILBERT><<<gN, 256, 0, st>>>(b.off, S, N, x, y, z, par,
                                                                  (unsigned long long *)s.key_lo, s.perm);
    FT_CUDA(cudaGetLastError());
    // (key, index) then set: 8 key digits, then the set id's digits
    static const int key_digits[8] = {0, 1, 2, 3, 4, 5, 6, 7};
    sort_pairs_fixed(s, (size_t)N, 1, 8, key_digits, st);
    if (S > 1) {
        batch_set_key_kernel<<<gN, 256, 0, st>>>(b.off, S, N, s.perm, (unsigned long long *)s.key_lo);
        FT_CUDA(cudaGetLastError());
        const int nd = (S - 1) < 256 ? 1 : (S - 1) < 65536 ? 2 : 3;
        sort_pairs_fixed(s, (size_t)N, 1, nd, key_digits, st);
    }
    // leaves; internal slots of parent = -1 and id / is_ghost / orig_idx = 0
    const size_t nodes = 2 * (size_t)N;
    FT_CUDA(cudaMemsetAsync(t.parent, 0xFF, nodes * sizeof(int32_t), st));
    FT_CUDA(cudaMemsetAsync(t.id, 0, nodes * sizeof(uint32_t), st));
    FT_CUDA(cudaMemsetAsync(t.is_ghost, 0, nodes, st));
    FT_CUDA(cudaMemsetAsync(t.orig_idx, 0, nodes * sizeof(int32_t), st));
    T *mnx = (T *)t.min_x, *mxx = (T *)t.max_x, *mny = (T *)t.min_y, *mxy = (T *)t.max_y, *mnz = (T *)t.min_z,
      *mxz = (T *)t.max_z;
    if (o.sfc_type == MORTON)
        batch_gather_kernel<T, MORTON><<<gN, 256, 0, st>>>(b.off, b.node_off, S, N, x, y, z, par, s.perm, id, ghost,
                                                           mnx, mxx, mny, mxy, mnz, mxz, t.id, t.is_ghost, t.orig_idx,
                                                           (unsigned long long *)s.key_lo);
    else
        batch_gather_kernel<T, PEANO_HILBERT><<<gN, 256, 0, st>>>(b.off, b.node_off, S, N, x, y, z, par, s.perm, id,
                                                                  ghost, mnx, mxx, mny, mxy, mnz, mxz, t.id,
                                                                  t.is_ghost, t.orig_idx,
                                                                  (unsigned long long *)s.key_lo);
    FT_CUDA(cudaGetLastError());
    const int gK = grid_of((size_t)N, 256, sm * 32);
    if (o.sfc_type == MORTON)
        batch_karras_kernel<0><<<gK, 256, 0, st>>>(b.off, b.node_off, b.rec_off, S, N,
                                                   (const unsigned long long *)s.key_lo, t.left_child, t.right_child,
                                                   t.parent, s.leafcount);
    else
        batch_karras_kernel<1><<<gK, 256, 0, st>>>(b.off, b.node_off, b.rec_off, S, N,
                                                   (const unsigned long long *)s.key_lo, t.left_child, t.right_child,
                                                   t.parent, s.leafcount);
    FT_CUDA(cudaGetLastError());
    // arrival counters of the sets' internal nodes (at most N - 1 of them), and in the last
    // slot the streaming refit's leaf counter
    FT_CUDA(cudaMemsetAsync(s.counters, 0, (size_t)N * sizeof(int32_t), st));
    batch_refit_stream_kernel<T><<<grid_of((size_t)N, 256, sm * 8), 256, 0, st>>>(
        b.off, b.node_off, b.rec_off, S, N, t.left_child, t.right_child, t.parent, mnx, mxx, mny, mxy, mnz, mxz,
        (NodeRec<T> *)s.recs, s.height, s.counters, s.leafcount, s.counters + (N - 1));
    batch_collapse_kernel<T><<<gK, 256, 0, st>>>(b.off, b.node_off, b.rec_off, S, N, t.left_child, t.right_child,
                                                 mnx, mxx, mny, mxy, mnz, mxz, (WideRec<T> *)s.wide);
    batch_heights_kernel<<<grid_of((size_t)S, 256, sm * 4), 256, 0, st>>>(b.off, b.rec_off, S, s.height,
                                                                          b.set_height);
    FT_CUDA(cudaGetLastError());
}

// The persistent launch (batch_persistent): offsets prepared, the scheduling words reset, the
// build order computed, then one kernel builds every set and, with `query`, answers its
// self-kNN rows (tied rows replayed by a second launch).  No host synchronisation and no
// allocation, so it is captured in the build + query graph like the launch sequence.
struct PersistQuery {
    int       k    = 0;
    bool      excl = true;
    uint64_t *idx  = nullptr;
    void     *dist = nullptr;
};
static void batch_build_persistent(Context &ctx, BatchImpl &b, const long long *in_off, size_t S, size_t N,
                                   const void *x, const void *y, const void *z, const uint32_t *id,
                                   const int8_t *ghost, const PersistQuery *q, cudaStream_t st) {
    if (S < 1 || S > b.max_sets) fail(FT_ERR_INVALID_ARGUMENT, "num_sets must be in [1, max_sets]");
    if (N > b.max_points) fail(FT_ERR_INVALID_ARGUMENT, "num_points exceeds the batch's max_points");
    b.S                = S;
    b.N                = N;
    b.built            = true;
    b.all.num_leaves   = N;
    b.all.num_internal = N;
    batch_prep_kernel<<<1, kPrepThreads, 0, st>>>(in_off, (int)S, (long long)N, b.off, b.node_off, b.rec_off,
                                                  ctx.status);
    FT_CUDA(cudaGetLastError());
    FT_CUDA(cudaMemsetAsync(b.ctl, 0, 4 * sizeof(uint32_t), st));
    FT_CUDA(cudaMemsetAsync(b.ready, 0xFF, S * sizeof(int32_t), st));
    FT_CUDA(cudaMemsetAsync(b.chunk_next, 0, S * sizeof(int32_t), st));
    if (q) FT_CUDA(cudaMemsetAsync(b.counters, 0, 8 * sizeof(uint32_t), st));
    batch_order_kernel<<<1, 1024, 0, st>>>(b.off, (int)S, b.order);
    FT_CUDA(cudaGetLastError());
    PersistLaunch p;
    p.off = b.off; p.node_off = b.node_off; p.rec_off = b.rec_off; p.S = (int)S;
    p.x = x; p.y = y; p.z = z; p.id = id; p.ghost = ghost;
    p.all = b.all; p.scr = &b.scr; p.bbox = b.bbox; p.set_height = b.set_height;
    p.order = b.order; p.ready = b.ready; p.chunk_next = b.chunk_next; p.ctl = b.ctl;
    p.query = q != nullptr && N > 0;
    if (p.query) {
        p.k = q->k; p.excl = q->excl; p.idx = q->idx; p.dist = q->dist;
        p.rr = b.rr; p.rw = b.rw; p.counters = b.counters;
    }
    batch_persistent(ctx, p, st);
    if (p.query)
        replay_exact(ctx, b.all, b.rr, b.rw, b.counters, q->k, q->excl, q->idx, q->dist, st, batch_dev(b));
}

void batch_build(Context &ctx, BatchImpl &b, const long long *in_off, size_t S, size_t N, const void *x,
                 const void *y, const void *z, const uint32_t *id, const int8_t *ghost, cudaStream_t st) {
    if (ctx.opts.coord_type == U64 || b.per_set_build) { // (126-bit keys: always) the per-set builds
        batch_build_persistent(ctx, b, in_off, S, N, x, y, z, id, ghost, nullptr, st);
        return;
    }
    if (S < 1 || S > b.max_sets) fail(FT_ERR_INVALID_ARGUMENT, "num_sets must be in [1, max_sets]");
    if (N > b.max_points) fail(FT_ERR_INVALID_ARGUMENT, "num_points exceeds the batch's max_points");
    b.S     = S;
    b.N     = N;
    b.built = true;
    b.all.num_leaves   = N;
    b.all.num_internal = N;
    switch (ctx.opts.coord_type) {
    case F32: batch_build_typed<float>(ctx, b, in_off, (const float *)x, (const float *)y, (const float *)z, id, ghost, st); break;
    case F64: batch_build_typed<double>(ctx, b, in_off, (const double *)x, (const double *)y, (const double *)z, id, ghost, st); break;
    case U32: batch_build_typed<uint32_t>(ctx, b, in_off, (const uint32_t *)x, (const uint32_t *)y, (const uint32_t *)z, id, ghost, st); break;
    default: fail(FT_ERR_INVALID_ARGUMENT, "unsupported coordinate type for batched sets");
    }
}

// Feature and bound scratch of the learned batched query (every leaf of the batch's capacity);
// the first learned query allocates it, later ones reuse it.
static void ensure_batch_learned(BatchImpl &b) {
    if (b.feats) return;
    const size_t P = std::max<size_t>(b.max_points, 1);
    b.feats        = dalloc<float>(P * FT_BOUND_FEATURES);
    b.bound        = dalloc<unsigned long long>(P);
    b.learned_cap  = P;
}

// model: null, or the learned radius bound (features -> prediction x inflation -> the walk's
// per-query bound; queries whose bound proves too small rerun the walk without it).
static void check_query_args(int k, const ft_query_options &q) {
    const int max_k = q.max_k > 0 ? q.max_k : 32;
    if (k > max_k)
        fail(FT_ERR_INVALID_ARGUMENT,
             "k exceeds _MAX_K_ template parameter. Instantiate self_knn_query with larger _MAX_K_.");
    if (k > 512) fail(FT_ERR_RUNTIME, "self_knn_query: k too large for shared memory.");
}

void batch_query(Context &ctx, BatchImpl &b, int k, bool excl, uint64_t *idx, void *dist, const ft_query_options &q,
                 cudaStream_t st, BoundModel *model, float inflation) {
    if (!b.built) fail(FT_ERR_INVALID_ARGUMENT, "the batch has not been built");
    check_query_args(k, q);
    if (model && k > 64) fail(FT_ERR_INVALID_ARGUMENT, "learned bound: k must be in [1, 64]");
    if (b.N == 0 || k <= 0) return;
    const void *bound = nullptr;
    if (model) {
        if (!b.feats) fail(FT_ERR_RUNTIME, "the batch's learned-bound scratch is missing");
        bound_features_batch(ctx, b.all, batch_dev(b), b.N, k, b.feats, st);
        bound_model_predict(ctx, *model, b.feats, b.N, inflation, nullptr, b.bound, st);
        bound = b.bound;
    }
    batch_self_knn(ctx, b.all, batch_dev(b), b.N, k, excl, idx, dist, q.method != FT_METHOD_PLAIN || model,
                   q.reserved[0], q.reserved[1], b.rr, b.rw, b.counters, st, bound, b.mw);
}

void batch_features(Context &ctx, BatchImpl &b, int k, float *out, cudaStream_t st) {
    if (!b.built) fail(FT_ERR_INVALID_ARGUMENT, "the batch has not been built");
    bound_features_batch(ctx, b.all, batch_dev(b), b.N, k, out, st);
}

void batch_query_learned(Context &ctx, BatchImpl &b, BoundModel &model, int k, bool excl, float inflation,
                         uint64_t *idx, void *dist, const ft_query_options &q, cudaStream_t st) {
    ensure_batch_learned(b);
    batch_query(ctx, b, k, excl, idx, dist, q, st, &model, inflation);
}

// Build + query as one CUDA graph: captured on the first call with these arguments (on the
// batch's own stream, in relaxed mode), then replayed on `st`.
void batch_build_query_graph(Context &ctx, BatchImpl &b, const long long *in_off, size_t S, size_t N, const void *x,
                             const void *y, const void *z, const uint32_t *id, const int8_t *ghost, int k, bool excl,
                             uint64_t *idx, void *dist, const ft_query_options &q, cudaStream_t st, BoundModel *model,
                             float inflation) {
    if (model) ensure_batch_learned(b); // before any capture: the captured graph allocates nothing
    GraphKey key;
    key.in_off = in_off; key.x = x; key.y = y; key.z = z; key.id = id; key.ghost = ghost;
    key.idx = idx; key.dist = dist; key.S = S; key.N = N; key.k = k; key.excl = excl ? 1 : 0;
    key.method = q.method; key.half = q.reserved[0]; key.variant = q.reserved[1];
    key.model = model; key.inflation = inflation;
    if (!(b.exec && key == b.key)) {
        if (b.exec) {
            FT_CUDA(cudaGraphExecDestroy(b.exec));
            b.exec = nullptr;
        }
        if (!b.cap_stream) FT_CUDA(cudaStreamCreateWithFlags(&b.cap_stream, cudaStreamNonBlocking));
        // argument errors are raised before the capture starts
        if (S < 1 || S > b.max_sets) fail(FT_ERR_INVALID_ARGUMENT, "num_sets must be in [1, max_sets]");
        if (N > b.max_points) fail(FT_ERR_INVALID_ARGUMENT, "num_points exceeds the batch's max_points");
        FT_CUDA(cudaStreamBeginCapture(b.cap_stream, cudaStreamCaptureModeRelaxed));
        cudaGraph_t graph = nullptr;
        try {
            // the persistent launch is the default for the fast walk's k (measured faster than
            // the launch sequence on the 4096-set workload); FT_METHOD_FAST names the sequence
            const bool persistent = q.method == FT_METHOD_PERSISTENT || q.method == FT_METHOD_DEFAULT;
            if (persistent && !model && k >= 1 && k <= 64) {
                check_query_args(k, q);
                PersistQuery pq;
                pq.k    = k;
                pq.excl = excl;
                pq.idx  = idx;
                pq.dist = dist;
                batch_build_persistent(ctx, b, in_off, S, N, x, y, z, id, ghost, &pq, b.cap_stream);
            } else {
                if (q.method == FT_METHOD_PERSISTENT)
                    batch_build_persistent(ctx, b, in_off, S, N, x, y, z, id, ghost, nullptr, b.cap_stream);
                else batch_build(ctx, b, in_off, S, N, x, y, z, id, ghost, b.cap_stream);
                batch_query(ctx, b, k, excl, idx, dist, q, b.cap_stream, model, inflation);
            }
        } catch (...) {
            cudaStreamEndCapture(b.cap_stream, &graph);
            if (graph) cudaGraphDestroy(graph);
            cudaGetLastError();
            throw;
        }
        FT_CUDA(cudaStreamEndCapture(b.cap_stream, &graph));
        cudaError_t e = cudaGraphInstantiate(&b.exec, graph, 0);
        cudaGraphDestroy(graph);
        FT_CUDA(e);
        b.key = key;
    }
    b.S     = S;
    b.N     = N;
    b.built = true;
    FT_CUDA(cudaGraphLaunch(b.exec, st));
}

// View of set s as a single tree (pointers into the batch).  Reads the set's offsets and
// height back (blocking).
void batch_tree_view(Context &ctx, BatchImpl &b, size_t s, ft_tree &out, cudaStream_t st) {
    if (!b.built) fail(FT_ERR_INVALID_ARGUMENT, "the batch has not been built");
    if (s >= b.S) fail(FT_ERR_INVALID_ARGUMENT, "set index out of range");
    long long o[2], no, ro;
    uint8_t   h = 0;
    FT_CUDA(cudaMemcpyAsync(o, b.off + s, 2 * sizeof(long long), cudaMemcpyDeviceToHost, st));
    FT_CUDA(cudaMemcpyAsync(&no, b.node_off + s, sizeof(long long), cudaMemcpyDeviceToHost, st));
    FT_CUDA(cudaMemcpyAsync(&ro, b.rec_off + s, sizeof(long long), cudaMemcpyDeviceToHost, st));
    FT_CUDA(cudaMemcpyAsync(&h, b.set_height + s, 1, cudaMemcpyDeviceToHost, st));
    FT_CUDA(cudaStreamSynchronize(st));
    if (b.views.size() < b.max_sets) b.views.resize(b.max_sets);
    if (!b.views[s]) b.views[s].reset(new TreeImpl());
    TreeImpl     &v  = *b.views[s];
    const size_t  cb = coord_bytes(ctx.opts.coord_type);
    const size_t  n  = (size_t)(o[1] - o[0]);
    v                = TreeImpl{};
    v.coord          = ctx.opts.coord_type;
    v.view           = true;
    v.recs           = (unsigned char *)b.scr.recs + (size_t)ro * 16 * cb;
    v.height         = b.scr.height + ro;
    v.leafcount      = b.scr.leafcount + ro;
    v.wide           = (unsigned char *)b.scr.wide + (size_t)ro * wide_bytes(ctx.opts.coord_type);
    v.height_root    = n >= 2 ? (int)h : 0;
    v.clean42        = false;
    std::memset(&out, 0, sizeof(out));
    const ft_tree &a = b.all;
    out.min_x        = (unsigned char *)a.min_x + no * cb;
    out.max_x        = (unsigned char *)a.max_x + no * cb;
    out.min_y        = (unsigned char *)a.min_y + no * cb;
    out.max_y        = (unsigned char *)a.max_y + no * cb;
    out.min_z        = (unsigned char *)a.min_z + no * cb;
    out.max_z        = (unsigned char *)a.max_z + no * cb;
    out.left_child   = a.left_child + ro;
    out.right_child  = a.right_child + ro;
    out.parent       = a.parent + no;
    out.id           = a.id + no;
    out.is_ghost     = a.is_ghost + no;
    out.orig_idx     = a.orig_idx + no;
    out.num_leaves   = n;
    out.num_internal = n > 0 ? n - 1 : 0;
    out.capacity     = 0;
    out.impl         = &v;
    // periodic integer sets with a coordinate at or above the period keep the reference
    // traversal (the same test the batched fast walk makes per set)
    if (n > 0 && ctx.opts.periodic && (ctx.opts.coord_type == U32 || ctx.opts.coord_type == U64)) {
        unsigned long long m[3] = {0, 0, 0};
        const void        *src[3] = {out.max_x, out.max_y, out.max_z};
        for (int a = 0; a < 3; ++a) FT_CUDA(cudaMemcpyAsync(&m[a], src[a], cb, cudaMemcpyDeviceToHost, st));
        FT_CUDA(cudaStreamSynchronize(st));
        const unsigned long long P = ctx.opts.coord_type == U64 ? (1ull << 42) : (1ull << 21);
        v.in_period                = m[0] < P && m[1] < P && m[2] < P;
    }
}

// Per-set boxes and root heights, for inspection (blocking).
void batch_set_info(Context &ctx, BatchImpl &b, void *bbox_out, uint8_t *height_out, cudaStream_t st) {
    if (!b.built) fail(FT_ERR_INVALID_ARGUMENT, "the batch has not been built");
    const size_t cb = coord_bytes(ctx.opts.coord_type);
    if (bbox_out) FT_CUDA(cudaMemcpyAsync(bbox_out, b.bbox, 6 * b.S * cb, cudaMemcpyDeviceToHost, st));
    if (height_out) FT_CUDA(cudaMemcpyAsync(height_out, b.set_height, b.S, cudaMemcpyDeviceToHost, st));
    FT_CUDA(cudaStreamSynchronize(st));
}

void batch_tune(Context &ctx, BatchImpl &b, int k, bool excl, ft_tune_result *out, cudaStream_t st) {
    if (!b.built) fail(FT_ERR_INVALID_ARGUMENT, "the batch has not been built");
    tune_batch_self_knn(ctx, b.all, batch_dev(b), b.N, k, excl, b.rr, b.rw, b.counters, out, st);
}

void batch_set_build_method(BatchImpl &b, int method) { b.per_set_build = method == FT_METHOD_PERSISTENT; }

void batch_stats(BatchImpl &b, ft_query_stats &out) {
    uint32_t w[8] = {0, 0, 0, 0, 0, 0, 0, 0};
    FT_CUDA(cudaMemcpy(w, b.counters, sizeof(w), cudaMemcpyDeviceToHost));
    out.queries  = (int64_t)b.N;
    out.replayed = w[0];
    unsigned long long v, v2;
    std::memcpy(&v, &w[2], sizeof(v));
    std::memcpy(&v2, &w[6], sizeof(v2));
    out.reserved[0] = (int64_t)(v + v2);
    out.reserved[1] = (int64_t)w[4];
    out.reserved[2] = (int64_t)v2;
}

} // namespace ft
