// ft_tune.cu -- per-shape autotuner of the build's sort tile and of the fast walk's launch.
//
// The reference picks one kernel shape per device: the sub-group width W from
// get_native_sub_group_width and the dispatchers of src/hlbvh.hpp:1828-1927 (MAXK <= 32 ->
// register heap, else the local-memory heap).  Here every choice gives the same rows bit for
// bit, so the choice is free to follow speed: the tuner times each candidate on the caller's
// own data and keeps the fastest for the shape, keyed by (kind, k, floor(log2 n)) in the
// context.  Later calls with default options take the kept choice.
//  * build: keys per thread of a onesweep tile (8 / 12 / 16 / 20 for one-word keys, 8 / 12 /
//    16 for two-word keys), timed over whole builds of the caller's points;
//  * self-kNN (single tree and batched sets): the walk variant (4-wide per-lane walk, compact
//    binary walk, group walk), the SFC seeding half-window (k/2, k, 2k) and the block shape
//    (two-warp blocks with 32-entry heaps, or one-warp blocks), timed on up to 2^18 queries
//    (four stretches of consecutive leaves, the order the walk takes them in) or, for a batch,
//    on the whole batch.
// Every candidate's rows are compared with the default's on the device; a difference is an
// error (it would be a bug in one of the walks), not a choice.
#include <cuda_runtime.h>

#include <algorithm>
#include <string>
#include <vector>

#include "ft_common.cuh"
#include "ft_internal.h"

namespace ft {

// Number of differing 64-bit words between a and b (n words).
__global__ void __launch_bounds__(256) count_diff_kernel(const unsigned long long *__restrict__ a,
                                                         const unsigned long long *__restrict__ b, size_t n,
                                                         unsigned long long *out) {
    unsigned long long c = 0;
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
        c += a[i] != b[i];
    for (int o = 16; o > 0; o >>= 1) c += __shfl_down_sync(0xffffffffu, c, o);
    if ((threadIdx.x & 31) == 0 && c) atomicAdd(out, c);
}

__global__ void __launch_bounds__(256) sample_ranks_kernel(int32_t *ids, int m, int n, int parts) {
    const int per = m / parts;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < m; i += gridDim.x * blockDim.x) {
        const int p     = min(i / per, parts - 1);
        const int start = (int)(((long long)(n - per) * p) / max(parts - 1, 1));
        ids[i]          = start + (i - p * per);
    }
}

namespace {

struct DevBuf {
    void *p = nullptr;
    explicit DevBuf(size_t bytes) {
        if (cudaMalloc(&p, std::max<size_t>(bytes, 16)) != cudaSuccess) {
            cudaGetLastError();
            p = nullptr;
            fail(FT_ERR_OUT_OF_MEMORY, "cudaMalloc of the autotuner's scratch failed");
        }
    }
    ~DevBuf() {
        if (p) cudaFree(p);
    }
    DevBuf(const DevBuf &)            = delete;
    DevBuf &operator=(const DevBuf &) = delete;
};

// Median of `reps` timed runs of fn on st (one untimed run first).
template <class F> float time_median(cudaStream_t st, int reps, F fn) {
    fn();
    cudaEvent_t e0, e1;
    FT_CUDA(cudaEventCreate(&e0));
    FT_CUDA(cudaEventCreate(&e1));
    std::vector<float> t;
    for (int r = 0; r < reps; ++r) {
        FT_CUDA(cudaEventRecord(e0, st));
        fn();
        FT_CUDA(cudaEventRecord(e1, st));
        FT_CUDA(cudaEventSynchronize(e1));
        float ms = 0.0f;
        FT_CUDA(cudaEventElapsedTime(&ms, e0, e1));
        t.push_back(ms);
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    std::sort(t.begin(), t.end());
    return t[t.size() / 2];
}

unsigned long long count_diff(const void *a, const void *b, size_t words, unsigned long long *scratch,
                              cudaStream_t st) {
    FT_CUDA(cudaMemsetAsync(scratch, 0, sizeof(unsigned long long), st));
    count_diff_kernel<<<(int)std::min<size_t>((words + 255) / 256, 148 * 8), 256, 0, st>>>(
        (const unsigned long long *)a, (const unsigned long long *)b, words, scratch);
    FT_CUDA(cudaGetLastError());
    unsigned long long h = 0;
    FT_CUDA(cudaMemcpyAsync(&h, scratch, sizeof(h), cudaMemcpyDeviceToHost, st));
    FT_CUDA(cudaStreamSynchronize(st));
    return h;
}

struct WalkCandidate {
    int variant, half, kc;
};

std::vector<WalkCandidate> walk_candidates(int k, bool batch) {
    const int                  kc_default = k <= 32 ? 32 : 64;
    std::vector<WalkCandidate> c;
    // the defaults first: the 4-wide walk (the compact binary walk for k <= 4), half-window k
    c.push_back({k <= 4 ? 2 : 4, k, kc_default});
    const int variants[3] = {4, 2, 5};
    const int halves[3]   = {k, std::max(1, k / 2), 2 * k};
    for (int v : variants)
        for (int h : halves) {
            if (batch && h != k) continue; // a whole batch per run: the half-window stays k
            for (int kc : {32, 64}) {
                if (kc < kc_default) continue;
                const WalkCandidate w{v, h, kc};
                bool dup = false;
                for (const auto &e : c) dup = dup || (e.variant == w.variant && e.half == w.half && e.kc == w.kc);
                if (!dup) c.push_back(w);
            }
        }
    return c;
}

void fill_result(ft_tune_result *out, const WalkCandidate &best, int items, float best_ms, float default_ms,
                 int candidates) {
    if (!out) return;
    *out               = ft_tune_result{};
    out->walk_variant  = best.variant;
    out->half_window   = best.half;
    out->block_threads = best.kc == 64 ? 32 : 64;
    out->sort_items    = items;
    out->candidates    = candidates;
    out->best_ms       = best_ms;
    out->default_ms    = default_ms;
}

} // namespace

void tune_self_knn(Context &ctx, const ft_tree &tr, int k, bool excl, ft_tune_result *out, cudaStream_t st) {
    const size_t n = tr.num_leaves;
    if (k < 1 || k > 64 || n < 2) fail(FT_ERR_INVALID_ARGUMENT, "autotuner: the fast walk needs 1 <= k <= 64 and 2+ leaves");
    const int m = (int)std::min<size_t>(n, size_t(1) << 18);
    DevBuf    ids(m * sizeof(int32_t)), ref_i(m * (size_t)k * 8), ref_d(m * (size_t)k * 8), ci(m * (size_t)k * 8),
        cd(m * (size_t)k * 8), diff(8);
    sample_ranks_kernel<<<(m + 255) / 256, 256, 0, st>>>((int32_t *)ids.p, m, (int)n, m < (1 << 18) ? 1 : 4);
    FT_CUDA(cudaGetLastError());
    const auto cand = walk_candidates(k, false);
    float      best_ms = 0.0f, default_ms = 0.0f;
    int        best = 0;
    for (size_t c = 0; c < cand.size(); ++c) {
        const WalkCandidate &w = cand[c];
        void *oi = c == 0 ? ref_i.p : ci.p, *od = c == 0 ? ref_d.p : cd.p;
        const float ms = time_median(st, 3, [&] {
            if (!fast_self_knn(ctx, tr, (const int32_t *)ids.p, (size_t)m, k, excl, (uint64_t *)oi, od, nullptr,
                               w.half, w.variant, st, w.kc))
                fail(FT_ERR_INVALID_ARGUMENT, "autotuner: the fast walk does not apply to this tree");
        });
        if (c > 0 && (count_diff(ci.p, ref_i.p, (size_t)m * k, (unsigned long long *)diff.p, st) ||
                      count_diff(cd.p, ref_d.p, (size_t)m * k, (unsigned long long *)diff.p, st)))
            fail(FT_ERR_RUNTIME, "autotuner: walk variant " + std::to_string(w.variant) + " (half-window " +
                                     std::to_string(w.half) + ") returned rows that differ from the default's");
        if (c == 0) default_ms = ms;
        if (c == 0 || ms < best_ms) {
            best_ms = ms;
            best    = (int)c;
        }
    }
    TuneChoice tc;
    tc.variant = cand[best].variant;
    tc.half    = cand[best].half;
    tc.kc      = cand[best].kc;
    ctx.tuned[tune_key(TUNE_SELF_KNN, k, n)] = tc;
    fill_result(out, cand[best], 0, best_ms, default_ms, (int)cand.size());
}

void tune_batch_self_knn(Context &ctx, const ft_tree &all, const BatchDev &bt, size_t num, int k, bool excl,
                         int32_t *rr, int32_t *rw, uint32_t *counters, ft_tune_result *out, cudaStream_t st) {
    if (k < 1 || k > 64 || num == 0) fail(FT_ERR_INVALID_ARGUMENT, "autotuner: the fast walk needs 1 <= k <= 64");
    DevBuf     ref_i(num * (size_t)k * 8), ref_d(num * (size_t)k * 8), ci(num * (size_t)k * 8),
        cd(num * (size_t)k * 8), diff(8);
    const auto cand = walk_candidates(k, true);
    float      best_ms = 0.0f, default_ms = 0.0f;
    int        best = 0;
    for (size_t c = 0; c < cand.size(); ++c) {
        const WalkCandidate &w = cand[c];
        void *oi = c == 0 ? ref_i.p : ci.p, *od = c == 0 ? ref_d.p : cd.p;
        const float ms = time_median(st, 1, [&] {
            batch_self_knn(ctx, all, bt, num, k, excl, (uint64_t *)oi, od, true, w.half, w.variant, rr, rw, counters,
                           st, nullptr, nullptr, w.kc);
        });
        if (c > 0 && (count_diff(ci.p, ref_i.p, num * k, (unsigned long long *)diff.p, st) ||
                      count_diff(cd.p, ref_d.p, num * k, (unsigned long long *)diff.p, st)))
            fail(FT_ERR_RUNTIME, "autotuner: batched walk variant " + std::to_string(w.variant) +
                                     " returned rows that differ from the default's");
        if (c == 0) default_ms = ms;
        if (c == 0 || ms < best_ms) {
            best_ms = ms;
            best    = (int)c;
        }
    }
    TuneChoice tc;
    tc.variant = cand[best].variant;
    tc.half    = cand[best].half;
    tc.kc      = cand[best].kc;
    ctx.tuned[tune_key(TUNE_BATCH, k, num)] = tc;
    fill_result(out, cand[best], 0, best_ms, default_ms, (int)cand.size());
}

void tune_build(Context &ctx, ft_tree &tree, const void *x, const void *y, const void *z, size_t n,
                ft_tune_result *out, cudaStream_t st) {
    if (n < 2) fail(FT_ERR_INVALID_ARGUMENT, "autotuner: the build needs 2+ points");
    const int  words = key_words_of(ctx.opts);
    int        count = 0;
    const int *items = sort_item_choices(words, &count);
    const size_t words8 = (n * sizeof(int32_t) + 7) / 8; // leaf order as 64-bit words (zero padded)
    DevBuf       ref(words8 * 8), cur(words8 * 8), diff(8);
    FT_CUDA(cudaMemsetAsync(ref.p, 0, words8 * 8, st));
    FT_CUDA(cudaMemsetAsync(cur.p, 0, words8 * 8, st));
    float      best_ms = 0.0f, default_ms = 0.0f;
    int        best = 0;
    for (int c = 0; c < count; ++c) {
        const float ms = time_median(st, 3, [&] {
            build_bvh(ctx, tree, x, y, z, n, nullptr, nullptr, nullptr, nullptr, st, items[c]);
        });
        // the leaf order (original index of every leaf slot) must not depend on the tile
        const int32_t *perm = tree.orig_idx + (n - 1);
        FT_CUDA(cudaMemcpyAsync(c == 0 ? ref.p : cur.p, perm, n * sizeof(int32_t), cudaMemcpyDeviceToDevice, st));
        if (c > 0 && count_diff(ref.p, cur.p, words8, (unsigned long long *)diff.p, st))
            fail(FT_ERR_RUNTIME, "autotuner: sort tile of " + std::to_string(items[c]) +
                                     " keys per thread gave a different leaf order");
        if (c == 0) default_ms = ms;
        if (c == 0 || ms < best_ms) {
            best_ms = ms;
            best    = c;
        }
    }
    TuneChoice tc;
    tc.items = items[best];
    ctx.tuned[tune_key(TUNE_BUILD, words, n)] = tc;
    if (out) {
        *out            = ft_tune_result{};
        out->sort_items = items[best];
        out->candidates = count;
        out->best_ms    = best_ms;
        out->default_ms = default_ms;
    }
}

} // namespace ft
