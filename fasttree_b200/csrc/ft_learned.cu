// ft_learned.cu -- learned radius bound for the fast self-kNN walk.  No counterpart in the
// reference.
//
// A small MLP predicts each query's k-th-neighbour distance from cheap tree features; the
// prediction, inflated, becomes the query's pruning bound in the fast walk (ft_fast.cu).  A
// query whose k-th distance ends above its bound, or that finds fewer than k points, is rerun
// by the reference traversal, so results stay bit-exact whatever the network predicts.
//
//  * bound_features_kernel: 12 features per query (all lengths in the walk's distance units),
//    chosen to be invariant to the point density so that a network trained on one draw
//    transfers to a larger one:
//      0-3   log2 diagonal of the leaf's ancestor boxes 2, 4, 6, 8 levels up;
//      4-7   log2 of the number of sorted SFC keys sharing the query's key prefix, at the
//            levels whose cells are 4, 2, 1 and 1/2 times the window distance of feature 10;
//      8     leaf depth minus log2 n;  9  log2 k;
//      10-11 log2 of the k-th and ceil(k/2)-th nearest distance among the SFC window of
//            ranks r-k .. r+k (the window the fast walk seeds from).
//  * MLP 12 -> 64 -> 64 -> 1 with GELU: weights, inputs and hidden activations rounded to
//    bfloat16, products accumulated in fp32.  Inputs are standardised with the training
//    set's mean / std.  The network predicts the standardised residual log2 d_k - feature 10
//    (the true k-th distance relative to the window's); the prediction adds feature 10 back.
//  * Training: per tile of 64 samples the forward and backward passes run in shared memory
//    and write one gradient partial per block; a fixed-order reduction sums them (so a
//    gradient is reproducible) and an Adam step updates the fp32 master weights and their
//    bfloat16 copies.
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <random>
#include <string>
#include <vector>

#include "ft_common.cuh"
#include "ft_internal.h"

namespace ft {

static constexpr int kFeat   = FT_BOUND_FEATURES; // 12
static constexpr int kHid    = 64;
static constexpr int kOffW1  = 0;                     // [kHid][kFeat], row j = hidden unit
static constexpr int kOffB1  = kOffW1 + kHid * kFeat; // 768
static constexpr int kOffW2  = kOffB1 + kHid;         // [kHid][kHid]
static constexpr int kOffB2  = kOffW2 + kHid * kHid;
static constexpr int kOffW3  = kOffB2 + kHid;
static constexpr int kOffB3  = kOffW3 + kHid;
static constexpr int kParams = kOffB3 + 1; // 5057
static_assert(kParams == FT_BOUND_MODEL_PARAMS, "parameter count");
static constexpr int kNorm    = 2 * kFeat + 2; // feature mean, 1/std; target mean, std
static constexpr int kTile    = 64;            // training samples per block
static constexpr int kTrainThreads = 256;

FT_D float bf16r(float x) { return __bfloat162float(__float2bfloat16_rn(x)); }
FT_D float gelu(float z) { return 0.5f * z * (1.0f + erff(z * 0.70710678118654752f)); }
FT_D float gelu_grad(float z) {
    return 0.5f * (1.0f + erff(z * 0.70710678118654752f)) + z * 0.39894228040143268f * expf(-0.5f * z * z);
}

// Floor of a length in distance units before its logarithm (0 is possible: coincident points).
template <class T> FT_HD double len_floor() { return Coord<T>::is_float ? 0x1p-60 : 0.5; }

// =========================================================================================
// Features
// =========================================================================================
template <class T> FT_D double box_diag(const TreeDev<T> &t, int a) {
    const double dx = (double)(T)(t.max_x[a] - t.min_x[a]), dy = (double)(T)(t.max_y[a] - t.min_y[a]),
                 dz = (double)(T)(t.max_z[a] - t.min_z[a]);
    return sqrt(dx * dx + dy * dy + dz * dz);
}

// Number of sorted keys sharing key[rank]'s top p bits (galloping + binary search from rank).
FT_D int prefix_count(const unsigned long long *klo, const unsigned long long *khi, int wide, int n, int rank, int p) {
    auto pre = [&](int j) -> unsigned long long {
        if (p == 0) return 0ull;
        return wide ? (khi[j] >> (62 - p)) : (klo[j] >> (63 - p));
    };
    const unsigned long long P = pre(rank);
    int good = rank, bad = -1;
    for (int s = 1;; s <<= 1) {
        const int j = rank - s;
        if (j < 0) break;
        if (pre(j) != P) {
            bad = j;
            break;
        }
        good = j;
        if (s > n) break;
    }
    while (good - bad > 1) {
        const int m = (good + bad) >> 1;
        if (pre(m) == P) good = m;
        else bad = m;
    }
    const int left = good;
    good = rank;
    bad  = n;
    for (int s = 1;; s <<= 1) {
        const int j = rank + s;
        if (j >= n) break;
        if (pre(j) != P) {
            bad = j;
            break;
        }
        good = j;
        if (s > n) break;
    }
    while (bad - good > 1) {
        const int m = (good + bad) >> 1;
        if (pre(m) == P) good = m;
        else bad = m;
    }
    return good - left + 1;
}

static constexpr int kFeatThreads = 128;
static constexpr int kMaxBoundK   = 64;

// Ascending bitonic sorting network over 64 register values (fully unrolled: every index
// is a compile-time constant, so the array stays in registers).
FT_D void bitonic_sort64(float (&v)[64]) {
#pragma unroll
    for (int size = 2; size <= 64; size <<= 1)
#pragma unroll
        for (int stride = size >> 1; stride > 0; stride >>= 1)
#pragma unroll
            for (int i = 0; i < 64; ++i) {
                const int j = i ^ stride;
                if (j > i) {
                    const float a = v[i], b = v[j];
                    const float lo = fminf(a, b), hi = fmaxf(a, b);
                    if ((i & size) == 0) {
                        v[i] = lo;
                        v[j] = hi;
                    } else {
                        v[i] = hi;
                        v[j] = lo;
                    }
                }
            }
}

// v[i] for a run-time i without dynamic register indexing.
FT_D float pick64(const float (&v)[64], int i) {
    float r = 0.0f;
#pragma unroll
    for (int j = 0; j < 64; ++j) r = (j == i) ? v[j] : r;
    return r;
}

template <class T, int PER>
__global__ void __launch_bounds__(kFeatThreads)
    bound_features_kernel(TreeDev<T> t_all, BatchDev bt, const int32_t *__restrict__ parent_all,
                          const unsigned long long *klo_all, const unsigned long long *khi_all,
                          const int32_t *__restrict__ leaf_ids, int num, int k, const T *__restrict__ qx,
                          const T *__restrict__ qy, const T *__restrict__ qz, float *__restrict__ out,
                          uint32_t *status) {
    using D = typename Coord<T>::dist_t;
    const int q = blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= num) return;
    // batched sets: query q is leaf q - off[s] of the set s holding it, and every array below
    // is that set's (its own tree, parents and sorted keys)
    TreeDev<T>                t      = t_all;
    const int32_t            *parent = parent_all;
    const unsigned long long *klo = klo_all, *khi = khi_all;
    int                       set_rank = -1;
    if (bt.off) {
        const int s = find_set(bt.off, bt.S, q);
        t           = set_view(t_all, bt, s);
        parent      = parent_all + bt.node_off[s];
        klo         = klo_all + bt.off[s];
        khi         = khi_all ? khi_all + bt.off[s] : nullptr; // high words: 126-bit keys only
        set_rank    = q - (int)bt.off[s];
    }
    const int  n   = t.n;
    // external query points (qx != null): leaf_ids holds each point's SFC rank (the lower
    // bound of its key among the sorted keys); the leaf there stands for the point, and the
    // window is the 2k leaves [r - k, r + k) seen from the point itself
    const bool ext  = qx != nullptr;
    const int  rank = set_rank >= 0 ? set_rank : ext ? min(max(leaf_ids[q], 0), n - 1) : (leaf_ids ? leaf_ids[q] : q);
    float     *f    = out + (size_t)q * kFeat;
    if (rank < 0 || rank >= n) {
        atomicOr(status, STATUS_BAD_INPUT);
        for (int i = 0; i < kFeat; ++i) f[i] = 0.0f;
        return;
    }
    const double unit = Coord<T>::dist_shift ? 1.0 / (double)(1ull << Coord<T>::dist_shift) : 1.0;
    const double lf   = len_floor<T>();
    const int    slot = rank + n - 1;

    // ancestors 2, 4, 6, 8 levels up (the root when the path is shorter) and the depth
    int node = slot, depth = 0, anc[4] = {0, 0, 0, 0}, got = 0;
    while (node != 0 && depth < 4096) {
        const int p = parent[node];
        if (p < 0 || p >= n - 1) break;
        node = p;
        ++depth;
        if ((depth & 1) == 0 && depth <= 8) anc[got++] = node;
    }
    for (int i = 0; i < 4; ++i) f[i] = (float)log2(fmax(box_diag(t, i < got ? anc[i] : 0) * unit, lf));

    f[8] = (float)((double)depth - log2((double)n));
    f[9] = (float)log2((double)k);

    // k-th and ceil(k/2)-th nearest distance in the SFC window
    const T   px = ext ? qx[q] : t.min_x[slot], py = ext ? qy[q] : t.min_y[slot], pz = ext ? qz[q] : t.min_z[slot];
    const int kk = min(k, kMaxBoundK);
    const int r0 = max(0, rank - k), r1 = min(n - 1, ext ? rank + k - 1 : rank + k);
    auto      wdist = [&](int j) -> float {
        const int s = j + n - 1;
        return (float)Metric<T>::template dist<(PER != 0), (PER == 2)>(px, py, pz, t.min_x[s], t.max_x[s],
                                                                       t.min_y[s], t.max_y[s], t.min_z[s],
                                                                       t.max_z[s]);
    };
    float wk = 0.0f, wk2 = 0.0f;
    if (k <= 32) {
        // the 64 window slots in registers, sorted by a bitonic network (empty slots +inf)
        float v[64];
#pragma unroll
        for (int i = 0; i < 64; ++i) {
            const int j = rank - k + ((i < k || ext) ? i : i + 1); // a self query skips its own leaf
            v[i]        = (i < 2 * k && j >= r0 && j <= r1) ? wdist(j) : __int_as_float(0x7f800000);
        }
        bitonic_sort64(v);
        const int cnt = ext ? (r1 - r0 + 1) : (r1 - r0); // window leaves other than a self query's own
        if (cnt > 0) {
            const int m = min(kk, cnt);
            wk          = pick64(v, m - 1);
            wk2         = pick64(v, min((kk + 1) / 2, m) - 1);
        }
    } else {
        // max-heap of the kk smallest (local memory)
        float hp[kMaxBoundK];
        int   cnt = 0;
        for (int j = r0; j <= r1; ++j) {
            if (j == rank && !ext) continue;
            const float vv = wdist(j);
            if (cnt < kk) { // sift up
                int i = cnt++;
                while (i > 0) {
                    const int p = (i - 1) >> 1;
                    if (hp[p] >= vv) break;
                    hp[i] = hp[p];
                    i     = p;
                }
                hp[i] = vv;
            } else if (vv < hp[0]) { // replace the maximum, sift down
                int i = 0;
                for (;;) {
                    int l = 2 * i + 1, c = i;
                    if (l >= kk) break;
                    float cv = vv;
                    if (hp[l] > cv) { c = l; cv = hp[l]; }
                    if (l + 1 < kk && hp[l + 1] > cv) { c = l + 1; cv = hp[l + 1]; }
                    if (c == i) break;
                    hp[i] = cv;
                    i     = c;
                }
                hp[i] = vv;
            }
        }
        // heapsort ascending: hp[0..cnt)
        for (int m = cnt; m > 1; --m) {
            const float last = hp[m - 1];
            hp[m - 1]        = hp[0];
            int i = 0, size = m - 1;
            for (;;) {
                int l = 2 * i + 1, c = i;
                if (l >= size) break;
                float cv = last;
                if (hp[l] > cv) { c = l; cv = hp[l]; }
                if (l + 1 < size && hp[l + 1] > cv) { c = l + 1; cv = hp[l + 1]; }
                if (c == i) break;
                hp[i] = cv;
                i     = c;
            }
            hp[i] = last;
        }
        if (cnt) {
            wk  = hp[min(kk, cnt) - 1];
            wk2 = hp[min((kk + 1) / 2, cnt) - 1];
        }
    }
    const double lwk = 0.5 * log2(fmax((double)wk, lf * lf));
    f[10]            = (float)lwk;
    f[11]            = (float)(0.5 * log2(fmax((double)wk2, lf * lf)));

    // SFC-prefix occupancy at the levels whose cells are 4, 2, 1, 1/2 window distances wide:
    // a level-L cell is 2^(bits-L) coordinate units for integer keys and 2^-L of the box's
    // largest side for float keys
    const int wide = Coord<T>::key_words == 2;
    const int lv   = wide ? 20 : 21; // usable levels: 3L top bits within one key word
    double    base;
    if constexpr (Coord<T>::is_float) {
        const double side = fmax(fmax((double)(t.max_x[0] - t.min_x[0]), (double)(t.max_y[0] - t.min_y[0])),
                                 (double)(t.max_z[0] - t.min_z[0]));
        base = log2(fmax(side, lf));
    } else {
        base = (double)Coord<T>::bits;
    }
    const double lw = lwk + (double)Coord<T>::dist_shift; // log2 window distance, coordinate units
    for (int i = 0; i < 4; ++i) {
        const int L = (int)fmin(fmax(floor(base - lw - (double)(2 - i)), 0.0), (double)lv);
        f[4 + i]    = (float)log2((double)prefix_count(klo, khi, wide, n, rank, 3 * L));
    }
}

// Training target of a result row: 0.5 log2 of its k-th distance (NaN when the row has
// fewer than k neighbours).
template <class D>
__global__ void bound_targets_kernel(const unsigned long long *__restrict__ idx, const D *__restrict__ dist, int num,
                                     int k, double lf2, float *out) {
    const int q = blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= num) return;
    const size_t at = (size_t)q * k + (k - 1);
    out[q]          = idx[at] == ~0ull ? __int_as_float(0x7fc00000) : (float)(0.5 * log2(fmax((double)dist[at], lf2)));
}

// =========================================================================================
// MLP
// =========================================================================================
// Shared-memory copy of the network as fp32 values of the bfloat16 weights (training tiles).
struct SmemNet {
    float w1t[kFeat * kHid]; // [i][j]
    float b1[kHid];
    float w2[kHid * kHid];  // [j][i]
    float w2t[kHid * kHid]; // [i][j]
    float b2[kHid];
    float w3[kHid];
    float b3;
    float mu[kFeat], isd[kFeat];
    float t_mu, t_sd;
};

FT_D void load_net(SmemNet &s, const __nv_bfloat16 *__restrict__ pb, const float *__restrict__ norm) {
    for (int e = threadIdx.x; e < kHid * kFeat; e += blockDim.x) {
        const int j = e / kFeat, i = e % kFeat;
        s.w1t[i * kHid + j] = __bfloat162float(pb[kOffW1 + e]);
    }
    for (int e = threadIdx.x; e < kHid * kHid; e += blockDim.x) {
        const int j = e / kHid, i = e % kHid;
        const float w        = __bfloat162float(pb[kOffW2 + e]);
        s.w2[e]              = w;
        s.w2t[i * kHid + j]  = w;
    }
    for (int e = threadIdx.x; e < kHid; e += blockDim.x) {
        s.b1[e] = __bfloat162float(pb[kOffB1 + e]);
        s.b2[e] = __bfloat162float(pb[kOffB2 + e]);
        s.w3[e] = __bfloat162float(pb[kOffW3 + e]);
    }
    if (threadIdx.x < kFeat) {
        s.mu[threadIdx.x]  = norm[threadIdx.x];
        s.isd[threadIdx.x] = norm[kFeat + threadIdx.x];
    }
    if (threadIdx.x == 0) {
        s.b3   = __bfloat162float(pb[kOffB3]);
        s.t_mu = norm[2 * kFeat];
        s.t_sd = norm[2 * kFeat + 1];
    }
}

// Standardised input rounded to bfloat16.
FT_D float in_feat(const SmemNet &s, const float *raw, int i) { return bf16r((raw[i] - s.mu[i]) * s.isd[i]); }

// =========================================================================================
// Inference on the 5th-generation tensor cores (tcgen05, accumulators in tensor memory).
// Persistent CTAs of 128 threads take tiles of 128 queries:
//   A1 [128 x 16] = standardised features in bfloat16 (K padded from 12 with zeros)
//   D1 [128 x 64] = A1 x W1^T          one tcgen05.mma M=128 N=64 K=16, fp32 in TMEM
//   A2 [128 x 64] = bf16(gelu(D1 + b1)) epilogue: tcgen05.ld -> registers -> shared memory
//   D2 [128 x 64] = A2 x W2^T          four K=16 steps into the same 64 TMEM columns
//   y             = w3 . bf16(gelu(D2 + b2)) + b3, one query per thread (TMEM lane = row)
// Operands sit in shared memory in the canonical no-swizzle K-major layout: 8-row x 16-byte
// core matrices, adjacent along K 128 bytes apart (leading byte offset), adjacent along
// M / N (K/8) x 128 bytes apart (stride byte offset).  One thread issues the MMAs; their
// completion reaches an mbarrier through tcgen05.commit, and every wait on it is bounded.
// =========================================================================================
static constexpr int kTcRows  = 128;
static constexpr int kTcCols  = 64; // TMEM columns per CTA (fp32 accumulator N = 64)
static constexpr int kK1      = 16; // layer-1 K (12 features + 4 zero columns)

struct TcSmem {
    __align__(16) uint16_t w1[kHid * kK1];   // B operand of layer 1, canonical layout
    __align__(16) uint16_t w2[kHid * kHid];  // B operand of layer 2
    __align__(16) uint16_t a1[kTcRows * kK1];
    __align__(16) uint16_t a2[kTcRows * kHid];
    float    b1[kHid], b2[kHid], w3[kHid];
    float    mu[kFeat], isd[kFeat];
    float    b3, t_mu, t_sd;
    uint64_t mbar;
    uint32_t tmem;
    int      abort;
};

// Byte offset of element (row, k) of an operand with K columns in the canonical layout.
FT_HD uint32_t canon(int row, int k, int K) {
    return (uint32_t)((((row >> 3) * (K >> 3) + (k >> 3)) * 128) + (row & 7) * 16 + (k & 7) * 2);
}

FT_D uint32_t smem_u32(const void *p) { return (uint32_t)__cvta_generic_to_shared(p); }

// Shared-memory matrix descriptor: start address, leading / stride byte offsets (all >> 4),
// the fixed 0b001 at bits 46-48, base offset 0, no swizzle.
FT_D uint64_t tc_desc(uint32_t saddr, uint32_t lbo, uint32_t sbo) {
    return (uint64_t)((saddr >> 4) & 0x3FFFu) | ((uint64_t)((lbo >> 4) & 0x3FFFu) << 16) |
           ((uint64_t)((sbo >> 4) & 0x3FFFu) << 32) | (1ull << 46);
}

// Instruction descriptor of kind::f16: fp32 accumulator, bf16 A and B, both K-major, N, M.
__host__ __device__ constexpr uint32_t tc_idesc(int M, int N) {
    return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(N >> 3) << 17) | ((uint32_t)(M >> 4) << 24);
}

FT_D void tc_mma(uint32_t d_tmem, uint64_t adesc, uint64_t bdesc, uint32_t idesc, uint32_t accumulate) {
    asm volatile("{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
                 "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(d_tmem),
                 "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate));
}
FT_D void tc_commit(uint32_t mbar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(mbar)
                 : "memory");
}
FT_D bool mbar_try_wait(uint32_t mbar, uint32_t phase) {
    uint32_t ok;
    asm volatile("{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
                 "selp.u32 %0, 1, 0, p;\n\t}\n"
                 : "=r"(ok)
                 : "r"(mbar), "r"(phase)
                 : "memory");
    return ok != 0;
}
// Bounded wait for an mbarrier phase; false when it gave up.
FT_D bool mbar_wait(uint32_t mbar, uint32_t phase) {
    for (long long it = 0; it < (1ll << 26); ++it) {
        if (mbar_try_wait(mbar, phase)) return true;
        if (it > 64) __nanosleep(64);
    }
    return false;
}
FT_D void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
FT_D void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
FT_D void fence_async_smem() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

// 16 consecutive fp32 columns of this thread's TMEM lane.
FT_D void tc_ld16(uint32_t taddr, float *v) {
    uint32_t r[16];
    asm volatile("tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, "
                 "%13, %14, %15}, [%16];"
                 : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
                   "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]),
                   "=r"(r[15])
                 : "r"(taddr));
#pragma unroll
    for (int i = 0; i < 16; ++i) v[i] = __uint_as_float(r[i]);
}
FT_D void tc_wait_ld() { asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory"); }

template <class D>
__global__ void __launch_bounds__(kTcRows)
    bound_predict_tc_kernel(const __nv_bfloat16 *__restrict__ pb, const float *__restrict__ norm,
                            const float *__restrict__ feats, int num, float inflation, float *pred, D *bound,
                            uint32_t *status) {
    extern __shared__ __align__(16) unsigned char smem_tc[];
    TcSmem        &s    = *reinterpret_cast<TcSmem *>(smem_tc);
    const int      tid  = threadIdx.x, warp = tid >> 5;
    const uint16_t *raw = reinterpret_cast<const uint16_t *>(pb);
    // weights into the canonical layouts (W1's columns 12..15 are zero)
    for (int e = tid; e < kHid * kK1; e += kTcRows) {
        const int j = e / kK1, k = e % kK1;
        *reinterpret_cast<uint16_t *>(reinterpret_cast<unsigned char *>(s.w1) + canon(j, k, kK1)) =
            k < kFeat ? raw[kOffW1 + j * kFeat + k] : (uint16_t)0;
    }
    for (int e = tid; e < kHid * kHid; e += kTcRows) {
        const int j = e / kHid, k = e % kHid;
        *reinterpret_cast<uint16_t *>(reinterpret_cast<unsigned char *>(s.w2) + canon(j, k, kHid)) = raw[kOffW2 + e];
    }
    for (int e = tid; e < kHid; e += kTcRows) {
        s.b1[e] = __bfloat162float(pb[kOffB1 + e]);
        s.b2[e] = __bfloat162float(pb[kOffB2 + e]);
        s.w3[e] = __bfloat162float(pb[kOffW3 + e]);
    }
    if (tid < kFeat) {
        s.mu[tid]  = norm[tid];
        s.isd[tid] = norm[kFeat + tid];
    }
    if (tid == 0) {
        s.b3    = __bfloat162float(pb[kOffB3]);
        s.t_mu  = norm[2 * kFeat];
        s.t_sd  = norm[2 * kFeat + 1];
        s.abort = 0;
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(&s.mbar)) : "memory");
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(&s.tmem)),
                     "r"(kTcCols)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    fence_async_smem();
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem  = s.tmem;
    const uint32_t mbar  = smem_u32(&s.mbar);
    const uint32_t lane0 = tmem + ((uint32_t)(32 * warp) << 16); // this warp's TMEM lanes
    const uint32_t id1 = tc_idesc(kTcRows, kHid), id2 = tc_idesc(kTcRows, kHid);
    const uint32_t a1 = smem_u32(s.a1), a2 = smem_u32(s.a2), w1 = smem_u32(s.w1), w2 = smem_u32(s.w2);
    uint32_t       phase = 0;
    unsigned char *sa1 = reinterpret_cast<unsigned char *>(s.a1), *sa2 = reinterpret_cast<unsigned char *>(s.a2);

    for (int tile = blockIdx.x; tile * kTcRows < num; tile += gridDim.x) {
        const int q = tile * kTcRows + tid;
        // ---- A1: this thread's row ----
        {
            __align__(16) uint16_t v[kK1];
#pragma unroll
            for (int k = 0; k < kK1; ++k) {
                float x = 0.0f;
                if (k < kFeat && q < num) x = (feats[(size_t)q * kFeat + k] - s.mu[k]) * s.isd[k];
                v[k] = __bfloat16_as_ushort(__float2bfloat16_rn(x));
            }
#pragma unroll
            for (int c = 0; c < kK1 / 8; ++c)
                *reinterpret_cast<uint4 *>(sa1 + canon(tid, 8 * c, kK1)) = *reinterpret_cast<const uint4 *>(v + 8 * c);
        }
        fence_async_smem();
        tc_fence_before();
        __syncthreads();
        if (tid == 0) {
            tc_fence_after();
            tc_mma(tmem, tc_desc(a1, 128, (kK1 / 8) * 128), tc_desc(w1, 128, (kK1 / 8) * 128), id1, 0u);
            tc_commit(mbar);
        }
        if (!mbar_wait(mbar, phase)) atomicOr(&s.abort, 1);
        phase ^= 1u;
        tc_fence_after();
        __syncthreads();
        if (s.abort) break;
        // ---- epilogue 1: bias, GELU, bf16 -> A2 row ----
        {
            float z[16];
#pragma unroll
            for (int c = 0; c < kHid / 16; ++c) {
                tc_ld16(lane0 + 16 * c, z);
                tc_wait_ld();
                __align__(16) uint16_t h[16];
#pragma unroll
                for (int i = 0; i < 16; ++i)
                    h[i] = __bfloat16_as_ushort(__float2bfloat16_rn(gelu(z[i] + s.b1[16 * c + i])));
                *reinterpret_cast<uint4 *>(sa2 + canon(tid, 16 * c, kHid))     = *reinterpret_cast<const uint4 *>(h);
                *reinterpret_cast<uint4 *>(sa2 + canon(tid, 16 * c + 8, kHid)) = *reinterpret_cast<const uint4 *>(h + 8);
            }
        }
        fence_async_smem();
        tc_fence_before();
        __syncthreads();
        if (tid == 0) {
            tc_fence_after();
#pragma unroll
            for (int ks = 0; ks < kHid / 16; ++ks) // K step of 16 = two core matrices = 256 bytes
                tc_mma(tmem, tc_desc(a2 + 256 * ks, 128, (kHid / 8) * 128), tc_desc(w2 + 256 * ks, 128, (kHid / 8) * 128),
                       id2, ks > 0 ? 1u : 0u);
            tc_commit(mbar);
        }
        if (!mbar_wait(mbar, phase)) atomicOr(&s.abort, 1);
        phase ^= 1u;
        tc_fence_after();
        __syncthreads();
        if (s.abort) break;
        // ---- epilogue 2: bias, GELU, bf16, output layer ----
        float y = s.b3;
        {
            float z[16];
#pragma unroll
            for (int c = 0; c < kHid / 16; ++c) {
                tc_ld16(lane0 + 16 * c, z);
                tc_wait_ld();
#pragma unroll
                for (int i = 0; i < 16; ++i) y = fmaf(s.w3[16 * c + i], bf16r(gelu(z[i] + s.b2[16 * c + i])), y);
            }
        }
        if (q < num) {
            const float lp = feats[(size_t)q * kFeat + 10] + fmaf(y, s.t_sd, s.t_mu);
            if (pred) pred[q] = lp;
            if (bound) {
                const double len = exp2((double)lp) * (double)inflation;
                const double b2  = len * len;
                if constexpr (std::is_same<D, double>::value) bound[q] = b2;
                else bound[q] = (b2 >= 1.8446744073709552e19) ? ~0ull : (unsigned long long)ceil(b2);
            }
        }
        tc_fence_before();
        __syncthreads(); // every lane has read D2 before the next tile's MMA overwrites it
        tc_fence_after();
    }
    if (s.abort) {
        if (tid == 0) atomicOr(status, STATUS_SPIN_LIMIT);
        mbar_wait(mbar, phase ^ 1u); // the phase that timed out: let its MMA finish (bounded) before freeing TMEM
    }
    tc_fence_before();
    __syncthreads();
    if (warp == 0) {
        tc_fence_after();
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(kTcCols) : "memory");
    }
}

// Training tile: forward + backward of 64 samples (rows[]) in shared memory; gradient of the
// mean squared error of the standardised target, summed over the tile, into part[block].
struct TrainSmem {
    SmemNet net;
    float   x[kTile][kFeat];
    float   z1[kTile][kHid]; // Z1, later dZ1
    float   h1[kTile][kHid];
    float   z2[kTile][kHid]; // Z2, later dZ2
    float   h2[kTile][kHid]; // H2, later dH1
    float   y[kTile], t[kTile], dy[kTile];
};

__global__ void __launch_bounds__(kTrainThreads)
    mlp_train_tile_kernel(const __nv_bfloat16 *__restrict__ pb, const float *__restrict__ norm,
                          const float *__restrict__ feats, const float *__restrict__ targets,
                          const int32_t *__restrict__ rows, int batch, float *part, float *loss_part) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    TrainSmem &s   = *reinterpret_cast<TrainSmem *>(smem_raw);
    const int  tid = threadIdx.x;
    const int  s0  = blockIdx.x * kTile;
    load_net(s.net, pb, norm);
    __syncthreads();
    const float inv_b = 1.0f / (float)batch;
    for (int e = tid; e < kTile * kFeat; e += kTrainThreads) {
        const int r = e / kFeat, i = e % kFeat;
        const int g = s0 + r;
        s.x[r][i]   = g < batch ? in_feat(s.net, feats + (size_t)rows[g] * kFeat, i) : 0.0f;
    }
    for (int r = tid; r < kTile; r += kTrainThreads) {
        const int g = s0 + r;
        s.t[r]      = g < batch ? (targets[rows[g]] - feats[(size_t)rows[g] * kFeat + 10] - s.net.t_mu) / s.net.t_sd
                                : 0.0f;
    }
    __syncthreads();
    // layer 1
    for (int e = tid; e < kTile * kHid; e += kTrainThreads) {
        const int r = e / kHid, j = e % kHid;
        float     z = s.net.b1[j];
#pragma unroll
        for (int i = 0; i < kFeat; ++i) z = fmaf(s.net.w1t[i * kHid + j], s.x[r][i], z);
        s.z1[r][j] = z;
        s.h1[r][j] = bf16r(gelu(z));
    }
    __syncthreads();
    // layer 2
    for (int e = tid; e < kTile * kHid; e += kTrainThreads) {
        const int r = e / kHid, j = e % kHid;
        float     z = s.net.b2[j];
#pragma unroll 16
        for (int i = 0; i < kHid; ++i) z = fmaf(s.net.w2t[i * kHid + j], s.h1[r][i], z);
        s.z2[r][j] = z;
        s.h2[r][j] = bf16r(gelu(z));
    }
    __syncthreads();
    // output, loss, dy (one warp per 32 samples, lanes over hidden units)
    {
        const int lane = tid & 31, w = tid >> 5;
        for (int r = w; r < kTile; r += kTrainThreads / 32) {
            float acc = s.net.w3[lane] * s.h2[r][lane] + s.net.w3[lane + 32] * s.h2[r][lane + 32];
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
            if (lane == 0) {
                const float y = acc + s.net.b3;
                const bool  v = s0 + r < batch;
                s.y[r]        = y;
                s.dy[r]       = v ? 2.0f * (y - s.t[r]) * inv_b : 0.0f;
            }
        }
    }
    __syncthreads();
    float *g = part + (size_t)blockIdx.x * kParams;
    if (tid == 0) {
        float l = 0.0f, db3 = 0.0f;
        for (int r = 0; r < kTile; ++r) {
            if (s0 + r < batch) l += (s.y[r] - s.t[r]) * (s.y[r] - s.t[r]);
            db3 += s.dy[r];
        }
        loss_part[blockIdx.x] = l;
        g[kOffB3]             = db3;
    }
    // dW3, then dZ2 = dy w3 gelu'(Z2) in place
    for (int j = tid; j < kHid; j += kTrainThreads) {
        float a = 0.0f;
        for (int r = 0; r < kTile; ++r) a = fmaf(s.dy[r], s.h2[r][j], a);
        g[kOffW3 + j] = a;
    }
    __syncthreads();
    for (int e = tid; e < kTile * kHid; e += kTrainThreads) {
        const int r = e / kHid, j = e % kHid;
        s.z2[r][j]  = s.dy[r] * s.net.w3[j] * gelu_grad(s.z2[r][j]);
    }
    __syncthreads();
    // dW2[j][i] = sum_r dZ2[r][j] H1[r][i];  db2
    for (int e = tid; e < kHid * kHid; e += kTrainThreads) {
        const int j = e / kHid, i = e % kHid;
        float     a = 0.0f;
        for (int r = 0; r < kTile; ++r) a = fmaf(s.z2[r][j], s.h1[r][i], a);
        g[kOffW2 + e] = a;
    }
    for (int j = tid; j < kHid; j += kTrainThreads) {
        float a = 0.0f;
        for (int r = 0; r < kTile; ++r) a += s.z2[r][j];
        g[kOffB2 + j] = a;
    }
    // dH1[r][i] = sum_j dZ2[r][j] W2[j][i] (into h2)
    for (int e = tid; e < kTile * kHid; e += kTrainThreads) {
        const int r = e / kHid, i = e % kHid;
        float     a = 0.0f;
#pragma unroll 16
        for (int j = 0; j < kHid; ++j) a = fmaf(s.z2[r][j], s.net.w2[j * kHid + i], a);
        s.h2[r][i] = a;
    }
    __syncthreads();
    for (int e = tid; e < kTile * kHid; e += kTrainThreads) {
        const int r = e / kHid, j = e % kHid;
        s.z1[r][j]  = s.h2[r][j] * gelu_grad(s.z1[r][j]);
    }
    __syncthreads();
    // dW1[j][i] = sum_r dZ1[r][j] X[r][i];  db1
    for (int e = tid; e < kHid * kFeat; e += kTrainThreads) {
        const int j = e / kFeat, i = e % kFeat;
        float     a = 0.0f;
        for (int r = 0; r < kTile; ++r) a = fmaf(s.z1[r][j], s.x[r][i], a);
        g[kOffW1 + e] = a;
    }
    for (int j = tid; j < kHid; j += kTrainThreads) {
        float a = 0.0f;
        for (int r = 0; r < kTile; ++r) a += s.z1[r][j];
        g[kOffB1 + j] = a;
    }
}

// Fixed-order sum of the per-block partials (reproducible gradient) and of the loss.
__global__ void mlp_reduce_kernel(const float *__restrict__ part, const float *__restrict__ loss_part, int blocks,
                                  int batch, float *grad, float *loss) {
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p < kParams) {
        float a = 0.0f;
        for (int b = 0; b < blocks; ++b) a += part[(size_t)b * kParams + p];
        grad[p] = a;
    }
    if (p == 0) {
        float l = 0.0f;
        for (int b = 0; b < blocks; ++b) l += loss_part[b];
        *loss = l / (float)batch;
    }
}

// Adam (bias-corrected) on the fp32 master weights; refreshes the bfloat16 copies.
__global__ void mlp_adam_kernel(float *params, float *m, float *v, const float *__restrict__ grad,
                                __nv_bfloat16 *pb, float lr, float b1, float b2, float eps, float c1, float c2) {
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= kParams) return;
    const float g  = grad[p];
    const float mm = b1 * m[p] + (1.0f - b1) * g;
    const float vv = b2 * v[p] + (1.0f - b2) * g * g;
    m[p]           = mm;
    v[p]           = vv;
    const float w  = params[p] - lr * (mm / c1) / (sqrtf(vv / c2) + eps);
    params[p]      = w;
    pb[p]          = __float2bfloat16_rn(w);
}

__global__ void mlp_to_bf16_kernel(const float *params, __nv_bfloat16 *pb) {
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p < kParams) pb[p] = __float2bfloat16_rn(params[p]);
}

// Minibatch rows: splitmix64(seed, step, i) mod n.
__global__ void mlp_rows_kernel(int32_t *rows, int batch, int n, unsigned long long seed, int step) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= batch) return;
    unsigned long long z = seed + 0x9E3779B97F4A7C15ull * ((unsigned long long)step * 0x100000001ull + i + 1);
    z                    = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z                    = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    z ^= z >> 31;
    rows[i] = (int32_t)(z % (unsigned long long)n);
}

__global__ void iota_kernel(int32_t *rows, int n) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) rows[i] = i;
}

// =========================================================================================
// Host side
// =========================================================================================
struct BoundModel {
    int            device  = 0;
    float         *params  = nullptr; // fp32 master
    float         *m       = nullptr, *v = nullptr, *grad = nullptr;
    __nv_bfloat16 *pb      = nullptr;
    float         *norm    = nullptr; // kNorm floats
    float         *part    = nullptr, *loss_part = nullptr, *loss = nullptr;
    int32_t       *rows    = nullptr;
    int            cap_rows = 0, cap_blocks = 0;
    int            step    = 0;
};

template <class X> static X *dmalloc(size_t count) {
    void *p = nullptr;
    cudaError_t e = cudaMalloc(&p, std::max<size_t>(count, 1) * sizeof(X));
    if (e != cudaSuccess) {
        cudaGetLastError();
        fail(FT_ERR_OUT_OF_MEMORY, "cudaMalloc of learned-bound storage failed");
    }
    return (X *)p;
}

void bound_model_free(BoundModel *b) {
    if (!b) return;
    void *ptrs[] = {b->params, b->m, b->v, b->grad, b->pb, b->norm, b->part, b->loss_part, b->loss, b->rows};
    for (void *p : ptrs)
        if (p) cudaFree(p);
    delete b;
}

// PyTorch-style initialisation: U(-1/sqrt(fan_in), 1/sqrt(fan_in)) for weights and biases.
static std::vector<float> init_params(unsigned long long seed) {
    std::mt19937_64                       rng(seed);
    std::vector<float>                    p(kParams);
    auto fill = [&](int off, int count, int fan_in) {
        std::uniform_real_distribution<float> u(-1.0f / std::sqrt((float)fan_in), 1.0f / std::sqrt((float)fan_in));
        for (int i = 0; i < count; ++i) p[off + i] = u(rng);
    };
    fill(kOffW1, kHid * kFeat, kFeat);
    fill(kOffB1, kHid, kFeat);
    fill(kOffW2, kHid * kHid, kHid);
    fill(kOffB2, kHid, kHid);
    fill(kOffW3, kHid, kHid);
    fill(kOffB3, 1, kHid);
    return p;
}

void bound_model_set_params(BoundModel &b, const float *host, cudaStream_t st) {
    FT_CUDA(cudaMemcpyAsync(b.params, host, kParams * sizeof(float), cudaMemcpyHostToDevice, st));
    mlp_to_bf16_kernel<<<(kParams + 255) / 256, 256, 0, st>>>(b.params, b.pb);
    FT_CUDA(cudaGetLastError());
    FT_CUDA(cudaMemsetAsync(b.m, 0, kParams * sizeof(float), st));
    FT_CUDA(cudaMemsetAsync(b.v, 0, kParams * sizeof(float), st));
    FT_CUDA(cudaStreamSynchronize(st));
    b.step = 0;
}

BoundModel *bound_model_create(Context &ctx, unsigned long long seed) {
    BoundModel *b = new BoundModel();
    try {
        b->device = ctx.device;
        b->params = dmalloc<float>(kParams);
        b->m      = dmalloc<float>(kParams);
        b->v      = dmalloc<float>(kParams);
        b->grad   = dmalloc<float>(kParams);
        b->pb     = dmalloc<__nv_bfloat16>(kParams);
        b->norm   = dmalloc<float>(kNorm);
        b->loss   = dmalloc<float>(1);
        std::vector<float> nrm(kNorm, 0.0f);
        for (int i = 0; i < kFeat; ++i) nrm[kFeat + i] = 1.0f;
        nrm[2 * kFeat + 1] = 1.0f;
        FT_CUDA(cudaMemcpy(b->norm, nrm.data(), kNorm * sizeof(float), cudaMemcpyHostToDevice));
        std::vector<float> p = init_params(seed);
        bound_model_set_params(*b, p.data(), nullptr);
    } catch (...) {
        bound_model_free(b);
        throw;
    }
    return b;
}

void bound_model_get_params(BoundModel &b, float *host) {
    FT_CUDA(cudaMemcpy(host, b.params, kParams * sizeof(float), cudaMemcpyDeviceToHost));
}

void bound_model_set_norm(BoundModel &b, const float *mean12, const float *std12, float t_mean, float t_std) {
    std::vector<float> nrm(kNorm);
    for (int i = 0; i < kFeat; ++i) {
        nrm[i]         = mean12[i];
        nrm[kFeat + i] = 1.0f / std::max(std12[i], 1e-3f);
    }
    nrm[2 * kFeat]     = t_mean;
    nrm[2 * kFeat + 1] = std::max(t_std, 1e-3f);
    FT_CUDA(cudaMemcpy(b.norm, nrm.data(), kNorm * sizeof(float), cudaMemcpyHostToDevice));
}

static void ensure_train(BoundModel &b, int batch) {
    const int blocks = (batch + kTile - 1) / kTile;
    if (batch > b.cap_rows) {
        if (b.rows) cudaFree(b.rows);
        b.rows     = nullptr;
        b.rows     = dmalloc<int32_t>(batch);
        b.cap_rows = batch;
    }
    if (blocks > b.cap_blocks) {
        if (b.part) cudaFree(b.part);
        if (b.loss_part) cudaFree(b.loss_part);
        b.part = b.loss_part = nullptr;
        b.part       = dmalloc<float>((size_t)blocks * kParams);
        b.loss_part  = dmalloc<float>(blocks);
        b.cap_blocks = blocks;
    }
}

static void train_tile_launch(BoundModel &b, const float *feats, const float *targets, int batch, cudaStream_t st) {
    const int    blocks = (batch + kTile - 1) / kTile;
    const size_t smem   = sizeof(TrainSmem);
    FT_CUDA(cudaFuncSetAttribute(mlp_train_tile_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    mlp_train_tile_kernel<<<blocks, kTrainThreads, smem, st>>>(b.pb, b.norm, feats, targets, b.rows, batch, b.part,
                                                              b.loss_part);
    mlp_reduce_kernel<<<(kParams + 255) / 256, 256, 0, st>>>(b.part, b.loss_part, blocks, batch, b.grad, b.loss);
    FT_CUDA(cudaGetLastError());
}

// Gradient of the mean squared error over samples [0, n) (no update).
void bound_model_gradient(BoundModel &b, const float *feats, const float *targets, int n, float *grad_host,
                          float *loss_host, cudaStream_t st) {
    ensure_train(b, n);
    iota_kernel<<<(n + 255) / 256, 256, 0, st>>>(b.rows, n);
    train_tile_launch(b, feats, targets, n, st);
    if (grad_host) FT_CUDA(cudaMemcpyAsync(grad_host, b.grad, kParams * sizeof(float), cudaMemcpyDeviceToHost, st));
    if (loss_host) FT_CUDA(cudaMemcpyAsync(loss_host, b.loss, sizeof(float), cudaMemcpyDeviceToHost, st));
    FT_CUDA(cudaStreamSynchronize(st));
}

// `steps` Adam steps on random minibatches of `batch` rows of [0, n).
void bound_model_fit(BoundModel &b, const float *feats, const float *targets, int n, int steps, int batch, float lr,
                     unsigned long long seed, float *loss_host, cudaStream_t st) {
    if (n <= 0 || steps <= 0) return;
    batch = std::max(1, batch);
    ensure_train(b, batch);
    const float b1 = 0.9f, b2 = 0.999f, eps = 1e-8f;
    for (int s = 0; s < steps; ++s) {
        mlp_rows_kernel<<<(batch + 255) / 256, 256, 0, st>>>(b.rows, batch, n, seed, b.step);
        train_tile_launch(b, feats, targets, batch, st);
        ++b.step;
        const float c1 = 1.0f - std::pow(b1, (float)b.step), c2 = 1.0f - std::pow(b2, (float)b.step);
        mlp_adam_kernel<<<(kParams + 255) / 256, 256, 0, st>>>(b.params, b.m, b.v, b.grad, b.pb, lr, b1, b2, eps, c1,
                                                             c2);
        FT_CUDA(cudaGetLastError());
        if (loss_host) FT_CUDA(cudaMemcpyAsync(loss_host + s, b.loss, sizeof(float), cudaMemcpyDeviceToHost, st));
    }
    if (loss_host) FT_CUDA(cudaStreamSynchronize(st));
}

// Inference runs on the tensor cores (bound_predict_tc_kernel): 4 CTAs of 128 threads per
// SM, each holding 64 TMEM columns (256 of the SM's 512 even with 8 resident), over tiles of
// 128 queries.
static_assert(sizeof(TcSmem) + 1024 >= 227 * 1024 / 8, "at most 8 CTAs per SM, 64 TMEM columns each");
void bound_model_predict(Context &ctx, BoundModel &b, const float *feats, size_t n, float inflation, float *pred,
                         void *bound, cudaStream_t st) {
    if (n == 0) return;
    const int    grid = (int)std::min<size_t>((n + kTcRows - 1) / kTcRows, (size_t)ctx.num_sms * 4);
    const size_t smem = sizeof(TcSmem) + 1024; // padding keeps residency at <= 8 CTAs per SM
    if (ctx.opts.coord_type == F32 || ctx.opts.coord_type == F64) {
        FT_CUDA(cudaFuncSetAttribute(bound_predict_tc_kernel<double>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     (int)smem));
        bound_predict_tc_kernel<double><<<grid, kTcRows, smem, st>>>(b.pb, b.norm, feats, (int)n, inflation, pred,
                                                                     (double *)bound, ctx.status);
    } else {
        FT_CUDA(cudaFuncSetAttribute(bound_predict_tc_kernel<unsigned long long>,
                                     cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
        bound_predict_tc_kernel<unsigned long long><<<grid, kTcRows, smem, st>>>(
            b.pb, b.norm, feats, (int)n, inflation, pred, (unsigned long long *)bound, ctx.status);
    }
    FT_CUDA(cudaGetLastError());
}

template <class T>
static void features_typed(Context &ctx, const ft_tree &tr, const int32_t *leaf_ids, int num, int k, const void *qx,
                           const void *qy, const void *qz, float *out, cudaStream_t st, const BatchDev &bt) {
    const TreeImpl &impl = *(const TreeImpl *)tr.impl;
    if (!impl.key_lo || (Coord<T>::key_words == 2 && !impl.key_hi))
        fail(FT_ERR_INVALID_ARGUMENT, "learned bound: the tree's sorted keys are missing");
    TreeDev<T>      tv   = tree_view<T>(tr);
    const int       grid = (num + kFeatThreads - 1) / kFeatThreads;
    met_dispatch<T>(metric_mode<T>(ctx.opts, tr), [&](auto M) {
        bound_features_kernel<T, decltype(M)::value><<<grid, kFeatThreads, 0, st>>>(
            tv, bt, tr.parent, (const unsigned long long *)impl.key_lo, (const unsigned long long *)impl.key_hi,
            leaf_ids, num, k, (const T *)qx, (const T *)qy, (const T *)qz, out, ctx.status);
    });
    FT_CUDA(cudaGetLastError());
}

// leaf_ids: self queries (null: every leaf); or, with qx/qy/qz, the SFC ranks of external
// query points; with bt, every leaf of a batch of sets.
static void features_impl(Context &ctx, const ft_tree &tr, const int32_t *leaf_ids, size_t num, int k,
                          const void *qx, const void *qy, const void *qz, float *out, cudaStream_t st,
                          const BatchDev &bt = {}) {
    switch (ctx.opts.coord_type) {
    case F32: features_typed<float>(ctx, tr, leaf_ids, (int)num, k, qx, qy, qz, out, st, bt); break;
    case F64: features_typed<double>(ctx, tr, leaf_ids, (int)num, k, qx, qy, qz, out, st, bt); break;
    case U32: features_typed<uint32_t>(ctx, tr, leaf_ids, (int)num, k, qx, qy, qz, out, st, bt); break;
    case U64: features_typed<unsigned long long>(ctx, tr, leaf_ids, (int)num, k, qx, qy, qz, out, st, bt); break;
    }
}

// The 12 features of every leaf of a batch of sets (`all` spans the concatenated arrays; its
// sorted keys are the sets' own, back to back).  Asynchronous; allocates nothing.
void bound_features_batch(Context &ctx, const ft_tree &all, const BatchDev &bt, size_t num, int k, float *out,
                          cudaStream_t st) {
    if (k < 1 || k > kMaxBoundK) fail(FT_ERR_INVALID_ARGUMENT, "learned bound: k must be in [1, 64]");
    if (num == 0) return;
    features_impl(ctx, all, nullptr, num, k, nullptr, nullptr, nullptr, out, st, bt);
}

static void check_bound_tree(const ft_tree &tr, int k) {
    const TreeImpl *impl = (const TreeImpl *)tr.impl;
    if (k < 1 || k > kMaxBoundK) fail(FT_ERR_INVALID_ARGUMENT, "learned bound: k must be in [1, 64]");
    if (!impl || impl->view || !impl->key_lo || impl->height_root < 0)
        fail(FT_ERR_INVALID_ARGUMENT, "learned bound: the tree must be built by ft_build_bvh / ft_build_tree");
}

void bound_features(Context &ctx, const ft_tree &tr, const int32_t *leaf_ids, size_t num, int k, float *out,
                    cudaStream_t st) {
    check_bound_tree(tr, k);
    if (num == 0 || tr.num_leaves == 0) return;
    features_impl(ctx, tr, leaf_ids, num, k, nullptr, nullptr, nullptr, out, st);
}

// Features of external query points: their SFC ranks first (the tree's own keys), then the
// features seen from each point.
void bound_features_points(Context &ctx, const ft_tree &tr, const void *qx, const void *qy, const void *qz,
                           size_t nq, int k, float *out, cudaStream_t st) {
    check_bound_tree(tr, k);
    if (!((const TreeImpl *)tr.impl)->own_keys)
        fail(FT_ERR_INVALID_ARGUMENT, "learned bound: the tree's keys must be this library's (ft_build_bvh "
                                      "without caller keys) to place external points");
    if (nq == 0 || tr.num_leaves == 0) return;
    query_seed_ranks(ctx, tr, qx, qy, qz, nq, st);
    features_impl(ctx, tr, ctx.seed_ranks, nq, k, qx, qy, qz, out, st);
}

void bound_targets(Context &ctx, const uint64_t *idx, const void *dist, size_t num, int k, float *out,
                   cudaStream_t st) {
    if (num == 0) return;
    const int grid = (int)((num + 255) / 256);
    if (ctx.opts.coord_type == F32 || ctx.opts.coord_type == F64)
        bound_targets_kernel<double><<<grid, 256, 0, st>>>((const unsigned long long *)idx, (const double *)dist,
                                                           (int)num, k, 0x1p-120, out);
    else
        bound_targets_kernel<unsigned long long><<<grid, 256, 0, st>>>((const unsigned long long *)idx,
                                                                       (const unsigned long long *)dist, (int)num, k,
                                                                       0.25, out);
    FT_CUDA(cudaGetLastError());
}

static void ensure_learned(Context &ctx, size_t num) {
    if (num <= ctx.learned_cap) return;
    if (ctx.learned_feats) cudaFree(ctx.learned_feats);
    if (ctx.learned_bound) cudaFree(ctx.learned_bound);
    ctx.learned_feats = nullptr;
    ctx.learned_bound = nullptr;
    ctx.learned_cap   = 0;
    const size_t cap  = num + num / 4 + 1024;
    ctx.learned_feats = dmalloc<float>(cap * kFeat);
    ctx.learned_bound = dmalloc<unsigned long long>(cap);
    ctx.learned_cap   = cap;
}

// knn_query of external points with the learned bound: features (from each point's SFC
// rank) -> bound -> the fast walk with the bound; misses and ties are rerun by knn_query's
// heap tier, so the output equals knn_query's.
void knn_learned(Context &ctx, const ft_tree &tr, BoundModel &b, const void *qx, const void *qy, const void *qz,
                 size_t nq, int k, int max_k, float inflation, uint64_t *idx, void *dist, const ft_query_options &q,
                 cudaStream_t st) {
    if (nq == 0 || k <= 0 || tr.num_leaves == 0) return;
    if (k > kMaxBoundK) fail(FT_ERR_INVALID_ARGUMENT, "learned bound: k must be in [1, 64]");
    ensure_learned(ctx, nq);
    bound_features_points(ctx, tr, qx, qy, qz, nq, k, ctx.learned_feats, st);
    bound_model_predict(ctx, b, ctx.learned_feats, nq, inflation, nullptr, ctx.learned_bound, st);
    ft_query_options qb = q;
    qb.method           = FT_METHOD_FAST;
    knn(ctx, tr, qx, qy, qz, nq, k, max_k, idx, dist, qb, st, ctx.learned_bound);
}

// Features -> bound -> bounded fast walk; scratch grows in the context.
void self_knn_learned(Context &ctx, const ft_tree &tr, BoundModel &b, const int32_t *leaf_ids, size_t num, int k,
                      bool excl, float inflation, uint64_t *idx, void *dist, const ft_query_options &q,
                      cudaStream_t st) {
    if (num == 0 || k <= 0 || tr.num_leaves == 0) return;
    if (k > kMaxBoundK) fail(FT_ERR_INVALID_ARGUMENT, "learned bound: k must be in [1, 64]");
    ensure_learned(ctx, num);
    bound_features(ctx, tr, leaf_ids, num, k, ctx.learned_feats, st);
    bound_model_predict(ctx, b, ctx.learned_feats, num, inflation, nullptr, ctx.learned_bound, st);
    self_knn(ctx, tr, leaf_ids, num, k, excl, idx, dist, q, st, ctx.learned_bound);
}

} // namespace ft
