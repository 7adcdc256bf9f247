// ft_build.cu -- HLBVH build on sm_100a: bounding box, SFC keys, onesweep radix sort of
// (key, original index), leaf gather, Karras radix-tree topology and the bottom-up box refit
// that also writes the traversal's node records.
//
// Reference pipeline: build_bvh (src/hlbvh.hpp:2165-2290) -> compute_bbox (462-572) ->
// sfc_encode (357-423) -> oneDPL sort (2202-2232) -> gather (2266-2279) -> build_tree
// (773-982: Karras 861-903, refit 925-969).
#include <cuda_runtime.h>

#include <algorithm>
#include <climits>
#include <cstring>
#include <mutex>
#include <vector>

#include "ft_build_dev.cuh"
#include "ft_common.cuh"
#include "ft_internal.h"

namespace ft {

static constexpr int kSpinLimit = 1 << 24;

size_t coord_bytes(int coord) { return (coord == F32 || coord == U32) ? 4 : 8; }

static int key_words(const ft_options &o) { return (o.coord_type == U64) ? 2 : 1; }

// Karras tie-break / prefix flavour: 0 Morton (clz64), 1 63-bit PH (clz64 - 1), 2 126-bit PH.
static int delta_kind(const ft_options &o) {
    if (o.sfc_type == MORTON) return 0;
    return (o.coord_type == U64) ? 2 : 1;
}

size_t ref_key_bytes(const ft_options &o) {
    if (o.sfc_type == MORTON) return 8;       // uint64 (src/sfc.morton.hpp:17)
    return (o.coord_type == U64) ? 24 : 12;   // {hs,is,ls} of 64- or 32-bit words
}

// =========================================================================================
// Bounding box: per-block partials, then one block folds them (two passes keep the result
// independent of scheduling); the fold is bb_fold.
// =========================================================================================
static constexpr int kBboxBlocks = 1184; // 8 x 148 SMs

template <class T>
__global__ void __launch_bounds__(kBboxThreads) bbox_partial_kernel(const T *__restrict__ x, const T *__restrict__ y,
                                                                    const T *__restrict__ z, size_t n, T *partial) {
    T m[6];
    bb_identity(m);
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
        T v[6] = {x[i], x[i], y[i], y[i], z[i], z[i]};
        bb_fold(m, v);
    }
    bb_block_reduce(m);
    if (threadIdx.x == 0)
        for (int d = 0; d < 6; ++d) partial[blockIdx.x * 6 + d] = m[d];
}

template <class T> __global__ void __launch_bounds__(kBboxThreads) bbox_final_kernel(const T *partial, int nparts, T *out) {
    T m[6];
    bb_identity(m);
    for (int b = threadIdx.x; b < nparts; b += blockDim.x) bb_fold(m, partial + 6 * b);
    bb_block_reduce(m);
    if (threadIdx.x == 0)
        for (int d = 0; d < 6; ++d) out[d] = m[d];
}

// =========================================================================================
// SFC keys (sfc_encode, src/hlbvh.hpp:357-423).  Internal key format: lo (and hi for the
// 126-bit Peano-Hilbert key of 42-bit integer positions).  Also writes perm = iota.
// =========================================================================================
template <class T, int SFC>
__global__ void __launch_bounds__(256) encode_kernel(const T *__restrict__ x, const T *__restrict__ y,
                                                     const T *__restrict__ z, size_t n, const T *__restrict__ bbox,
                                                     unsigned long long *klo, unsigned long long *khi, uint32_t *perm) {
    using C = Coord<T>;
    __shared__ uint8_t s_rot[48 * 8], s_sub[48 * 8];
    __shared__ T       s_par[6]; // lo, inv per axis
    for (int i = threadIdx.x; i < 48 * 8; i += blockDim.x) {
        s_rot[i] = c_rot[i];
        s_sub[i] = c_sub[i];
    }
    if constexpr (C::is_float)
        if (threadIdx.x < 3) sfc_axis_params(bbox[2 * threadIdx.x], bbox[2 * threadIdx.x + 1], s_par[2 * threadIdx.x],
                                             s_par[2 * threadIdx.x + 1]);
    __syncthreads();
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
        unsigned long long hi, lo;
        encode_point<T, SFC>(x[i], y[i], z[i], s_par, s_rot, s_sub, hi, lo);
        klo[i] = lo;
        if (C::key_words == 2) khi[i] = hi;
        perm[i] = (uint32_t)i;
    }
}

// Key layout conversions between the reference's sfc_key and the internal (hi, lo) pair.
// mode 0: Morton uint64; 1: {hs,is,ls} uint32; 2: {hs,is,ls} uint64.
__global__ void keys_from_ref_kernel(const void *ref, size_t n, int mode, unsigned long long *klo,
                                     unsigned long long *khi, uint32_t *perm) {
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
        if (mode == 0) {
            klo[i] = ((const unsigned long long *)ref)[i];
        } else if (mode == 1) {
            const uint32_t *w = (const uint32_t *)ref + 3 * i;
            klo[i]            = ((unsigned long long)w[1] << 32) | w[2];
        } else {
            const unsigned long long *w = (const unsigned long long *)ref + 3 * i;
            khi[i]                      = w[1];
            klo[i]                      = w[2];
        }
        if (perm) perm[i] = (uint32_t)i;
    }
}

__global__ void keys_to_ref_kernel(const unsigned long long *klo, const unsigned long long *khi, size_t n, int mode,
                                   void *ref) {
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
        if (mode == 0) {
            ((unsigned long long *)ref)[i] = klo[i];
        } else if (mode == 1) {
            uint32_t *w = (uint32_t *)ref + 3 * i;
            w[0]        = 0;
            w[1]        = (uint32_t)(klo[i] >> 32);
            w[2]        = (uint32_t)klo[i];
        } else {
            unsigned long long *w = (unsigned long long *)ref + 3 * i;
            w[0]                  = 0;
            w[1]                  = khi[i];
            w[2]                  = klo[i];
        }
    }
}

// =========================================================================================
// Onesweep LSD radix sort of (key, perm): 8-bit digits, one upfront histogram pass for all
// digit positions, then one pass per non-constant digit.  Each pass: a tile of 256 threads x
// ITEMS keys ranks its keys with warp match-any histograms, publishes its digit counts,
// resolves its global offsets by decoupled look-back over preceding tiles (tiles are
// numbered by an atomic ticket so every predecessor is running or done), stages the tile
// in shared memory in digit order and writes each digit run contiguously.  Stable, so equal
// keys keep their original index order.
// =========================================================================================
static constexpr int kSortThreads = 256;
static constexpr int kSortWarps   = kSortThreads / 32;
// Tile tickets of build_bvh's sort: [0, 16) one per digit pass, [16, 32) the two-word
// fallback's passes; [32] the fallback switch (a long run of equal high words).
static constexpr int kTicketWords = 64;
static constexpr uint32_t kFlagAgg = 1u << 30, kFlagInc = 2u << 30, kFlagMask = 3u << 30,
                          kCountMask = (1u << 30) - 1u;

// A onesweep tile: 256 threads x ITEMS keys (ITEMS 0: the default, 8; the autotuner chose 8
// on every shape measured -- 100K float64 Morton, 10M and 50M uint64 Peano-Hilbert points --
// where the larger tiles' registers leave one block per SM: 10M points, untuned 12-key tiles
// 2.83 ms against 2.15 ms).  The build's sort takes the tile the autotuner chose for the shape
// (sort_items); every tile size gives the same order.
template <int W, int ITEMS = 0> struct SortCfg {
    static constexpr int items = ITEMS ? ITEMS : 8;
    static constexpr int tile  = kSortThreads * items;
    static constexpr size_t smem = (size_t)tile * (8 * W + 4) + (size_t)kSortWarps * 256 * 4;
};
static constexpr int kSortItemsMin = 8; // the smallest tile sizes the look-back scratch

// Digit histograms of digit positions [d0, d0 + ND) (ND = 8 * W by default: every digit).
// enable: null, or a device word whose 0 makes the launch a no-op.
template <int W, int ND = 8 * W>
__global__ void __launch_bounds__(256) radix_hist_kernel(const unsigned long long *__restrict__ klo,
                                                         const unsigned long long *__restrict__ khi, size_t n,
                                                         uint32_t *hist, int d0 = 0,
                                                         const uint32_t *enable = nullptr) {
    constexpr int D = ND;
    if (enable && *enable == 0u) return;
    __shared__ uint32_t s[D * 256];
    for (int i = threadIdx.x; i < D * 256; i += blockDim.x) s[i] = 0;
    __syncthreads();
    const unsigned lane = threadIdx.x & 31;
    const size_t   stride = (size_t)gridDim.x * blockDim.x;
    for (size_t base = blockIdx.x * (size_t)blockDim.x; base < n; base += stride) {
        size_t i     = base + threadIdx.x;
        bool   valid = i < n;
        unsigned long long w[2] = {valid ? klo[i] : 0ull, (W == 2 && valid) ? khi[i] : 0ull};
        unsigned active = __ballot_sync(0xffffffffu, valid);
#pragma unroll
        for (int j = 0; j < D; ++j) {
            const int d     = d0 + j;
            unsigned  digit = (unsigned)(w[d >> 3] >> (8 * (d & 7))) & 255u;
            unsigned peers = __match_any_sync(0xffffffffu, valid ? digit : 256u + lane);
            if (valid && lane == (unsigned)(__ffs(peers) - 1)) atomicAdd(&s[j * 256 + digit], __popc(peers & active));
        }
    }
    __syncthreads();
    for (int i = threadIdx.x; i < D * 256; i += blockDim.x)
        if (s[i]) atomicAdd(&hist[d0 * 256 + i], s[i]);
}

// Exclusive offsets per digit position; skip[d] = 1 when one digit value holds every key.
// enable: as radix_hist_kernel's.
__global__ void radix_scan_kernel(uint32_t *hist, size_t n, uint32_t *skip, const uint32_t *enable = nullptr) {
    __shared__ uint32_t s[256];
    __shared__ int      s_full;
    if (enable && *enable == 0u) return;
    const int d = blockIdx.x, t = threadIdx.x;
    uint32_t  c = hist[d * 256 + t];
    if (t == 0) s_full = 0;
    __syncthreads();
    if ((size_t)c == n) s_full = 1;
    s[t] = c;
    __syncthreads();
    for (int off = 1; off < 256; off <<= 1) {
        uint32_t v = (t >= off) ? s[t - off] : 0u;
        __syncthreads();
        s[t] += v;
        __syncthreads();
    }
    hist[d * 256 + t] = s[t] - c;
    if (t == 0) skip[d] = (uint32_t)s_full;
}

FT_D uint32_t ld_volatile(const uint32_t *p) {
    uint32_t v;
    asm volatile("ld.volatile.global.u32 %0, [%1];" : "=r"(v) : "l"(p));
    return v;
}
FT_D void st_volatile(uint32_t *p, uint32_t v) { asm volatile("st.volatile.global.u32 [%0], %1;" ::"l"(p), "r"(v)); }

// One onesweep pass over every tile.  The grid is persistent (at most the CTAs resident at
// once): each CTA takes tiles by ticket until none are left, so a launch whose pass turns out
// to have nothing to do costs one wave.  Device-side switches keep the host out of the loop:
//  * enable (null or a device word): 0 makes the whole pass a no-op (passes of the two-word
//    fallback, which only runs when a long run of equal high words was found);
//  * skip (null or a device word): 1 when one digit value holds every key -- the pass then
//    copies its tiles unchanged, so the ping-pong order the host planned still holds.
// (8-key tiles are compiled for three resident blocks: 80 registers, no spills, 24 warps per SM)
template <int W, int IT = 0>
__global__ void __launch_bounds__(kSortThreads, (SortCfg<W, IT>::items <= 8 ? 3 : 1))
    onesweep_kernel(const unsigned long long *__restrict__ in_lo, const unsigned long long *__restrict__ in_hi,
                    const uint32_t *__restrict__ in_v, unsigned long long *__restrict__ out_lo,
                    unsigned long long *__restrict__ out_hi, uint32_t *__restrict__ out_v, size_t n, size_t num_tiles,
                    int word, int shift, const uint32_t *__restrict__ offsets, uint32_t *lookback,
                    uint32_t *tile_counter, const uint32_t *enable, const uint32_t *skip, uint32_t *status) {
    using Cfg           = SortCfg<W, IT>;
    constexpr int ITEMS = Cfg::items;
    constexpr int TILE  = Cfg::tile;
    if (enable && *enable == 0u) return; // grid-uniform
    const bool copy = skip && *skip != 0u;
    extern __shared__ __align__(16) unsigned char smem[];
    unsigned long long *s_lo = reinterpret_cast<unsigned long long *>(smem);
    unsigned long long *s_hi = s_lo + TILE; // only used when W == 2
    uint32_t           *s_v  = reinterpret_cast<uint32_t *>(s_lo + (size_t)TILE * W);
    uint32_t           *s_wh = s_v + TILE; // [warp][256]
    __shared__ uint32_t s_tile_excl[256];
    __shared__ uint32_t s_base[256];
    __shared__ uint32_t s_ticket;
    __shared__ uint32_t s_wsum[kSortWarps];

    const int      tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const unsigned lt_mask = (1u << lane) - 1u;
    for (;;) {
        if (tid == 0) s_ticket = atomicAdd(tile_counter, 1u);
        for (int i = tid; i < kSortWarps * 256; i += kSortThreads) s_wh[i] = 0;
        __syncthreads();
        const size_t tile = s_ticket;
        if (tile >= num_tiles) break; // grid-uniform per CTA
        const size_t base = tile * (size_t)TILE;

        if (copy) { // constant digit: the tile moves unchanged
            const size_t end = min(base + (size_t)TILE, n);
            for (size_t pos = base + tid; pos < end; pos += kSortThreads) {
                out_lo[pos] = in_lo[pos];
                if (W == 2) out_hi[pos] = in_hi[pos];
                out_v[pos] = in_v[pos];
            }
            __syncthreads();
            continue;
        }

        unsigned long long klo[ITEMS], khi[ITEMS];
        uint32_t           val[ITEMS], dig[ITEMS], rank[ITEMS];
#pragma unroll
        for (int i = 0; i < ITEMS; ++i) {
            size_t pos   = base + (size_t)warp * 32 * ITEMS + (size_t)i * 32 + lane;
            bool   valid = pos < n;
            klo[i]       = valid ? in_lo[pos] : 0ull;
            khi[i]       = (W == 2 && valid) ? in_hi[pos] : 0ull;
            val[i]       = valid ? in_v[pos] : 0u;
            unsigned long long w = (W == 2 && word == 1) ? khi[i] : klo[i];
            dig[i]       = valid ? (uint32_t)(w >> shift) & 255u : 256u + lane;
        }
        uint32_t *wh = s_wh + warp * 256;
#pragma unroll
        for (int i = 0; i < ITEMS; ++i) {
            unsigned peers  = __match_any_sync(0xffffffffu, dig[i]);
            bool     valid  = dig[i] < 256u;
            uint32_t before = valid ? wh[dig[i]] : 0u;
            __syncwarp();
            if (valid && lane == __ffs(peers) - 1) wh[dig[i]] = before + __popc(peers);
            __syncwarp();
            rank[i] = before + __popc(peers & lt_mask);
        }
        __syncthreads();

        // per-digit: warp exclusive prefixes and the tile count
        uint32_t run = 0;
#pragma unroll
        for (int w = 0; w < kSortWarps; ++w) {
            uint32_t c          = s_wh[w * 256 + tid];
            s_wh[w * 256 + tid] = run;
            run += c;
        }
        const uint32_t tile_count = run;

        // exclusive scan of tile counts over digits (block scan, 256 threads)
        uint32_t incl = tile_count;
#pragma unroll
        for (int off = 1; off < 32; off <<= 1) {
            uint32_t v = __shfl_up_sync(0xffffffffu, incl, off);
            if (lane >= off) incl += v;
        }
        if (lane == 31) s_wsum[warp] = incl;
        __syncthreads();
        uint32_t wpre = 0;
        for (int w = 0; w < warp; ++w) wpre += s_wsum[w];
        s_tile_excl[tid] = wpre + incl - tile_count;

        // decoupled look-back for digit tid (every earlier tile is held by a running CTA or
        // done, since tickets are taken in order and a CTA finishes its tile first)
        uint32_t *lb     = lookback + tile * 256;
        uint32_t  prefix = 0;
        if (tile == 0) {
            st_volatile(lb + tid, kFlagInc | tile_count);
        } else {
            st_volatile(lb + tid, kFlagAgg | tile_count);
            for (long long j = (long long)tile - 1; j >= 0; --j) {
                uint32_t sv;
                int      spins = 0;
                for (;;) {
                    sv = ld_volatile(lookback + (size_t)j * 256 + tid);
                    if (sv & kFlagMask) break;
                    if (++spins > 64) __nanosleep(32);
                    if (spins > kSpinLimit) break;
                }
                if (!(sv & kFlagMask)) {
                    atomicOr(status, STATUS_SPIN_LIMIT);
                    break;
                }
                prefix += sv & kCountMask;
                if (sv & kFlagInc) break;
            }
            st_volatile(lb + tid, kFlagInc | (prefix + tile_count));
        }
        s_base[tid] = offsets[tid] + prefix;
        __syncthreads();

        // stage the tile in digit order
#pragma unroll
        for (int i = 0; i < ITEMS; ++i) {
            if (dig[i] < 256u) {
                uint32_t lp = s_tile_excl[dig[i]] + s_wh[warp * 256 + dig[i]] + rank[i];
                s_lo[lp]    = klo[i];
                if (W == 2) s_hi[lp] = khi[i];
                s_v[lp] = val[i];
            }
        }
        __syncthreads();
        const int tile_n = (int)min((size_t)TILE, n - base);
        for (int j = tid; j < tile_n; j += kSortThreads) {
            unsigned long long lo = s_lo[j];
            unsigned long long hi = (W == 2) ? s_hi[j] : 0ull;
            unsigned long long w  = (W == 2 && word == 1) ? hi : lo;
            uint32_t           d  = (uint32_t)(w >> shift) & 255u;
            size_t             gp = (size_t)s_base[d] + (size_t)(j - (int)s_tile_excl[d]);
            if (gp >= n) { // only reachable after a failed look-back; never write out of bounds
                atomicOr(status, STATUS_SPIN_LIMIT);
                continue;
            }
            out_lo[gp]             = lo;
            if (W == 2) out_hi[gp] = hi;
            out_v[gp]              = s_v[j];
        }
        __syncthreads(); // the tile's shared memory is free for the next ticket
    }
}

// =========================================================================================
// Leaf gather (src/hlbvh.hpp:2266-2279): leaf slot n-1+i <- input point perm[i].
// =========================================================================================
template <class T>
__global__ void gather_kernel(const T *__restrict__ x, const T *__restrict__ y, const T *__restrict__ z,
                              const uint32_t *__restrict__ perm, size_t n, const uint32_t *__restrict__ id,
                              const int8_t *__restrict__ ghost, T *mnx, T *mxx, T *mny, T *mxy, T *mnz, T *mxz,
                              uint32_t *tid_out, int8_t *ghost_out, int32_t *orig_out) {
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
        uint32_t src  = perm[i];
        size_t   leaf = i + n - 1;
        T        a = x[src], b = y[src], c = z[src];
        mnx[leaf] = a;
        mxx[leaf] = a;
        mny[leaf] = b;
        mxy[leaf] = b;
        mnz[leaf] = c;
        mxz[leaf] = c;
        tid_out[leaf]   = id ? id[src] : src;
        ghost_out[leaf] = ghost ? ghost[src] : (int8_t)0;
        orig_out[leaf]  = (int32_t)src;
    }
}

// Refit-only update: leaf slot n-1+i takes the new position of the point it already holds
// (input index orig_idx[n-1+i], or i itself when the positions come in leaf order).  An
// index outside [0, n) leaves the slot unchanged and sets the bad-input status bit.
template <class T>
__global__ void refit_gather_kernel(const T *__restrict__ x, const T *__restrict__ y, const T *__restrict__ z,
                                    const int32_t *__restrict__ orig, size_t n, T *mnx, T *mxx, T *mny, T *mxy,
                                    T *mnz, T *mxz, uint32_t *status) {
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
        const size_t  leaf = i + n - 1;
        const int64_t src  = orig ? (int64_t)orig[leaf] : (int64_t)i;
        if (src < 0 || src >= (int64_t)n) {
            atomicOr(status, STATUS_BAD_INPUT);
            continue;
        }
        const T a = x[src], b = y[src], c = z[src];
        mnx[leaf] = a;
        mxx[leaf] = a;
        mny[leaf] = b;
        mxy[leaf] = b;
        mnz[leaf] = c;
        mxz[leaf] = c;
    }
}

// Leaf init of build_tree with caller arrays (src/hlbvh.hpp:906-923).
template <class T>
__global__ void leaf_init_kernel(const T *sx, const T *sy, const T *sz, size_t n, const uint32_t *sid,
                                 const int8_t *sghost, const int32_t *sorig, T *mnx, T *mxx, T *mny, T *mxy,
                                 T *mnz, T *mxz, uint32_t *tid_out, int8_t *ghost_out, int32_t *orig_out) {
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
        size_t leaf = i + n - 1;
        mnx[leaf] = mxx[leaf] = sx[i];
        mny[leaf] = mxy[leaf] = sy[i];
        mnz[leaf] = mxz[leaf] = sz[i];
        if (sid) tid_out[leaf] = sid[i];
        if (sghost) ghost_out[leaf] = sghost[i];
        if (sorig) orig_out[leaf] = sorig[i];
    }
}

// =========================================================================================
// Karras 2012 radix-tree topology (src/hlbvh.hpp:852-903).  delta() is the common prefix
// length of two sorted keys (get_common_prefix_length, 283-340), with the index tie-break
// for equal keys.
// =========================================================================================
template <int KIND>
__global__ void __launch_bounds__(256) karras_kernel(const unsigned long long *__restrict__ klo,
                                                     const unsigned long long *__restrict__ khi, int n,
                                                     int32_t *left, int32_t *right, int32_t *parent,
                                                     int32_t *leaves) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n - 1; i += gridDim.x * blockDim.x)
        karras_node<KIND>(klo, khi, n, i, left, right, parent, leaves);
}

// =========================================================================================
// Bottom-up refit (src/hlbvh.hpp:925-969): climbs from the leaves, refit_step per level.
// =========================================================================================
// A climb ends at its first arrival at a node, so one thread per leaf (refit_leaf) leaves most
// lanes of a warp idle while its longest climb goes on (about 5 of 32 lanes active).  Here the
// warps of a grid of a few blocks per SM take leaves in chunks from a device counter (*work,
// zero at launch), and a lane whose climb ended takes the warp's next leaf: one climb step
// per lane and loop iteration.  The merges, boxes, records and heights are those of one climb
// per leaf (min / max do not depend on the order of the arrivals).
template <class T>
__global__ void __launch_bounds__(256) refit_stream_kernel(int n, const int32_t *__restrict__ left,
                                                           const int32_t *__restrict__ right,
                                                           const int32_t *__restrict__ parent, T *mnx, T *mxx,
                                                           T *mny, T *mxy, T *mnz, T *mxz, NodeRec<T> *recs,
                                                           uint8_t *height, int32_t *counters,
                                                           const int32_t *__restrict__ leaves, int32_t *work) {
    T *const       soa[6] = {mnx, mxx, mny, mxy, mnz, mxz};
    const unsigned FULL   = 0xffffffffu;
    const int      lane   = threadIdx.x & 31;
    constexpr int  kChunk = 256;
    int            next = 0, end = 0; // the warp's chunk of leaves [next, end) (warp-uniform)
    bool           more = true;       // the counter may still hold leaves (warp-uniform)
    int            curr = -1, steps = 0;
    for (;;) {
        // lanes without a climb take the chunk's next leaves, in lane order
        unsigned idle = __ballot_sync(FULL, curr < 0);
        while (idle && more) {
            if (next >= end) {
                int b = 0;
                if (lane == 0) b = atomicAdd(work, kChunk);
                b = __shfl_sync(FULL, b, 0);
                if (b >= n) {
                    more = false;
                    break;
                }
                next = b;
                end  = min(b + kChunk, n);
            }
            const int take = min(__popc(idle), end - next);
            const int rank = __popc(idle & ((1u << lane) - 1u));
            if (curr < 0 && rank < take) {
                curr  = next + rank + n - 1;
                steps = 0;
            }
            next += take;
            idle = __ballot_sync(FULL, curr < 0);
        }
        if (!__any_sync(FULL, curr >= 0)) break;
        if (curr >= 0) curr = ++steps < n ? refit_step<T>(curr, n, left, right, parent, soa, recs, height, counters,
                                                           leaves)
                                          : -1;
    }
}

// 4-wide records of every internal node (collapse_node), after the refit.
template <class T>
__global__ void __launch_bounds__(256) collapse_kernel(int n, const int32_t *__restrict__ left,
                                                       const int32_t *__restrict__ right, const T *mnx,
                                                       const T *mxx, const T *mny, const T *mxy, const T *mnz,
                                                       const T *mxz, WideRec<T> *wide) {
    const T *const soa[6] = {mnx, mxx, mny, mxy, mnz, mxz};
    for (int v = blockIdx.x * blockDim.x + threadIdx.x; v < n - 1; v += gridDim.x * blockDim.x)
        collapse_node<T>(v, n, left, right, soa, wide);
}

// =========================================================================================
// Host orchestration
// =========================================================================================
static int grid_for(size_t n, int threads, int max_blocks = 148 * 16) {
    size_t b = (n + threads - 1) / threads;
    if (b < 1) b = 1;
    return (int)std::min<size_t>(b, (size_t)max_blocks);
}

template <class T> static void *alloc_dev(size_t count) {
    void *p = nullptr;
    if (count == 0) count = 1;
    cudaError_t e = cudaMalloc(&p, count * sizeof(T));
    if (e != cudaSuccess) {
        cudaGetLastError();
        fail(FT_ERR_OUT_OF_MEMORY, "cudaMalloc of build scratch failed");
    }
    return p;
}

void free_scratch(TreeImpl &s) {
    void *ptrs[] = {s.recs, s.height, s.counters, s.leafcount, s.wide, s.key_lo, s.key_hi, s.tmp_lo, s.tmp_hi,
                    s.perm, s.tmp_perm, s.bbox, s.bbox_partial, s.hist, s.lookback, s.tile_counter, s.status};
    for (void *p : ptrs)
        if (p) cudaFree(p);
    int coord = s.coord;
    s         = TreeImpl{};
    s.coord   = coord;
}

static size_t sort_tiles(size_t n, int W) { // the most tiles any tile size makes
    (void)W;
    const size_t tile = (size_t)kSortThreads * kSortItemsMin;
    return (n + tile - 1) / tile;
}

void ensure_scratch(TreeImpl &s, const ft_options &o, size_t n) {
    if (n <= s.cap && s.key_lo) return;
    free_scratch(s);
    size_t cap = n + n / 2 + 1024;
    int    W   = key_words(o);
    size_t cb  = coord_bytes(o.coord_type);
    s.coord    = o.coord_type;
    s.cap      = cap;
    s.recs     = alloc_dev<unsigned char>((cap > 1 ? cap - 1 : 1) * 16 * cb);
    s.height   = (uint8_t *)alloc_dev<uint8_t>(cap);
    s.counters = (int32_t *)alloc_dev<int32_t>(cap);
    s.leafcount = (int32_t *)alloc_dev<int32_t>(cap);
    s.wide      = alloc_dev<unsigned char>((cap > 1 ? cap - 1 : 1) * wide_bytes(o.coord_type));
    s.key_lo   = (uint64_t *)alloc_dev<uint64_t>(cap);
    s.tmp_lo   = (uint64_t *)alloc_dev<uint64_t>(cap);
    if (W == 2) {
        s.key_hi = (uint64_t *)alloc_dev<uint64_t>(cap);
        s.tmp_hi = (uint64_t *)alloc_dev<uint64_t>(cap);
    }
    s.perm         = (uint32_t *)alloc_dev<uint32_t>(cap);
    s.tmp_perm     = (uint32_t *)alloc_dev<uint32_t>(cap);
    s.bbox         = alloc_dev<uint64_t>(6);
    s.bbox_partial = alloc_dev<uint64_t>((size_t)kBboxBlocks * 6);
    s.hist         = (uint32_t *)alloc_dev<uint32_t>(16 * 256 + 16);
    s.lookback_words = 16 * sort_tiles(cap, W) * 256;
    s.lookback     = (uint32_t *)alloc_dev<uint32_t>(s.lookback_words);
    s.tile_counter = (uint32_t *)alloc_dev<uint32_t>(kTicketWords);
    s.status       = (uint32_t *)alloc_dev<uint32_t>(4);
    FT_CUDA(cudaMemset(s.status, 0, 16));
}

template <class T>
static void bbox_typed(const void *x, const void *y, const void *z, size_t n, void *partial, void *out,
                       cudaStream_t st) {
    int blocks = grid_for(n, kBboxThreads, kBboxBlocks);
    bbox_partial_kernel<T><<<blocks, kBboxThreads, 0, st>>>((const T *)x, (const T *)y, (const T *)z, n, (T *)partial);
    bbox_final_kernel<T><<<1, kBboxThreads, 0, st>>>((const T *)partial, blocks, (T *)out);
    FT_CUDA(cudaGetLastError());
}

void compute_bbox(Context &ctx, TreeImpl *scratch, const void *x, const void *y, const void *z, size_t n,
                  void *bbox_dev, cudaStream_t st) {
    void *partial = scratch->bbox_partial;
    switch (ctx.opts.coord_type) {
    case F32: bbox_typed<float>(x, y, z, n, partial, bbox_dev, st); break;
    case F64: bbox_typed<double>(x, y, z, n, partial, bbox_dev, st); break;
    case U32: bbox_typed<uint32_t>(x, y, z, n, partial, bbox_dev, st); break;
    case U64: bbox_typed<unsigned long long>(x, y, z, n, partial, bbox_dev, st); break;
    }
}

template <class T>
static void encode_typed(const ft_options &o, const void *x, const void *y, const void *z, size_t n,
                         const void *bbox, TreeImpl &s, cudaStream_t st) {
    int blocks = grid_for(n, 256);
    if (o.sfc_type == MORTON)
        encode_kernel<T, MORTON><<<blocks, 256, 0, st>>>((const T *)x, (const T *)y, (const T *)z, n,
                                                         (const T *)bbox, (unsigned long long *)s.key_lo,
                                                         (unsigned long long *)s.key_hi, s.perm);
    else
        encode_kernel<T, PEANO_HILBERT><<<blocks, 256, 0, st>>>((const T *)x, (const T *)y, (const T *)z, n,
                                                                (const T *)bbox, (unsigned long long *)s.key_lo,
                                                                (unsigned long long *)s.key_hi, s.perm);
    FT_CUDA(cudaGetLastError());
}

static void encode(const ft_options &o, const void *x, const void *y, const void *z, size_t n, const void *bbox,
                   TreeImpl &s, cudaStream_t st) {
    switch (o.coord_type) {
    case F32: encode_typed<float>(o, x, y, z, n, bbox, s, st); break;
    case F64: encode_typed<double>(o, x, y, z, n, bbox, s, st); break;
    case U32: encode_typed<uint32_t>(o, x, y, z, n, bbox, s, st); break;
    case U64: encode_typed<unsigned long long>(o, x, y, z, n, bbox, s, st); break;
    }
}

static int ref_key_mode(const ft_options &o) {
    if (o.sfc_type == MORTON) return 0;
    return (o.coord_type == U64) ? 2 : 1;
}

void sfc_encode_ref_layout(Context &ctx, TreeImpl &s, const void *x, const void *y, const void *z, size_t n,
                           const void *bbox_dev, void *keys_ref_dev, cudaStream_t st) {
    encode(ctx.opts, x, y, z, n, bbox_dev, s, st);
    keys_to_ref_kernel<<<grid_for(n, 256), 256, 0, st>>>((const unsigned long long *)s.key_lo,
                                                          (const unsigned long long *)s.key_hi, n,
                                                          ref_key_mode(ctx.opts), keys_ref_dev);
    FT_CUDA(cudaGetLastError());
}

// Two-word keys, second stage: after the passes over the high word, runs of equal high
// words are put in (low word, input index) order.  The thread at the start of each run
// insertion-sorts it in place when it holds at most kRunCap keys (stable, so equal keys keep
// the index order the high-word passes left); a longer run sets flag[0], which switches on
// the low-word and high-word passes queued behind this kernel.
static constexpr int kRunCap = 32;

__global__ void __launch_bounds__(256) hi_run_fixup_kernel(unsigned long long *__restrict__ klo,
                                                           const unsigned long long *__restrict__ khi,
                                                           uint32_t *__restrict__ perm, size_t n, uint32_t *flag) {
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i + 1 < n; i += (size_t)gridDim.x * blockDim.x) {
        const unsigned long long h = khi[i];
        if (khi[i + 1] != h || (i > 0 && khi[i - 1] == h)) continue; // not the start of a run
        size_t e = i + 2;
        while (e < n && e - i <= (size_t)kRunCap && khi[e] == h) ++e;
        if (e - i > (size_t)kRunCap) {
            atomicOr(flag, 1u);
            continue;
        }
        for (size_t j = i + 1; j < e; ++j) {
            const unsigned long long kl = klo[j];
            const uint32_t           pv = perm[j];
            size_t                   m  = j;
            while (m > i && klo[m - 1] > kl) {
                klo[m]  = klo[m - 1];
                perm[m] = perm[m - 1];
                --m;
            }
            klo[m]  = kl;
            perm[m] = pv;
        }
    }
}

// Zeroes `words` words at p when *enable is set (the fallback's look-back status words).
__global__ void __launch_bounds__(256) zero_if_kernel(uint32_t *p, size_t words, const uint32_t *enable) {
    if (*enable == 0u) return;
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < words; i += (size_t)gridDim.x * blockDim.x)
        p[i] = 0u;
}

// Persistent grid of a onesweep pass: the CTAs resident at once (three per SM with the
// tile's shared memory), never more than the tiles.
template <int W, int IT = 0> static unsigned sort_grid(size_t tiles) {
    static int per_sm = 0, sms = 0;
    static std::once_flag once;
    std::call_once(once, [] {
        int dev = 0;
        if (cudaGetDevice(&dev) != cudaSuccess ||
            cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess ||
            cudaFuncSetAttribute(onesweep_kernel<W, IT>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)SortCfg<W, IT>::smem) != cudaSuccess ||
            cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, onesweep_kernel<W, IT>, kSortThreads,
                                                          SortCfg<W, IT>::smem) != cudaSuccess) {
            cudaGetLastError();
            per_sm = 1;
            sms    = 148;
        }
        per_sm = std::max(per_sm, 1);
    });
    return (unsigned)std::max<size_t>(1, std::min<size_t>(tiles, (size_t)per_sm * (size_t)sms));
}

// The key sort of build_bvh, with no host synchronisation.  One-word keys: histograms of the
// eight digits, then eight passes (a constant digit's pass copies).  Two-word keys: the
// high word's eight passes, then runs of equal high words of at most 32 keys are ordered by
// (low word, input index) in place; a longer run switches on, on the device, the full
// two-word sort from that order (histograms of the low word, then the eight low-word and the
// eight high-word passes: an even number, so the host's ping-pong order is the same whether
// they run or not).
template <int W, int IT = 0> static void sort_impl(TreeImpl &s, size_t n, cudaStream_t st) {
    using Cfg            = SortCfg<W, IT>;
    const int      D     = 8 * W;
    const size_t   tiles = (n + Cfg::tile - 1) / Cfg::tile;
    const unsigned grid  = sort_grid<W, IT>(tiles);
    FT_CUDA(cudaFuncSetAttribute(onesweep_kernel<W, IT>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)Cfg::smem));
    FT_CUDA(cudaMemsetAsync(s.hist, 0, (16 * 256 + 16) * sizeof(uint32_t), st));
    FT_CUDA(cudaMemsetAsync(s.tile_counter, 0, kTicketWords * sizeof(uint32_t), st));
    uint32_t *skip_dev = s.hist + 16 * 256;
    uint32_t *fallback = s.tile_counter + 32;
    // histograms of the digit positions [d0, d0 + 8) of one key word
    auto histogram = [&](int d0, const uint32_t *enable) {
        radix_hist_kernel<W, 8><<<grid_for(n, 256, 148 * 4), 256, 0, st>>>(
            (const unsigned long long *)s.key_lo, (const unsigned long long *)s.key_hi, n, s.hist, d0, enable);
        radix_scan_kernel<<<8, 256, 0, st>>>(s.hist + d0 * 256, n, skip_dev + d0, enable);
        FT_CUDA(cudaGetLastError());
    };
    auto pass = [&](int d, uint32_t *ticket, const uint32_t *enable) {
        onesweep_kernel<W, IT><<<grid, kSortThreads, Cfg::smem, st>>>(
            (const unsigned long long *)s.key_lo, (const unsigned long long *)s.key_hi, s.perm,
            (unsigned long long *)s.tmp_lo, (unsigned long long *)s.tmp_hi, s.tmp_perm, n, tiles, d >> 3,
            8 * (d & 7), s.hist + d * 256, s.lookback + (size_t)d * tiles * 256, ticket, enable, skip_dev + d,
            s.status);
        FT_CUDA(cudaGetLastError());
        std::swap(s.key_lo, s.tmp_lo);
        std::swap(s.key_hi, s.tmp_hi);
        std::swap(s.perm, s.tmp_perm);
    };
    histogram(W == 2 ? 8 : 0, nullptr);
    FT_CUDA(cudaMemsetAsync(s.lookback, 0, (size_t)D * tiles * 256 * sizeof(uint32_t), st));
    if constexpr (W == 1) {
        for (int d = 0; d < 8; ++d) pass(d, s.tile_counter + d, nullptr);
    } else {
        // high-word passes first; equal high words are rare for data spread over the box (a
        // 62-bit prefix of the curve), so a fix-up of their short runs replaces the low-word
        // passes
        for (int d = 8; d < 16; ++d) pass(d, s.tile_counter + d, nullptr);
        hi_run_fixup_kernel<<<grid_for(n, 256), 256, 0, st>>>((unsigned long long *)s.key_lo,
                                                              (const unsigned long long *)s.key_hi, s.perm, n,
                                                              fallback);
        FT_CUDA(cudaGetLastError());
        // a long run of equal high words: the full two-word sort from the current order (it is
        // stable, and within equal keys the current order is the input index order)
        histogram(0, fallback);
        zero_if_kernel<<<grid_for((size_t)D * tiles * 256, 256, 148 * 8), 256, 0, st>>>(
            s.lookback, (size_t)D * tiles * 256, fallback);
        FT_CUDA(cudaGetLastError());
        for (int d = 0; d < 16; ++d) pass(d, s.tile_counter + 16 + d, fallback);
    }
}

// The same sort over a fixed list of digit positions (every listed pass runs; no skips and no
// fallback), used by the batched build and the query order.
template <int W> static void sort_fixed_impl(TreeImpl &s, size_t n, int ndig, const int *digits, cudaStream_t st) {
    using Cfg            = SortCfg<W>;
    const int      D     = 8 * W;
    const size_t   tiles = (n + Cfg::tile - 1) / Cfg::tile;
    const unsigned grid  = sort_grid<W>(tiles);
    FT_CUDA(cudaMemsetAsync(s.hist, 0, (16 * 256 + 16) * sizeof(uint32_t), st));
    radix_hist_kernel<W><<<grid_for(n, 256, 148 * 4), 256, 0, st>>>((const unsigned long long *)s.key_lo,
                                                                      (const unsigned long long *)s.key_hi, n,
                                                                      s.hist);
    radix_scan_kernel<<<D, 256, 0, st>>>(s.hist, n, s.hist + 16 * 256);
    FT_CUDA(cudaGetLastError());
    FT_CUDA(cudaMemsetAsync(s.lookback, 0, (size_t)D * tiles * 256 * sizeof(uint32_t), st));
    FT_CUDA(cudaMemsetAsync(s.tile_counter, 0, 16 * sizeof(uint32_t), st));
    FT_CUDA(cudaFuncSetAttribute(onesweep_kernel<W>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)Cfg::smem));
    for (int i = 0; i < ndig; ++i) {
        const int d = digits[i];
        onesweep_kernel<W><<<grid, kSortThreads, Cfg::smem, st>>>(
            (const unsigned long long *)s.key_lo, (const unsigned long long *)s.key_hi, s.perm,
            (unsigned long long *)s.tmp_lo, (unsigned long long *)s.tmp_hi, s.tmp_perm, n, tiles, d >> 3, 8 * (d & 7),
            s.hist + d * 256, s.lookback + (size_t)d * tiles * 256, s.tile_counter + d, nullptr, nullptr, s.status);
        FT_CUDA(cudaGetLastError());
        std::swap(s.key_lo, s.tmp_lo);
        std::swap(s.key_hi, s.tmp_hi);
        std::swap(s.perm, s.tmp_perm);
    }
}

void sort_pairs_fixed(TreeImpl &s, size_t n, int words, int ndigits, const int *digits, cudaStream_t st) {
    if (n < 2 || ndigits <= 0) return;
    if (words == 1) sort_fixed_impl<1>(s, n, ndigits, digits, st);
    else sort_fixed_impl<2>(s, n, ndigits, digits, st);
}

size_t sort_lookback_words(size_t n, int words) { return 16 * sort_tiles(n, words) * 256; }

// items: keys per thread of a onesweep tile (0: the default for the key width).
static void sort_keys(const ft_options &o, TreeImpl &s, size_t n, cudaStream_t st, int items = 0) {
    if (n < 2) return;
    if (key_words(o) == 1) {
        switch (items) {
        case 12: sort_impl<1, 12>(s, n, st); break;
        case 16: sort_impl<1, 16>(s, n, st); break;
        case 20: sort_impl<1, 20>(s, n, st); break;
        default: sort_impl<1>(s, n, st); break; // 8
        }
    } else {
        switch (items) {
        case 12: sort_impl<2, 12>(s, n, st); break;
        case 16: sort_impl<2, 16>(s, n, st); break;
        default: sort_impl<2>(s, n, st); break; // 8
        }
    }
}

const int *sort_item_choices(int words, int *count) {
    static const int one[4] = {8, 12, 16, 20}, two[3] = {8, 12, 16}; // the default first
    *count = words == 1 ? 4 : 3;
    return words == 1 ? one : two;
}

template <class T> struct SoA {
    T *mnx, *mxx, *mny, *mxy, *mnz, *mxz;
    explicit SoA(const ft_tree &t)
        : mnx((T *)t.min_x), mxx((T *)t.max_x), mny((T *)t.min_y), mxy((T *)t.max_y), mnz((T *)t.min_z),
          mxz((T *)t.max_z) {}
};

template <class T>
static void topology_and_refit(const ft_options &o, ft_tree &t, TreeImpl &s, size_t n, cudaStream_t st,
                               Context *prof = nullptr) {
    if (n < 2) {
        s.height_root = 0;
        stage_mark(prof, BS_TOPOLOGY, st);
        stage_mark(prof, BS_REFIT, st);
        stage_mark(prof, BS_RECORDS, st);
        return;
    }
    FT_CUDA(cudaMemsetAsync(t.parent, 0xFF, (2 * n - 1) * sizeof(int32_t), st)); // -1 (849)
    int blocks = grid_for(n, 256, 148 * 32);
    const unsigned long long *lo = (const unsigned long long *)s.key_lo, *hi = (const unsigned long long *)s.key_hi;
    switch (delta_kind(o)) {
    case 0: karras_kernel<0><<<blocks, 256, 0, st>>>(lo, hi, (int)n, t.left_child, t.right_child, t.parent, s.leafcount); break;
    case 1: karras_kernel<1><<<blocks, 256, 0, st>>>(lo, hi, (int)n, t.left_child, t.right_child, t.parent, s.leafcount); break;
    default: karras_kernel<2><<<blocks, 256, 0, st>>>(lo, hi, (int)n, t.left_child, t.right_child, t.parent, s.leafcount); break;
    }
    FT_CUDA(cudaGetLastError());
    stage_mark(prof, BS_TOPOLOGY, st);
    // arrival counters of the n - 1 internal nodes, then the streaming refit's leaf counter
    FT_CUDA(cudaMemsetAsync(s.counters, 0, n * sizeof(int32_t), st));
    SoA<T> a(t);
    refit_stream_kernel<T><<<grid_for(n, 256, 148 * 8), 256, 0, st>>>(
        (int)n, t.left_child, t.right_child, t.parent, a.mnx, a.mxx, a.mny, a.mxy, a.mnz, a.mxz,
        (NodeRec<T> *)s.recs, s.height, s.counters, s.leafcount, s.counters + (n - 1));
    stage_mark(prof, BS_REFIT, st);
    collapse_kernel<T><<<blocks, 256, 0, st>>>((int)n, t.left_child, t.right_child, a.mnx, a.mxx, a.mny, a.mxy,
                                               a.mnz, a.mxz, (WideRec<T> *)s.wide);
    FT_CUDA(cudaGetLastError());
    stage_mark(prof, BS_RECORDS, st);
}

template <class T>
static void build_bvh_typed(Context &ctx, ft_tree &t, const void *x, const void *y, const void *z, size_t n,
                            const uint32_t *id, const int8_t *ghost, const void *bbox_host, void *caller_keys,
                            cudaStream_t st, int sort_items) {
    TreeImpl &s = *(TreeImpl *)t.impl;
    ensure_scratch(s, ctx.opts, n);
    stage_mark(&ctx, BS_START, st);
    // 1. bounding box.  Only the float encode reads it; integer encoding ignores it, so an
    // integer tree always keeps its true box (the query distance mode depends on it).
    if (bbox_host && Coord<T>::is_float)
        FT_CUDA(cudaMemcpyAsync(s.bbox, bbox_host, 6 * sizeof(T), cudaMemcpyHostToDevice, st));
    else compute_bbox(ctx, &s, x, y, z, n, s.bbox, st);
    stage_mark(&ctx, BS_BBOX, st);
    // 2. keys + iota permutation
    if (caller_keys) {
        keys_from_ref_kernel<<<grid_for(n, 256), 256, 0, st>>>(caller_keys, n, ref_key_mode(ctx.opts),
                                                               (unsigned long long *)s.key_lo,
                                                               (unsigned long long *)s.key_hi, s.perm);
        FT_CUDA(cudaGetLastError());
    } else {
        encode(ctx.opts, x, y, z, n, s.bbox, s, st);
    }
    stage_mark(&ctx, BS_ENCODE, st);
    // 3. sort (key, perm), with the tile the autotuner chose for this shape
    if (sort_items <= 0) {
        auto it = ctx.tuned.find(tune_key(TUNE_BUILD, key_words(ctx.opts), n));
        if (it != ctx.tuned.end()) sort_items = it->second.items;
    }
    sort_keys(ctx.opts, s, n, st, sort_items);
    stage_mark(&ctx, BS_SORT, st);
    if (caller_keys) {
        keys_to_ref_kernel<<<grid_for(n, 256), 256, 0, st>>>((const unsigned long long *)s.key_lo,
                                                              (const unsigned long long *)s.key_hi, n,
                                                              ref_key_mode(ctx.opts), caller_keys);
        FT_CUDA(cudaGetLastError());
    }
    // 4. gather into leaf slots; internal slots of id / is_ghost / orig_idx are zeroed
    SoA<T> a(t);
    if (n > 1) {
        FT_CUDA(cudaMemsetAsync(t.id, 0, (n - 1) * sizeof(uint32_t), st));
        FT_CUDA(cudaMemsetAsync(t.is_ghost, 0, (n - 1) * sizeof(int8_t), st));
        FT_CUDA(cudaMemsetAsync(t.orig_idx, 0, (n - 1) * sizeof(int32_t), st));
    }
    gather_kernel<T><<<grid_for(n, 256), 256, 0, st>>>((const T *)x, (const T *)y, (const T *)z, s.perm, n, id, ghost,
                                                       a.mnx, a.mxx, a.mny, a.mxy, a.mnz, a.mxz, t.id, t.is_ghost,
                                                       t.orig_idx);
    FT_CUDA(cudaGetLastError());
    if (n == 1) FT_CUDA(cudaMemsetAsync(t.parent, 0xFF, sizeof(int32_t), st));
    stage_mark(&ctx, BS_GATHER, st);
    // 5. topology + refit
    topology_and_refit<T>(ctx.opts, t, s, n, st, &ctx);
    ctx.bprof.recorded = ctx.bprof.on;
}

void build_bvh(Context &ctx, ft_tree &t, const void *x, const void *y, const void *z, size_t n, const uint32_t *id,
               const int8_t *ghost, const void *bbox_host, void *caller_keys, cudaStream_t st, int sort_items) {
    switch (ctx.opts.coord_type) {
    case F32: build_bvh_typed<float>(ctx, t, x, y, z, n, id, ghost, bbox_host, caller_keys, st, sort_items); break;
    case F64: build_bvh_typed<double>(ctx, t, x, y, z, n, id, ghost, bbox_host, caller_keys, st, sort_items); break;
    case U32: build_bvh_typed<uint32_t>(ctx, t, x, y, z, n, id, ghost, bbox_host, caller_keys, st, sort_items); break;
    case U64: build_bvh_typed<unsigned long long>(ctx, t, x, y, z, n, id, ghost, bbox_host, caller_keys, st, sort_items); break;
    }
}

int key_words_of(const ft_options &o) { return key_words(o); }

template <class T>
static void build_tree_typed(Context &ctx, ft_tree &t, const void *keys_ref, const void *sx, const void *sy,
                             const void *sz, const uint32_t *sid, const int8_t *sghost, const int32_t *sorig,
                             cudaStream_t st) {
    TreeImpl &s = *(TreeImpl *)t.impl;
    size_t    n = t.num_leaves;
    ensure_scratch(s, ctx.opts, n);
    keys_from_ref_kernel<<<grid_for(n, 256), 256, 0, st>>>(keys_ref, n, ref_key_mode(ctx.opts),
                                                           (unsigned long long *)s.key_lo,
                                                           (unsigned long long *)s.key_hi, nullptr);
    FT_CUDA(cudaGetLastError());
    SoA<T> a(t);
    if (sx && sy && sz)
        leaf_init_kernel<T><<<grid_for(n, 256), 256, 0, st>>>((const T *)sx, (const T *)sy, (const T *)sz, n, sid,
                                                              sghost, sorig, a.mnx, a.mxx, a.mny, a.mxy, a.mnz,
                                                              a.mxz, t.id, t.is_ghost, t.orig_idx);
    FT_CUDA(cudaGetLastError());
    if (n == 1) FT_CUDA(cudaMemsetAsync(t.parent, 0xFF, sizeof(int32_t), st));
    topology_and_refit<T>(ctx.opts, t, s, n, st);
}

// Refit-only update of a built tree (no reference counterpart: the reference rebuilds).  The
// keys, leaf order and topology stay; the leaves take the new positions and the bottom-up
// refit recomputes every internal box, the node records, heights and 4-wide records.  The
// result is the tree build_tree (src/hlbvh.hpp:773-982) makes from the same sorted keys with
// the new positions as its leaf arrays.
template <class T>
static void refit_typed(ft_tree &t, const void *x, const void *y, const void *z, size_t n, bool leaf_order,
                        cudaStream_t st) {
    TreeImpl &s = *(TreeImpl *)t.impl;
    SoA<T>    a(t);
    refit_gather_kernel<T><<<grid_for(n, 256), 256, 0, st>>>((const T *)x, (const T *)y, (const T *)z,
                                                             leaf_order ? nullptr : t.orig_idx, n, a.mnx, a.mxx,
                                                             a.mny, a.mxy, a.mnz, a.mxz, s.status);
    FT_CUDA(cudaGetLastError());
    if (n < 2) return;
    const int blocks = grid_for(n, 256, 148 * 32);
    FT_CUDA(cudaMemsetAsync(s.counters, 0, n * sizeof(int32_t), st));
    refit_stream_kernel<T><<<grid_for(n, 256, 148 * 8), 256, 0, st>>>(
        (int)n, t.left_child, t.right_child, t.parent, a.mnx, a.mxx, a.mny, a.mxy, a.mnz, a.mxz,
        (NodeRec<T> *)s.recs, s.height, s.counters, s.leafcount, s.counters + (n - 1));
    collapse_kernel<T><<<blocks, 256, 0, st>>>((int)n, t.left_child, t.right_child, a.mnx, a.mxx, a.mny, a.mxy,
                                               a.mnz, a.mxz, (WideRec<T> *)s.wide);
    FT_CUDA(cudaGetLastError());
}

void refit_bvh(Context &ctx, ft_tree &t, const void *x, const void *y, const void *z, size_t n, bool leaf_order,
               cudaStream_t st) {
    switch (ctx.opts.coord_type) {
    case F32: refit_typed<float>(t, x, y, z, n, leaf_order, st); break;
    case F64: refit_typed<double>(t, x, y, z, n, leaf_order, st); break;
    case U32: refit_typed<uint32_t>(t, x, y, z, n, leaf_order, st); break;
    case U64: refit_typed<unsigned long long>(t, x, y, z, n, leaf_order, st); break;
    }
}

// Topology, internal boxes, node records, heights and 4-wide records recomputed from the
// tree's sorted keys and leaf slots (an imported tree).
void recompute_from_keys(Context &ctx, ft_tree &t, cudaStream_t st) {
    TreeImpl &s = *(TreeImpl *)t.impl;
    size_t    n = t.num_leaves;
    switch (ctx.opts.coord_type) {
    case F32: topology_and_refit<float>(ctx.opts, t, s, n, st); break;
    case F64: topology_and_refit<double>(ctx.opts, t, s, n, st); break;
    case U32: topology_and_refit<uint32_t>(ctx.opts, t, s, n, st); break;
    case U64: topology_and_refit<unsigned long long>(ctx.opts, t, s, n, st); break;
    }
}

void build_tree_from_keys(Context &ctx, ft_tree &t, const void *keys_ref, const void *sx, const void *sy,
                          const void *sz, const uint32_t *sid, const int8_t *sghost, const int32_t *sorig,
                          cudaStream_t st) {
    switch (ctx.opts.coord_type) {
    case F32: build_tree_typed<float>(ctx, t, keys_ref, sx, sy, sz, sid, sghost, sorig, st); break;
    case F64: build_tree_typed<double>(ctx, t, keys_ref, sx, sy, sz, sid, sghost, sorig, st); break;
    case U32: build_tree_typed<uint32_t>(ctx, t, keys_ref, sx, sy, sz, sid, sghost, sorig, st); break;
    case U64: build_tree_typed<unsigned long long>(ctx, t, keys_ref, sx, sy, sz, sid, sghost, sorig, st); break;
    }
}

} // namespace ft
