// ft_cta_build.cuh -- one thread block builds one point set's whole tree: the per-set body of
// the persistent batched launch (ft_batch_build_knn with FT_BATCH_PERSISTENT).
//
// The steps and their results are those of build_bvh on the set alone (src/hlbvh.hpp:
// 2165-2290): the set's bounding box (462-572), its SFC keys (357-423), the keys sorted with
// their input indices (2202-2232; equal keys in input order), the leaf gather (2266-2279),
// the Karras topology (861-903) and the bottom-up refit (925-969) -- here one agglomerative
// climb that yields the same tree, numbering and boxes -- then this library's 4-wide
// records.  Only the schedule differs: every step runs inside the block, with block barriers
// between them, over the set's slice of the batch's arrays.  The key sort is a stable LSD
// radix sort over 8-bit digits whose tiles the block takes in order, so a tile's place in
// the output follows from the running digit offsets -- no look-back between blocks.
#pragma once

#include "ft_build_dev.cuh"
#include "ft_common.cuh"

namespace ft {

// ---- order-preserving unsigned images of coordinates (atomic min / max of set boxes) ----
template <class T> struct Ord;
template <> struct Ord<float> {
    using type = unsigned int;
    static FT_D type bits(float f) {
        unsigned int u = __float_as_uint(f);
        return (u & 0x80000000u) ? ~u : (u | 0x80000000u);
    }
    static FT_D float value(type u) { return __uint_as_float((u & 0x80000000u) ? (u & 0x7fffffffu) : ~u); }
};
template <> struct Ord<double> {
    using type = unsigned long long;
    static FT_D type bits(double f) {
        unsigned long long u = (unsigned long long)__double_as_longlong(f);
        return (u >> 63) ? ~u : (u | 0x8000000000000000ull);
    }
    static FT_D double value(type u) {
        return __longlong_as_double((long long)((u >> 63) ? (u & 0x7fffffffffffffffull) : ~u));
    }
};
template <> struct Ord<uint32_t> {
    using type = unsigned int;
    static FT_D type     bits(uint32_t v) { return v; }
    static FT_D uint32_t value(type u) { return u; }
};
template <> struct Ord<unsigned long long> {
    using type = unsigned long long;
    static FT_D type               bits(unsigned long long v) { return v; }
    static FT_D unsigned long long value(type u) { return u; }
};

// Where one block writes one set's tree: the set's slices of the batch's arrays.
template <class T> struct CtaTreeOut {
    T          *mnx, *mxx, *mny, *mxy, *mnz, *mxz; // node boxes (2n - 1 slots from node_off)
    int32_t    *left, *right, *parent;            // internal slots from rec_off; parent per node
    uint32_t   *id;
    int8_t     *ghost;
    int32_t    *orig;
    NodeRec<T> *recs;
    WideRec<T> *wide;
    uint8_t    *height;
    int32_t    *counters, *leaves;
};

// Exclusive prefix sums of a[0..256) in place, by the block's first warp (8 entries a lane).
FT_D void cta_scan256(uint32_t *a) {
    if (threadIdx.x < 32) {
        const int lane = threadIdx.x;
        uint32_t  v[8], sum = 0;
#pragma unroll
        for (int i = 0; i < 8; ++i) {
            v[i] = a[lane * 8 + i];
            sum += v[i];
        }
        uint32_t incl = sum;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const uint32_t u = __shfl_up_sync(0xffffffffu, incl, o);
            if (lane >= o) incl += u;
        }
        uint32_t run = incl - sum;
#pragma unroll
        for (int i = 0; i < 8; ++i) {
            a[lane * 8 + i] = run;
            run += v[i];
        }
    }
}

// Dynamic shared memory of a block's set build (bytes): the sort's tile staging, its per-warp
// digit counts and three 256-entry digit tables, then the Peano-Hilbert tables.  The build
// keeps almost nothing in static shared memory, so that the query phase's blocks, whose
// heaps reuse this region, pack as densely as the standalone walk's.
template <int KW, int PT, int ITEMS> constexpr size_t cta_sort_bytes() {
    return (size_t)PT * ITEMS * (8 * KW + 4) + (size_t)(PT / 32) * 256 * 4 + 3 * 256 * 4;
}
template <int KW, int PT, int ITEMS> constexpr size_t cta_sort_smem() {
    return cta_sort_bytes<KW, PT, ITEMS>() + 2 * 48 * 8;
}

// Stable LSD radix sort of (key, value) pairs [0, n) by one block of PT threads: 8-bit digits
// of the low word, then (KW == 2) of the high word, so the order is (high, low) with equal
// keys in their incoming order.  Ping-pong between the A and B buffers; a digit that is the
// same for every key is skipped.  Returns true when the sorted pairs end in B.
template <int KW, int PT, int ITEMS>
FT_D bool cta_sort(unsigned long long *alo, unsigned long long *ahi, uint32_t *av, unsigned long long *blo,
                   unsigned long long *bhi, uint32_t *bv, int n, unsigned char *smem) {
    constexpr int  WARPS = PT / 32, TILE = PT * ITEMS;
    const unsigned FULL  = 0xffffffffu;
    unsigned long long *s_lo = reinterpret_cast<unsigned long long *>(smem);
    unsigned long long *s_hi = s_lo + TILE; // KW == 2 only
    uint32_t           *s_v  = reinterpret_cast<uint32_t *>(s_lo + (size_t)TILE * KW);
    uint32_t           *s_wh = s_v + TILE; // [warp][digit] running counts within a tile
    uint32_t           *s_off = s_wh + WARPS * 256, *s_excl = s_off + 256, *s_cnt = s_excl + 256;
    __shared__ int      s_skip;
    const int      tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const unsigned lt_mask = (1u << lane) - 1u;
    bool           in_b    = false;
    for (int pass = 0; pass < 8 * KW; ++pass) {
        const int                 word = pass >> 3, shift = 8 * (pass & 7);
        const unsigned long long *ilo = in_b ? blo : alo, *ihi = in_b ? bhi : ahi;
        const uint32_t           *iv  = in_b ? bv : av;
        unsigned long long       *olo = in_b ? alo : blo, *ohi = in_b ? ahi : bhi;
        uint32_t                 *ov  = in_b ? av : bv;
        auto digit_of = [&](unsigned long long lo, unsigned long long hi) -> uint32_t {
            return (uint32_t)(((KW == 2 && word == 1) ? hi : lo) >> shift) & 255u;
        };
        // histogram of this digit
        for (int i = tid; i < 256; i += PT) s_off[i] = 0;
        if (tid == 0) s_skip = 0;
        __syncthreads();
        for (int base = 0; base < n; base += PT) {
            const int      i     = base + tid;
            const bool     valid = i < n;
            const uint32_t d     = valid ? digit_of(ilo[i], KW == 2 ? ihi[i] : 0ull) : 256u + lane;
            const unsigned peers = __match_any_sync(FULL, d);
            if (valid && lane == __ffs(peers) - 1) atomicAdd(&s_off[d], (uint32_t)__popc(peers));
        }
        __syncthreads();
        for (int i = tid; i < 256; i += PT)
            if (s_off[i] == (uint32_t)n) s_skip = 1;
        __syncthreads();
        const bool skip = s_skip != 0;
        __syncthreads();
        if (skip) continue; // block-uniform: every key has the same digit
        cta_scan256(s_off);
        __syncthreads();
        for (int tb = 0; tb < n; tb += TILE) {
            for (int i = tid; i < WARPS * 256; i += PT) s_wh[i] = 0;
            __syncthreads();
            unsigned long long klo[ITEMS], khi[ITEMS];
            uint32_t           val[ITEMS], dig[ITEMS], rank[ITEMS];
#pragma unroll
            for (int i = 0; i < ITEMS; ++i) {
                const int  pos   = tb + warp * 32 * ITEMS + i * 32 + lane;
                const bool valid = pos < n;
                klo[i]           = valid ? ilo[pos] : 0ull;
                khi[i]           = (KW == 2 && valid) ? ihi[pos] : 0ull;
                val[i]           = valid ? iv[pos] : 0u;
                dig[i]           = valid ? digit_of(klo[i], khi[i]) : 256u + lane;
            }
            uint32_t *wh = s_wh + warp * 256;
#pragma unroll
            for (int i = 0; i < ITEMS; ++i) {
                const unsigned peers  = __match_any_sync(FULL, dig[i]);
                const bool     valid  = dig[i] < 256u;
                const uint32_t before = valid ? wh[dig[i]] : 0u;
                __syncwarp();
                if (valid && lane == __ffs(peers) - 1) wh[dig[i]] = before + (uint32_t)__popc(peers);
                __syncwarp();
                rank[i] = before + (uint32_t)__popc(peers & lt_mask);
            }
            __syncthreads();
            // per digit: exclusive prefixes over the warps, and the tile's count
            for (int d = tid; d < 256; d += PT) {
                uint32_t run = 0;
#pragma unroll
                for (int w = 0; w < WARPS; ++w) {
                    const uint32_t c  = s_wh[w * 256 + d];
                    s_wh[w * 256 + d] = run;
                    run += c;
                }
                s_cnt[d]  = run;
                s_excl[d] = run;
            }
            __syncthreads();
            cta_scan256(s_excl);
            __syncthreads();
            // stage the tile in digit order
#pragma unroll
            for (int i = 0; i < ITEMS; ++i) {
                if (dig[i] < 256u) {
                    const uint32_t lp = s_excl[dig[i]] + s_wh[warp * 256 + dig[i]] + rank[i];
                    s_lo[lp]          = klo[i];
                    if (KW == 2) s_hi[lp] = khi[i];
                    s_v[lp] = val[i];
                }
            }
            __syncthreads();
            // each digit's run goes to the digit's running offset
            const int tile_n = min(TILE, n - tb);
            for (int j = tid; j < tile_n; j += PT) {
                const unsigned long long lo = s_lo[j];
                const unsigned long long hi = (KW == 2) ? s_hi[j] : 0ull;
                const uint32_t           d  = digit_of(lo, hi);
                const uint32_t           gp = s_off[d] + ((uint32_t)j - s_excl[d]);
                olo[gp]                     = lo;
                if (KW == 2) ohi[gp] = hi;
                ov[gp] = s_v[j];
            }
            __syncthreads();
            for (int d = tid; d < 256; d += PT) s_off[d] += s_cnt[d];
            __syncthreads();
        }
        in_b = !in_b;
    }
    return in_b;
}

// Common-prefix length of the sorted keys at positions x and x + 1: the Karras delta of that
// adjacent pair (src/hlbvh.hpp:852-859; equal keys compare by index).
template <int KIND>
FT_D int adjacent_delta(const unsigned long long *klo, const unsigned long long *khi, int x) {
    const unsigned long long a = klo[x], b = klo[x + 1];
    if (KIND == 2) {
        const unsigned long long ah = khi[x], bh = khi[x + 1];
        if (ah != bh) return clz64(ah ^ bh) - 2;
        if (a != b) return 62 + clz64(a ^ b);
    } else if (a != b) {
        return clz64(a ^ b) - (KIND == 1 ? 1 : 0);
    }
    return (KIND == 2 ? 126 : 63) + clz64((unsigned long long)x ^ (unsigned long long)(x + 1));
}

// Topology and refit of one set in one bottom-up climb per leaf (the agglomerative form of
// the binary radix tree, Apetrei 2014).  A node covering leaves [l, r] has its parent on the
// side whose adjacent delta is larger: at split r (it is the left child) when
// delta(r) > delta(l - 1), else at split l - 1 (the right child); the two deltas are never
// equal (between them lie keys sharing a longer prefix).  It is therefore the Karras tree of
// the same keys, and the climb gives each node the Karras number: a left child [l, r] is
// internal node r, a right child internal node l, the root 0; a one-leaf range is its leaf.
// At each split the first arrival leaves its far end in slot[split] (an acquire-release
// exchange) and stops; the second forms the parent, merges the two boxes in (left, right)
// order as the refit does (src/hlbvh.hpp:925-969), and climbs on.  Each internal node's
// children, parent links, box, record, height and leaf count are written by the thread
// that formed it, before its own exchange, so a sibling that reads them (through L2) after
// the exchange sees them.  delta: n - 1 adjacent deltas; slot: n - 1 words set to -1.
template <class T>
FT_D void climb_build(int j, int n, const int *__restrict__ delta, int *slot, const CtaTreeOut<T> &o) {
    T *const soa[6] = {o.mnx, o.mxx, o.mny, o.mxy, o.mnz, o.mxz};
    int      l = j, r = j;
    T        box[6];
#pragma unroll
    for (int d = 0; d < 6; ++d) box[d] = __ldcg(soa[d] + (j + n - 1));
    int      lc = -1, rc = -1, h = 0; // the current node's children (internal) and height
    T        lb[6], rb[6];
    int      hl = 0, hr = 0, nl = 1, nr = 1; // the children's heights and leaf counts
    for (int steps = 0; steps <= n; ++steps) {
        const bool root = (l == 0 && r == n - 1);
        const bool up_right = !root && (l == 0 || (r != n - 1 && delta[r] > delta[l - 1]));
        const int  ci = (l == r) ? l + n - 1 : root ? 0 : (up_right ? r : l);
        if (l != r) { // an internal node, formed by this thread: write it out
            o.left[ci]  = lc;
            o.right[ci] = rc;
            o.parent[lc] = ci;
            o.parent[rc] = ci;
            o.leaves[ci] = r - l + 1;
#pragma unroll
            for (int d = 0; d < 6; ++d) __stcg(soa[d] + ci, box[d]);
            NodeRec<T> rec;
#pragma unroll
            for (int d = 0; d < 6; ++d) {
                rec.lb[d] = lb[d];
                rec.rb[d] = rb[d];
            }
            rec.l = lc;
            rec.r = rc;
#pragma unroll
            for (int d = 0; d < (int)(sizeof(rec.pad) / 4); ++d) rec.pad[d] = 0;
            rec.pad[0] = (int32_t)rec_child_info((uint32_t)nl, (uint32_t)hl);
            rec.pad[1] = (int32_t)rec_child_info((uint32_t)nr, (uint32_t)hr);
            o.recs[ci] = rec;
            __stcg(o.height + ci, (uint8_t)min(h, 255));
        }
        if (root) return;
        const int split = up_right ? r : l - 1;
        int       prev;
        asm volatile("atom.acq_rel.gpu.global.exch.b32 %0, [%1], %2;"
                     : "=r"(prev)
                     : "l"(slot + split), "r"(up_right ? l : r)
                     : "memory");
        if (prev < 0) return; // first arrival: the sibling forms the parent
        // the sibling: [split + 1, prev] on the right, or [prev, split] on the left
        const int sl = up_right ? split + 1 : prev, sr = up_right ? prev : split;
        const int si = (sl == sr) ? sl + n - 1 : (up_right ? sl : sr);
        T         sb[6];
#pragma unroll
        for (int d = 0; d < 6; ++d) sb[d] = __ldcg(soa[d] + si);
        const int sh = (sl == sr) ? 0 : (int)__ldcg(o.height + si);
        if (up_right) { // this node on the left
            lc = ci;
            rc = si;
#pragma unroll
            for (int d = 0; d < 6; ++d) {
                lb[d] = box[d];
                rb[d] = sb[d];
            }
            hl = h;
            hr = sh;
            nl = r - l + 1;
            nr = sr - sl + 1;
            r  = sr;
        } else {
            lc = si;
            rc = ci;
#pragma unroll
            for (int d = 0; d < 6; ++d) {
                lb[d] = sb[d];
                rb[d] = box[d];
            }
            hl = sh;
            hr = h;
            nl = sr - sl + 1;
            nr = r - l + 1;
            l  = sl;
        }
#pragma unroll
        for (int d = 0; d < 3; ++d) {
            box[2 * d]     = box_min(lb[2 * d], rb[2 * d]);
            box[2 * d + 1] = box_max(lb[2 * d + 1], rb[2 * d + 1]);
        }
        h = 1 + max(hl, hr);
    }
}

// The whole build of one non-empty set of n points by one block of PT threads.
//  x/y/z/id/ghost: the set's input slices; klo/khi/perm (A) and tlo/thi/tperm (B): the set's
//  sort buffers -- on return A holds the sorted keys and input indices (as the single-tree
//  build's key arrays do); bbox_out: the set's box (6 coordinates); set_height: its root height.
// KIND: the Karras delta (0 Morton, 1 63-bit Peano-Hilbert, 2 126-bit).
template <class T, int SFC, int KIND, int PT, int ITEMS>
FT_D void cta_build_set(int n, const T *__restrict__ x, const T *__restrict__ y, const T *__restrict__ z,
                        const uint32_t *id, const int8_t *ghost, unsigned long long *klo, unsigned long long *khi,
                        uint32_t *perm, unsigned long long *tlo, unsigned long long *thi, uint32_t *tperm,
                        const CtaTreeOut<T> &o, T *bbox_out, uint8_t *set_height, unsigned char *smem) {
    using C          = Coord<T>;
    constexpr int KW = C::key_words;
    const int     tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    __shared__ T        s_box[PT / 32][6];
    __shared__ T        s_par[6];
    uint8_t            *s_rot = smem + cta_sort_bytes<KW, PT, ITEMS>(), *s_sub = s_rot + 48 * 8;
    for (int i = tid; i < 48 * 8; i += PT) {
        s_rot[i] = c_rot[i];
        s_sub[i] = c_sub[i];
    }
    // 1. bounding box (the reference's minimum / maximum folds)
    T m[6];
    bb_identity(m);
    for (int i = tid; i < n; i += PT) {
        T v[6] = {x[i], x[i], y[i], y[i], z[i], z[i]};
        bb_fold(m, v);
    }
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) {
        T u[6];
#pragma unroll
        for (int d = 0; d < 6; ++d) u[d] = __shfl_down_sync(0xffffffffu, m[d], off);
        bb_fold(m, u);
    }
    if (lane == 0)
#pragma unroll
        for (int d = 0; d < 6; ++d) s_box[warp][d] = m[d];
    __syncthreads();
    if (tid == 0) {
        T b[6];
#pragma unroll
        for (int d = 0; d < 6; ++d) b[d] = s_box[0][d];
        for (int w = 1; w < PT / 32; ++w) bb_fold(b, s_box[w]);
#pragma unroll
        for (int d = 0; d < 6; ++d) bbox_out[d] = b[d];
#pragma unroll
        for (int d = 0; d < 3; ++d) {
            if constexpr (C::is_float) sfc_axis_params(b[2 * d], b[2 * d + 1], s_par[2 * d], s_par[2 * d + 1]);
            else s_par[2 * d] = s_par[2 * d + 1] = T(0);
        }
    }
    __syncthreads();
    // 2. keys, input index as the value
    for (int i = tid; i < n; i += PT) {
        unsigned long long hi, lo;
        encode_point<T, SFC>(x[i], y[i], z[i], s_par, s_rot, s_sub, hi, lo);
        klo[i] = lo;
        if (KW == 2) khi[i] = hi;
        perm[i] = (uint32_t)i;
    }
    __syncthreads();
    // 3. sort
    const bool in_b = cta_sort<KW, PT, ITEMS>(klo, khi, perm, tlo, thi, tperm, n, smem);
    if (in_b) { // back into A, where the tree's keys live
        for (int i = tid; i < n; i += PT) {
            klo[i] = tlo[i];
            if (KW == 2) khi[i] = thi[i];
            perm[i] = tperm[i];
        }
        __syncthreads();
    }
    // 4. leaves; internal slots of id / is_ghost / orig_idx are 0 and the root's parent is -1
    for (int j = tid; j < n; j += PT) {
        const uint32_t src  = perm[j];
        const int      leaf = n - 1 + j;
        const T        a = x[src], b = y[src], c = z[src];
        o.mnx[leaf]   = a;
        o.mxx[leaf]   = a;
        o.mny[leaf]   = b;
        o.mxy[leaf]   = b;
        o.mnz[leaf]   = c;
        o.mxz[leaf]   = c;
        o.id[leaf]    = id ? id[src] : src;
        o.ghost[leaf] = ghost ? ghost[src] : (int8_t)0;
        o.orig[leaf]  = (int32_t)src;
    }
    for (int i = tid; i < n - 1; i += PT) {
        o.id[i]    = 0u;
        o.ghost[i] = (int8_t)0;
        o.orig[i]  = 0;
    }
    if (tid == 0) o.parent[0] = -1;
    if (n < 2) {
        if (tid == 0) *set_height = 0;
        __syncthreads();
        return;
    }
    // 5-6. topology and refit in one climb per leaf: the adjacent deltas (into the sort's
    // spare buffer), the exchange slots, then the climbs
    int *delta = reinterpret_cast<int *>(tlo);
    for (int x = tid; x < n - 1; x += PT) {
        delta[x]      = adjacent_delta<KIND>(klo, KW == 2 ? khi : nullptr, x);
        o.counters[x] = -1;
    }
    __syncthreads();
    for (int j = tid; j < n; j += PT) climb_build<T>(j, n, delta, o.counters, o);
    __syncthreads();
    T *const soa[6] = {o.mnx, o.mxx, o.mny, o.mxy, o.mnz, o.mxz};
    // 7. 4-wide records (boxes read through L2, where the refit wrote them)
    for (int v = tid; v < n - 1; v += PT) {
        int       ch[4] = {-1, -1, -1, -1};
        int       c     = 0;
        const int l = o.left[v], r = o.right[v];
        if (l >= n - 1) ch[c++] = l;
        else {
            ch[c++] = o.left[l];
            ch[c++] = o.right[l];
        }
        if (r >= n - 1) ch[c++] = r;
        else {
            ch[c++] = o.left[r];
            ch[c++] = o.right[r];
        }
        WideRec<T> w;
#pragma unroll
        for (int i = 0; i < 4; ++i) {
#pragma unroll
            for (int d = 0; d < 6; ++d) w.box[i][d] = ch[i] >= 0 ? __ldcg(soa[d] + ch[i]) : T(0);
            w.child[i] = ch[i];
        }
        o.wide[v] = w;
    }
    if (tid == 0) *set_height = __ldcg(o.height);
    __syncthreads();
}

} // namespace ft
