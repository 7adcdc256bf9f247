// ft_fast.cu -- fast self-kNN and knn_query with exact fallback (FT_METHOD_FAST, the default).
//
// A warp takes 32 consecutive queries (sorted leaves, or external points sorted by their
// SFC rank), so its lanes work on neighbouring parts of the tree.
//  1. Seeding: each lane inserts the leaves of its SFC window [r - h, r + h] into its heap
//     (a max-heap of k entries in shared memory), so the heap is full, and pruning effective,
//     before the walk starts.
//  2. Walk (default): each lane walks its own query over 4-wide records (the grandchildren of
//     a binary node, built after the refit): up to four box distances per step, leaves go to
//     the heap, the nearest needed internal node is walked next and the others are stacked
//     farthest first.  Every loop iteration is one expansion, so the lanes run the same
//     instructions except the heap insertion.  The binary walks (per-lane, compact, warp-
//     shared) remain selectable.
//  3. Exactness: the result set is the exact k nearest; only the order among equal distances
//     can differ from the reference (its visit order and heap history decide it).  A lane
//     flags its query when any tie could matter -- equal distances inside the top k, a
//     candidate at exactly the current k-th distance left out, an eviction that leaves an
//     equal maximum (nodes at exactly the k-th distance are walked, not pruned, so such
//     candidates are seen) -- or when an optional per-query bound cut off a possible
//     neighbour, or its stack would overflow.  Flagged queries are rerun by the reference
//     traversal (exact_replay_kernel, or knn_query's heap tier for external points).  On trees
//     of height 63 or more the reference's stack guard drops subtrees; a query whose
//     neighbourhood it could reach is replayed too (stack_guard_reaches).
#include <cuda.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <mutex>
#include <string>
#include <type_traits>

#include "ft_build_dev.cuh"
#include "ft_common.cuh"
#include "ft_cta_build.cuh"
#include "ft_internal.h"

namespace ft {

static constexpr int kFastStack = 64;
#ifndef FT_XB_MAX_QUERIES
#define FT_XB_MAX_QUERIES (1 << 21)
#endif
#ifndef FT_FAST_MINB
#define FT_FAST_MINB 10
#endif
// Two warps per block: each thread's heap takes k x 8 B of shared memory (16 KB per 64 threads
// at k = 32); the 4-wide walk is compiled for 10 such blocks per SM (20 warps, 96 registers a
// thread; measured on 10M clustered points: 9 / 10 / 11 / 12 / 13 blocks 52.7 / 48.8 / 52.1 /
// 52.0 / 56.2 ms, the tighter budgets spilling).
static constexpr int kFastWarps = 2;
static constexpr int kFastThreads = 32 * kFastWarps;
// Warps per block for a heap capacity: k <= 32 heaps take 8 KB per warp (two-warp blocks);
// 64-entry heaps take 16 KB per warp, in one-warp blocks.
template <int KC> constexpr int fast_warps() { return KC > 32 ? 1 : kFastWarps; }
// The fast walk's heap entries are 8 bytes: a float key of the distance and the leaf rank.
// Float coordinates' distances are float sums widened to double (node_distance_sq), so their
// key is the distance itself, exactly.  Other types key a distance by rounding it toward zero
// to a float, which keeps the order (a < b implies key(a) <= key(b)): every decision the
// heap takes on two different keys is the one the exact distances would take, and a decision
// on equal keys (a candidate at the k-th key, an eviction leaving an equal maximum, equal keys
// in the sorted result) flags the query for the exact replay, as exact ties already do.  The
// output distances are recomputed exactly from the leaves.  8 bytes instead of 12 (16 with
// alignment) an entry keep more warps resident and make the sifts 32-bit.
template <class T> using heap_dist_t = float;
template <class T> constexpr bool heap_keyed() { return !std::is_same<T, float>::value; }
template <class T> FT_D float heap_key(typename Coord<T>::dist_t d) {
    if constexpr (!heap_keyed<T>()) return (float)d;
    else if constexpr (Coord<T>::is_float) return __double2float_rz(d);
    else return __ull2float_rz(d);
}
// The largest distance whose key is `key` (so a distance above it has a larger key).
template <class T> FT_D typename Coord<T>::dist_t heap_key_ub(float key) {
    if constexpr (!heap_keyed<T>()) {
        return (double)key;
    } else if constexpr (Coord<T>::is_float) {
        // distances are not negative; FLT_MAX keys every double from FLT_MAX up, infinity and
        // NaN key only themselves
        if (!(key < FLT_MAX)) return key == FLT_MAX ? DBL_MAX : (double)key;
        const float up = __uint_as_float(__float_as_uint(key) + 1u); // the next float
        return __longlong_as_double(__double_as_longlong((double)up) - 1ll); // the double below it
    } else {
        if (key < 16777216.0f) return (unsigned long long)key; // below 2^24 the key is exact
        const float up = __uint_as_float(__float_as_uint(key) + 1u); // an integer from 2^24 up
        return up >= 18446744073709551616.0f ? ~0ull : (unsigned long long)up - 1ull;
    }
}

// Group walk (variant 5): a lower bound of the walk's distance from every point of the
// group box [g0, g1] (per axis) to a node box b (minx, maxx, miny, maxy, minz, maxz).  Each
// axis gap is measured from the group's nearer side, so it is no larger than the gap from
// any point inside the group box, and the distance is monotone in the three gaps (rounded
// subtraction, products and sums of non-negative values included).  Periodic trees: the
// clean 42-bit form only (coordinates below 2^42, group coordinates masked); on the circle,
// the group interval and the node interval are disjoint exactly when the two gaps a, b and
// the two lengths add up to one period, and then every group point is at least min(a, b)
// from the node.
template <class T, int PER>
FT_D typename Coord<T>::dist_t group_lb(const T g0[3], const T g1[3], const T b[6]) {
    using C = Coord<T>;
    if constexpr (C::is_float) {
        const T dx = c_fmax(sub_rn(b[0], g1[0]), c_fmax(T(0), sub_rn(g0[0], b[1])));
        const T dy = c_fmax(sub_rn(b[2], g1[1]), c_fmax(T(0), sub_rn(g0[1], b[3])));
        const T dz = c_fmax(sub_rn(b[4], g1[2]), c_fmax(T(0), sub_rn(g0[2], b[5])));
        return (double)add_rn(add_rn(mul_rn(dx, dx), mul_rn(dy, dy)), mul_rn(dz, dz));
    } else {
        unsigned long long a[3];
#pragma unroll
        for (int i = 0; i < 3; ++i) {
            const T lo = b[2 * i], hi = b[2 * i + 1];
            if constexpr (PER == 2) {
                constexpr unsigned long long M = (1ull << C::bits) - 1ull;
                const unsigned long long ga = ((unsigned long long)lo - (unsigned long long)g1[i]) & M;
                const unsigned long long gb = ((unsigned long long)g0[i] - (unsigned long long)hi) & M;
                const unsigned long long span =
                    ((unsigned long long)g1[i] - (unsigned long long)g0[i]) + ((unsigned long long)hi - lo);
                const unsigned long long g = ga < gb ? ga : gb;
                a[i] = (ga + gb + span > M + 1ull) ? 0ull : (unsigned long long)(uint32_t)(g >> C::dist_shift);
            } else {
                a[i] = g1[i] < lo   ? (unsigned long long)(T)(lo - g1[i]) >> C::dist_shift
                       : g0[i] > hi ? (unsigned long long)(T)(g0[i] - hi) >> C::dist_shift
                                    : 0ull;
            }
        }
        return Metric<T>::sq(a[0]) + Metric<T>::sq(a[1]) + Metric<T>::sq(a[2]);
    }
}

// Signed offset of coordinate v from the group's corner o (integer coordinates): the
// wrapped 42-bit difference for the clean periodic metric, else the plain difference.
template <class T, int PER> FT_D long long group_offset(T v, T o) {
    if constexpr (PER == 2) {
        constexpr int sh = 64 - Coord<T>::bits;
        return (long long)(((unsigned long long)v - (unsigned long long)o) << sh) >> sh;
    } else {
        return (long long)((unsigned long long)v - (unsigned long long)o);
    }
}

// Float lower bound of the exact integer distance between a staged leaf (offsets e.xyz from
// the group's corner) and a query (offsets q), given gerr >= the error of |e - q| against the
// exact gap G on any axis (2^-21 of the largest offset magnitude: two conversions and one
// subtraction, each within 2^-24 of its magnitude, with a factor of two to spare).  Per axis
// the exact term is floor(G / 2^shift) > G / 2^shift - 1 >= (|e - q| - gerr) / 2^shift - 1,
// and scale = 2^-shift (1 - 2^-20) absorbs the roundings of that bound, so each float term is
// at most the exact one and the float sum of squares is at most the exact sum times
// (1 + 2^-22).  A leaf is skipped only when that sum, shrunk by 2^-16, still exceeds the
// lane's radius rounded up: then the exact distance exceeds the radius too.
FT_D float group_filter(const float4 &e, const float q[3], float gerr, float scale) {
    const float lx = fmaxf(0.0f, fmaf(fabsf(e.x - q[0]) - gerr, scale, -1.0f));
    const float ly = fmaxf(0.0f, fmaf(fabsf(e.y - q[1]) - gerr, scale, -1.0f));
    const float lz = fmaxf(0.0f, fmaf(fabsf(e.z - q[2]) - gerr, scale, -1.0f));
    return fmaf(lz, lz, fmaf(ly, ly, lx * lx));
}

// A distance rounded up to a float (non-negative values): the 4-wide walk's key threshold for
// float coordinates, whose keys are the distances themselves.
template <class D> FT_D float stack_key_up(D d) {
    if constexpr (std::is_floating_point<D>::value) return __double2float_ru((double)d);
    else return __ull2float_ru((unsigned long long)d);
}

template <class T> FT_D T coord_top() {
    if constexpr (std::is_same<T, float>::value) return 3.402823466e38f;
    else if constexpr (std::is_same<T, double>::value) return 1.7976931348623157e308;
    else return ~T(0);
}
template <class T> FT_D T coord_bottom() {
    if constexpr (Coord<T>::is_float) return -coord_top<T>();
    else return T(0);
}

// The reference's traversal stack (MAX_STACK_DEPTH 64) pushes the children of a popped
// internal node only while fewer than 62 entries are in use (src/hlbvh.hpp:1152, 1359, 1618,
// 1788); on taller trees it drops them.  It pushes the farther child first and the nearer
// one on top, so the entries below a popped node never change: after popping node v the
// stack holds exactly the number of nearer-child turns (ld2 <= rd2 takes the left child) on
// the root-to-v path, whatever the heap did.  The guard therefore fires only at an internal
// node whose path has 62 such turns, and it can change the query's rows only when that node
// lies within the query's k-th distance dk: a subtree beyond dk holds no neighbour, and no
// point under a node is nearer than the node's box.  Returns true when some internal node
// with 62 nearer-child turns lies within dk (then the reference traversal reruns the query).
// The search follows a child only while its subtree is tall enough to still reach 62 turns
// at an internal node (height >= 63 - turns); that slack never grows along a path and a far
// turn spends one, so trees of height <= 62 need no search and taller ones are searched near
// their tallest paths only.  Bounded: a search that runs long answers true.
// stk: scratch of kGuardStack entries (the walk's own stack, free by then).
static constexpr int kGuardStack = 80;
template <class T, int PER, bool COH = false>
FT_D bool stack_guard_reaches(const TreeDev<T> &t, T px, T py, T pz, typename Coord<T>::dist_t dk,
                              unsigned long long *stk) {
    using D = typename Coord<T>::dist_t;
    const int n = t.n;
    if (n < 2 || (int)t.height[0] < 63) return false;
    constexpr int kCap = kGuardStack; // entries: (node << 8) | nearer-child turns from the root
    int                sp     = 1;
    int                budget = 4096;
    stk[0]                    = 0ull;
    while (sp > 0) {
        if (--budget < 0) return true;
        const unsigned long long e = stk[--sp];
        const int                u = (int)(e >> 8), s = (int)(e & 255ull);
        T                        lb[6], rb[6];
        int                      l, r;
        load_rec<T, COH>(t.recs, u, lb, rb, l, r);
        const D    ld2 = Metric<T>::template dist<(PER != 0), (PER == 2)>(px, py, pz, lb[0], lb[1], lb[2], lb[3],
                                                                         lb[4], lb[5]);
        const D    rd2 = Metric<T>::template dist<(PER != 0), (PER == 2)>(px, py, pz, rb[0], rb[1], rb[2], rb[3],
                                                                         rb[4], rb[5]);
        const bool left_near = ld2 <= rd2;
#pragma unroll
        for (int side = 0; side < 2; ++side) {
            const int c  = side == 0 ? l : r;
            const D   dc = side == 0 ? ld2 : rd2;
            const int sc = s + (((side == 0) == left_near) ? 1 : 0);
            if (c >= n - 1 || dc > dk) continue; // a leaf, or no neighbour below it
            if (sc >= 62) return true;            // popped with 62 entries below it: dropped
            if ((int)t.height[c] + sc < 63) continue;
            if (sp >= kCap) return true;
            stk[sp++] = ((unsigned long long)c << 8) | (unsigned long long)sc;
        }
    }
    return false;
}

// Slot of this lane's entry in a list whose length is *count, for the lanes with `take`: one
// atomic per warp, and a warp's entries stay together in lane order (so a later launch over
// the list takes neighbouring queries in one warp).  Every lane of the warp must call it.
FT_D uint32_t warp_append(uint32_t *count, bool take, int lane) {
    const unsigned m    = __ballot_sync(0xffffffffu, take);
    uint32_t       base = 0;
    if (m) {
        const int leader = __ffs(m) - 1;
        if (lane == leader) base = atomicAdd(count, (uint32_t)__popc(m));
        base = __shfl_sync(0xffffffffu, base, leader);
    }
    return base + (uint32_t)__popc(m & ((1u << lane) - 1u));
}

template <class T> FT_D T warp_min_t(T v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        const T w = __shfl_xor_sync(0xffffffffu, v, o);
        v         = w < v ? w : v;
    }
    return v;
}
template <class T> FT_D T warp_max_t(T v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        const T w = __shfl_xor_sync(0xffffffffu, v, o);
        v         = w > v ? w : v;
    }
    return v;
}

// Queries handed from one launch of the walk to the next (bound misses): list entry i is
// output row rows[i] and, for self queries on one tree, leaf rank ranks[i]; *count entries.
struct QueryList {
    const int32_t  *ranks = nullptr;
    const int32_t  *rows  = nullptr;
    const uint32_t *count = nullptr; // null: no list, the launch covers queries [0, num)
};
// Where a launch sends the queries whose pruning bound proved too small (null rows: they
// join the replay list like the other flagged queries).
struct MissList {
    int32_t  *ranks = nullptr;
    int32_t  *rows  = nullptr;
    uint32_t *count = nullptr;
};
struct ListArgs {
    QueryList lst;
    MissList  miss;
};

// One warp's 32 queries: entries [qbase, qbase + 32) of [0, num) -- query rows, or entries of
// the list `lst` when it is given.  NW: warps of the calling block (the heaps are laid out
// per thread of the block); COH: tree records read through L2 (the persistent batch kernel,
// whose blocks read trees that other blocks built earlier in the same launch).
template <class T, int PER, int KC, int VAR, int NW = fast_warps<KC>(), bool COH = false, bool XB = false>
FT_D void fast_warp(const int qbase, const QueryList &lst, const MissList &miss, unsigned char *smem,
                    TreeDev<T> t_all, BatchDev bt, const T *__restrict__ qx, const T *__restrict__ qy,
                    const T *__restrict__ qz, const uint32_t *__restrict__ order,
                    const int32_t *__restrict__ leaf_ids, int num, int k, int half_window, int exclude_self,
                    int ret_orig, const typename Coord<T>::dist_t *__restrict__ bound,
                    unsigned long long *__restrict__ out_idx, typename Coord<T>::dist_t *__restrict__ out_dist,
                    int32_t *__restrict__ replay_ranks, int32_t *__restrict__ replay_rows, uint32_t *replay_count,
                    uint32_t *status, unsigned long long *visit_count) {
    using D = typename Coord<T>::dist_t;
    constexpr int kFastWarps = NW, kFastThreads = 32 * kFastWarps; // the block's shape
    using H      = heap_dist_t<T>;
    H       *hd  = reinterpret_cast<H *>(smem);
    int32_t *hix = reinterpret_cast<int32_t *>(hd + k * kFastThreads); // heaps sized for k (<= KC)
    __shared__ int32_t s_node[kFastWarps][kFastStack];
    // the 4-wide walk's per-lane stack, then the stack-guard test's scratch
    unsigned long long lane_stack[96];
    static_assert(sizeof(lane_stack) / sizeof(lane_stack[0]) >= kGuardStack, "guard scratch");

    const int      tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const unsigned FULL = 0xffffffffu;
    if (qbase >= num) return; // warp-uniform
    // External query points are walked in the order `order` (sorted by SFC rank, so a warp
    // takes neighbouring queries); q is the output row.  A listed launch takes rows from the
    // list (inactive lanes borrow the first lane's row, which is valid).
    const bool listed = lst.count != nullptr;
    bool       active = qbase + lane < num;
    const int  q      = listed ? lst.rows[active ? qbase + lane : qbase]
                               : ((qx && order && active) ? (int)order[qbase + lane] : qbase + lane);
    // Batched sets: each lane walks the tree of the set its query belongs to (rank local to
    // the set, output row global).
    TreeDev<T> t            = t_all;
    int        rank         = 0;
    bool       force_replay = false;
    if (bt.off) {
        const int qs = (active || listed) ? q : num - 1;
        const int s  = find_set(bt.off, bt.S, qs);
        t            = set_view(t_all, bt, s);
        rank         = qs - (int)bt.off[s];
        bool outside = false;
        if constexpr (PER != 0 && !Coord<T>::is_float) {
            // periodic integer set with a coordinate at or above the period (root box maxima):
            // the box distance is not monotone there, so only the reference traversal applies
            constexpr unsigned long long P = 1ull << Coord<T>::bits;
            outside = outside || (unsigned long long)t.max_x[0] >= P || (unsigned long long)t.max_y[0] >= P ||
                      (unsigned long long)t.max_z[0] >= P;
        }
        if (active && outside) {
            force_replay = true;
            active       = false;
        }
    } else if (listed && !qx) {
        rank = active ? lst.ranks[qbase + lane] : 0;
    } else {
        rank = active ? (leaf_ids ? leaf_ids[q] : q) : 0;
    }
    const int n = t.n;
#define HD(s) hd[(s) * kFastThreads + tid]
#define HI(s) hix[(s) * kFastThreads + tid]

    // External query points (knn_query): leaf_ids holds each point's SFC rank, the centre of
    // its seeding window (-1: no window); there is no self leaf.
    const bool ext = qx != nullptr;
    if (!ext && active && (rank < 0 || rank >= n)) {
        atomicOr(status, STATUS_BAD_INPUT);
        for (int i = 0; i < k; ++i) {
            out_idx[(size_t)q * k + i]  = ~0ull;
            out_dist[(size_t)q * k + i] = dist_missing<D>();
        }
        active = false;
        rank   = 0;
    }
    const bool seeded   = !ext || rank >= 0;
    if (ext) rank = min(max(rank, 0), n - 1);
    const int  slot      = rank + n - 1;
    const T    px        = ext ? qx[active ? q : 0] : t.min_x[slot];
    const T    py        = ext ? qy[active ? q : 0] : t.min_y[slot];
    const T    pz        = ext ? qz[active ? q : 0] : t.min_z[slot];
    const int  self_leaf = (exclude_self && !ext) ? slot : -1;
    const D   B         = (bound && active) ? bound[q] : dist_heap_max<D>();

    int  count = 0;
    H    hk    = H(0); // key of the k-th entry (the heap's root) once the heap is full
    D    hmax  = D(0); // the largest distance with that key: at least the k-th distance
    D    thr   = B;    // pruning threshold: B until the heap is full, then min(B, hmax)
    bool flag  = false;
    // The same threshold on keys (the 4-wide walk prunes, orders and stacks by key): a distance
    // within thr has a key within kthr (keyed: thr is hmax or B, and d <= hmax gives
    // key(d) <= hk, d <= B gives key(d) <= key(B); float coordinates: the key is the distance
    // and kthr is thr rounded up), so a node whose key exceeds kthr is surely beyond thr.
    const H kB   = heap_keyed<T>() ? heap_key<T>(B) : stack_key_up<D>(B);
    H       kthr = kB;
    auto    set_thr = [&]() {
        thr = hmax < B ? hmax : B;
        if constexpr (heap_keyed<T>()) kthr = hk < kB ? hk : kB;
        else kthr = stack_key_up<D>(thr);
    };

    // exact distance of the query to a leaf (by rank), as the walk computes it
    auto exact = [&](int32_t leaf) -> D {
        const int s = leaf + n - 1;
        const T   x = t.min_x[s], y = t.min_y[s], z = t.min_z[s];
        return Metric<T>::template dist<(PER != 0), (PER == 2)>(px, py, pz, x, x, y, y, z, z);
    };
    // Keyed heaps: the entries sharing the k-th key sit at the top of the max-heap, and
    // exchanging leaves between equal keys keeps the heap valid.  Finds the slot of the
    // exactly largest of them (the root's slot first), its distance, and whether another
    // entry ties it exactly.  Used with XB (external queries, whose replay -- knn_query's
    // heap tier -- costs far more than the self queries' replay): without it a candidate or
    // an eviction on the k-th key flags the query instead.
    auto kth_exact = [&](int &slot, D &dmax, bool &tie) {
        slot = 0;
        dmax = exact(HI(0));
        tie  = false;
        for (int s2 = 1; s2 < k; ++s2)
            if (HD(s2) == hk) {
                const D e = exact(HI(s2));
                if (e > dmax) {
                    dmax = e;
                    slot = s2;
                    tie  = false;
                } else if (!(e < dmax)) {
                    tie = true; // equal (or not comparable)
                }
            }
    };
    // id: the leaf's rank (original indices are looked up when the rows are written); kd: the
    // distance's key, heap_key(d2)
    auto insert_k = [&](D d2, H kd, int32_t id) {
        if (count < k) {
            int i = count;
            while (i > 0) {
                int p  = (i - 1) >> 1;
                H   pd = HD(p);
                if (kd <= pd) break;
                HD(i) = pd;
                HI(i) = HI(p);
                i     = p;
            }
            HD(i) = kd;
            HI(i) = id;
            ++count;
            if (count == k) {
                hk   = HD(0);
                hmax = heap_key_ub<T>(hk);
                set_thr();
            }
        } else if (kd < hk) {
            if constexpr (heap_keyed<T>() && XB) {
                // another entry shares the k-th key: evict the exactly largest of them
                if ((k > 1 && HD(1) == hk) || (k > 2 && HD(2) == hk)) {
                    int  slot;
                    D    dmax;
                    bool tie;
                    kth_exact(slot, dmax, tie);
                    if (tie) flag = true; // which of the tied leaves stays is the reference's order
                    if (slot != 0) {
                        const int32_t tmp = HI(0);
                        HI(0)             = HI(slot);
                        HI(slot)          = tmp;
                    }
                }
            }
            const H old = hk;
            int     i   = 0;
            for (;;) {
                int l = 2 * i + 1;
                if (l >= k) break;
                int r  = l + 1;
                int c  = i;
                H   cd = kd;
                H   ld = HD(l);
                if (ld > cd) {
                    c  = l;
                    cd = ld;
                }
                if (r < k) {
                    H rd = HD(r);
                    if (rd > cd) {
                        c  = r;
                        cd = rd;
                    }
                }
                if (c == i) break;
                HD(i) = cd;
                HI(i) = HI(c);
                i     = c;
            }
            HD(i) = kd;
            HI(i) = id;
            hk    = HD(0);
            hmax  = heap_key_ub<T>(hk);
            set_thr();
            // an equal distance stays at the boundary (keyed: the entries left on the old key
            // are exactly nearer than the one evicted, unless tied, flagged above)
            if (!(heap_keyed<T>() && XB) && hk == old) flag = true;
        } else if (kd == hk) {
            if constexpr (heap_keyed<T>() && XB) {
                // the candidate's key is the k-th key: compare it exactly with the largest entry
                // on that key, and take that entry's place (same key: the heap stays valid)
                int  slot;
                D    dmax;
                bool tie;
                kth_exact(slot, dmax, tie);
                if (d2 < dmax) {
                    HI(slot) = id;
                    if (tie) flag = true;
                } else if (!(d2 > dmax)) {
                    flag = true; // a candidate at exactly the k-th distance was left out
                }
            } else {
                flag = true; // a candidate at exactly the k-th distance was left out
            }
        }
    };
    auto insert = [&](D d2, int32_t id) { insert_k(d2, heap_key<T>(d2), id); };

    // ---- 1. seed from the SFC window ----
    const int W  = seeded ? min(n, 2 * half_window + 1) : 0;
    const int w0 = active ? max(0, min(rank - half_window, n - W)) : 0;
    const int w1 = active ? w0 + W - 1 : -1;
    for (int j = 0; j < W; ++j) {
        const int leaf = w0 + j;
        if (active && leaf + n - 1 != self_leaf) {
            // a leaf's box is its point (min == max): read the min arrays only
            const int s  = leaf + n - 1;
            const T   x = t.min_x[s], y = t.min_y[s], z = t.min_z[s];
            const D   d2 = Metric<T>::template dist<(PER != 0), (PER == 2)>(px, py, pz, x, x, y, y, z, z);
            insert(d2, leaf);
        }
    }

    // ---- 2. walk ----
    D   sd[kFastStack];
    int sp = 1;
    sd[0]  = Metric<T>::template dist<(PER != 0), (PER == 2)>(px, py, pz, t.min_x[0], t.max_x[0], t.min_y[0], t.max_y[0], t.min_z[0],
                                          t.max_z[0]);
    long long budget = 2ll * n + 64;
    long long visits = 0;
    // A node is needed unless it is strictly beyond the lane's bound or its k-th distance.
    // Nodes at exactly the k-th distance are walked (not pruned), so any other point at
    // that distance reaches insert() and raises the tie flag there.
    auto needs = [&](D d2) { return active && !(d2 > thr); };
    bool group_done = false;
    if constexpr (VAR == 5) {
        // Group walk: the warp's 32 queries (neighbours on the curve) walk the tree once
        // together.  Lanes expand up to 32 records at a time from a shared stack and keep a
        // child when its distance from the group's box is within the largest of the lanes'
        // radii (k-th distance or bound); kept leaves are staged in shared memory and every
        // lane then tests every staged leaf against its own radius.  Radii only shrink, so a
        // pruned node is beyond every lane's final k-th distance, and every leaf a lane needs
        // (ties at its k-th distance included) reaches its heap.
        // Integer coordinates: the staged leaves hold float offsets from the group's corner,
        // and a lane first evaluates a float lower bound of the exact distance (group_filter);
        // only leaves that pass get the exact distance and the heap, so the exact 64-bit
        // arithmetic and the divergent insertions run for a few leaves per lane.
        // Used when every lane's heap is already full (seeded) on a single tree with the open,
        // float or clean periodic metric; other warps take the 4-wide walk.
        constexpr bool FILT    = !Coord<T>::is_float;
        constexpr int  kGStack = 256, kGCand = 128;
        __shared__ int32_t g_stk[kFastWarps][kGStack];
        __shared__ float4  g_cf[kFastWarps][FILT ? kGCand : 1];  // offsets x, y, z; slot bits in w
        __shared__ T       g_cx[kFastWarps][FILT ? 1 : kGCand], g_cy[kFastWarps][FILT ? 1 : kGCand],
            g_cz[kFastWarps][FILT ? 1 : kGCand];
        __shared__ int32_t g_cs[kFastWarps][FILT ? 1 : kGCand];
        bool finite = true;
        if constexpr (Coord<T>::is_float)
            finite = !active || (isfinite((double)px) && isfinite((double)py) && isfinite((double)pz));
        const bool can = !bt.off && PER != 1 && n > 1 && __all_sync(FULL, (!active || count >= k) && finite) &&
                         __any_sync(FULL, active);
        auto gm = [](T v) -> T {
            if constexpr (PER == 2) return (T)((unsigned long long)v & ((1ull << Coord<T>::bits) - 1ull));
            else return v;
        };
        const T pv[3] = {gm(px), gm(py), gm(pz)};
        T       g0[3], g1[3];
        D       R = D(0);
        float   qf[3] = {0.0f, 0.0f, 0.0f}, gerr = 0.0f;
        bool    ok = can;
        auto radius = [&]() { return warp_max_t<D>(active ? (hmax < B ? hmax : B) : D(0)); };
        if (can) {
#pragma unroll
            for (int a = 0; a < 3; ++a) {
                g0[a] = warp_min_t<T>(active ? pv[a] : coord_top<T>());
                g1[a] = warp_max_t<T>(active ? pv[a] : coord_bottom<T>());
            }
            R = radius();
            if constexpr (FILT) {
                // every staged leaf is within span + (sqrt(R) + 1) 2^shift of the group's
                // corner on each axis; offsets below 2^40 keep the float filter's error bound
                // (and the periodic differences unwrapped)
                double span = 0.0;
#pragma unroll
                for (int a = 0; a < 3; ++a) span = fmax(span, (double)(unsigned long long)(g1[a] - g0[a]));
                const double lam = span + (sqrt((double)R) + 2.0) * (double)(1ull << Coord<T>::dist_shift);
                ok   = lam < 0x1p40;
                gerr = (float)(lam * 0x1p-21);
#pragma unroll
                for (int a = 0; a < 3; ++a) qf[a] = (float)group_offset<T, PER>(pv[a], g0[a]);
            }
        }
        if (ok) {
            group_done = true;
            int  top = 1, cc = 0;
            bool overflow = false;
            if (lane == 0) g_stk[warp][0] = 0;
            __syncwarp();
            auto offer = [&](D d2, int s) {
                const int leaf = s - (n - 1);
                if (active && !(d2 > hmax) && !(d2 > B) && (leaf < w0 || leaf > w1) && s != self_leaf)
                    insert(d2, leaf);
            };
            auto flush = [&]() {
                if constexpr (FILT) {
                    // per word of 32 staged leaves: the float filter against the lane's
                    // current radius sets one bit per leaf that may be within it, then each
                    // lane takes the exact distance of its set bits and offers them to its
                    // heap (the warp loops as long as its busiest lane)
                    constexpr float kScale = 1.0f / (float)(1ull << Coord<T>::dist_shift) * (1.0f - 0x1p-20f);
                    for (int w = 0; w < cc; w += 32) {
                        const D     H    = hmax < B ? hmax : B;
                        const float Hup  = (float)H * (1.0f + 0x1p-20f);
                        const int   nw   = min(32, cc - w);
                        uint32_t    bits = 0;
#pragma unroll 4
                        for (int j = 0; j < nw; ++j) {
                            const float f = group_filter(g_cf[warp][w + j], qf, gerr, kScale);
                            bits |= (uint32_t)(!(f * (1.0f - 0x1p-16f) > Hup)) << j;
                        }
                        if (!active) bits = 0;
                        while (bits) {
                            const int j = __ffs(bits) - 1;
                            bits &= bits - 1;
                            const int s = __float_as_int(g_cf[warp][w + j].w);
                            const T   x = t.min_x[s], y = t.min_y[s], z = t.min_z[s];
                            offer(Metric<T>::template dist<(PER != 0), (PER == 2)>(px, py, pz, x, x, y, y, z, z), s);
                        }
                    }
                } else {
                    // every lane tests every staged leaf (two at a time, loads ahead of insertions)
                    for (int c = 0; c < cc; c += 2) {
                        const int c1 = c + 1 < cc ? c + 1 : c;
                        const T   x0 = g_cx[warp][c], y0 = g_cy[warp][c], z0 = g_cz[warp][c];
                        const T   x1 = g_cx[warp][c1], y1 = g_cy[warp][c1], z1 = g_cz[warp][c1];
                        const int s0 = g_cs[warp][c], s1 = g_cs[warp][c1];
                        const D   d0 = Metric<T>::template dist<(PER != 0), (PER == 2)>(px, py, pz, x0, x0, y0, y0, z0, z0);
                        const D   d1 = Metric<T>::template dist<(PER != 0), (PER == 2)>(px, py, pz, x1, x1, y1, y1, z1, z1);
                        offer(d0, s0);
                        if (c1 != c) offer(d1, s1);
                    }
                }
                visits += cc;
                cc = 0;
                R  = radius();
                __syncwarp();
            };
            while (top > 0) {
                if (--budget < 0) {
                    if (lane == 0) atomicOr(status, STATUS_TRAVERSAL_LIMIT);
                    overflow = true;
                    break;
                }
                // pop up to 32 records, leaving room for four children each
                const int m = min(min(top, 32), (kGStack - top) / 3);
                if (m <= 0) {
                    overflow = true; // the stack is full: the queries go to the replay
                    break;
                }
                const int base = top - m;
                const int node = lane < m ? g_stk[warp][base + lane] : -1;
                top            = base;
                __syncwarp();
                T        bx[4][6];
                int      ch[4] = {-1, -1, -1, -1};
                unsigned kl = 0, ki = 0;
                if (node >= 0) {
                    ++visits;
                    load_wide<T, COH>(t.wide, node, bx, ch);
#pragma unroll
                    for (int i = 0; i < 4; ++i)
                        if (ch[i] >= 0 && !(group_lb<T, PER>(g0, g1, bx[i]) > R)) {
                            if (ch[i] >= n - 1) kl |= 1u << i;
                            else ki |= 1u << i;
                        }
                }
                const int nl = __popc(kl), ni = __popc(ki);
                int       incl = nl | (ni << 16);
#pragma unroll
                for (int o = 1; o < 32; o <<= 1) {
                    const int v = __shfl_up_sync(FULL, incl, o);
                    if (lane >= o) incl += v;
                }
                const int tot = __shfl_sync(FULL, incl, 31);
                if (cc + (tot & 0xffff) > kGCand) flush();
                int pl = cc + (incl & 0xffff) - nl, pi = top + (incl >> 16) - ni;
#pragma unroll
                for (int i = 0; i < 4; ++i) {
                    if ((kl >> i) & 1u) {
                        if constexpr (FILT) {
                            g_cf[warp][pl] = make_float4((float)group_offset<T, PER>(bx[i][0], g0[0]),
                                                         (float)group_offset<T, PER>(bx[i][2], g0[1]),
                                                         (float)group_offset<T, PER>(bx[i][4], g0[2]),
                                                         __int_as_float(ch[i]));
                        } else {
                            g_cx[warp][pl] = bx[i][0];
                            g_cy[warp][pl] = bx[i][2];
                            g_cz[warp][pl] = bx[i][4];
                            g_cs[warp][pl] = ch[i];
                        }
                        ++pl;
                    }
                    if ((ki >> i) & 1u) g_stk[warp][pi++] = ch[i];
                }
                cc += tot & 0xffff;
                top += tot >> 16;
                __syncwarp();
            }
            if (overflow) flag = true;
            else flush();
        }
    }
    if constexpr (VAR == 2) {
        // per-lane walk over internal nodes only: leaf children go to the heap as soon as
        // their parent is expanded, the nearer internal child is walked next from registers
        // and only the farther one is stacked.  Every iteration is one expansion, so lanes
        // of a warp run the same instructions.
        int  sn[kFastStack];
        int  cur  = 0;
        bool have = active && n > 1 && needs(sd[0]);
        sp        = 0;
        while (have) {
            if (--budget < 0) {
                atomicOr(status, STATUS_TRAVERSAL_LIMIT);
                break;
            }
            ++visits;
            T   lb[6], rb[6];
            int l, r;
            load_rec<T, COH>(t.recs, cur, lb, rb, l, r);
            const D    ld2 = Metric<T>::template dist<(PER != 0), (PER == 2)>(px, py, pz, lb[0], lb[1], lb[2], lb[3], lb[4], lb[5]);
            const D    rd2 = Metric<T>::template dist<(PER != 0), (PER == 2)>(px, py, pz, rb[0], rb[1], rb[2], rb[3], rb[4], rb[5]);
            const bool lleaf = l >= n - 1, rleaf = r >= n - 1;
            if (lleaf && needs(ld2) && (l - (n - 1) < w0 || l - (n - 1) > w1) && l != self_leaf)
                insert(ld2, l - (n - 1));
            if (rleaf && needs(rd2) && (r - (n - 1) < w0 || r - (n - 1) > w1) && r != self_leaf)
                insert(rd2, r - (n - 1));
            const bool li = !lleaf && needs(ld2), ri = !rleaf && needs(rd2);
            if (li && ri) {
                const bool ln = ld2 <= rd2;
                if (sp >= kFastStack) {
                    atomicOr(status, STATUS_TRAVERSAL_LIMIT);
                    break;
                }
                sn[sp] = ln ? r : l;
                sd[sp] = ln ? rd2 : ld2;
                ++sp;
                cur = ln ? l : r;
            } else if (li) {
                cur = l;
            } else if (ri) {
                cur = r;
            } else {
                have = false;
                while (sp > 0) {
                    --sp;
                    if (needs(sd[sp])) {
                        cur  = sn[sp];
                        have = true;
                        break;
                    }
                }
            }
        }
        sp = 0;
    }
    if constexpr (VAR == 4 || VAR == 5) {
        // per-lane walk over the 4-wide records: each step evaluates up to four grandchildren
        // (half the dependent steps of the binary walk); leaves go to the heap, the nearest
        // needed internal node is walked next and the others are stacked farthest first.  A
        // full stack hands the query to the replay instead of dropping anything.
        constexpr int kWideStack = sizeof(lane_stack) / sizeof(lane_stack[0]);
        const int     ws0 = w0 + n - 1, ws1 = w1 + n - 1; // the seeding window in slot numbers
        // Children are judged, ordered and stacked by their keys (a key is at most the
        // distance, and within kthr whenever the distance is within thr): stack entries hold the
        // node index in the low word and its key in the high word (one 8-byte local-memory access
        // per push or pop), and a popped node is dropped only when its key exceeds kthr.
        unsigned long long *st = lane_stack;
        int           cur  = 0;
        int           wsp  = 0;
        bool          have = !group_done && active && n > 1 && needs(sd[0]);
        while (have) {
            if (--budget < 0) {
                atomicOr(status, STATUS_TRAVERSAL_LIMIT);
                break;
            }
            ++visits;
            T   bx[4][6];
            int ch[4];
            load_wide<T, COH>(t.wide, cur, bx, ch);
            D        d[4];
            H        kf[4]; // the distances' keys
            bool     in[4]; // needed internal child
            unsigned lm = 0; // leaves to offer to the heap
            auto needs_k = [&](H key) { return active && !(key > kthr); };
#pragma unroll
            for (int i = 0; i < 4; ++i) {
                d[i] = ch[i] >= 0 ? Metric<T>::template dist<(PER != 0), (PER == 2)>(
                                        px, py, pz, bx[i][0], bx[i][1], bx[i][2], bx[i][3], bx[i][4], bx[i][5])
                                  : dist_heap_max<D>();
                kf[i] = heap_key<T>(d[i]);
                const bool leaf = ch[i] >= n - 1;
                if (leaf && needs_k(kf[i]) && (ch[i] < ws0 || ch[i] > ws1) && ch[i] != self_leaf) lm |= 1u << i;
            }
            // one insertion site: lanes whose leaves sit at different child positions insert
            // together (the warp loops as often as its lane with the most leaves)
            while (lm) {
                const int i  = __ffs(lm) - 1;
                lm &= lm - 1;
                const D   di = i == 0 ? d[0] : i == 1 ? d[1] : i == 2 ? d[2] : d[3];
                const H   ki = i == 0 ? kf[0] : i == 1 ? kf[1] : i == 2 ? kf[2] : kf[3];
                const int ci = i == 0 ? ch[0] : i == 1 ? ch[1] : i == 2 ? ch[2] : ch[3];
                if (needs_k(ki)) insert_k(di, ki, ci - (n - 1)); // the threshold may have tightened
            }
#pragma unroll
            for (int i = 0; i < 4; ++i) in[i] = ch[i] >= 0 && ch[i] < n - 1 && needs_k(kf[i]);
            // order the needed internal children farthest first (4-element network on the keys;
            // children that are not needed, -1, sort behind the needed ones)
            int oc[4] = {ch[0], ch[1], ch[2], ch[3]};
            H   od[4];
#pragma unroll
            for (int i = 0; i < 4; ++i) od[i] = in[i] ? kf[i] : H(-1);
            auto cx = [&](int a, int b) {
                if (od[a] < od[b]) {
                    const int tc = oc[a];
                    const H   td = od[a];
                    oc[a]        = oc[b];
                    od[a]        = od[b];
                    oc[b]        = tc;
                    od[b]        = td;
                }
            };
            cx(0, 1);
            cx(2, 3);
            cx(0, 2);
            cx(1, 3);
            cx(1, 2);
            const int nv = (int)in[0] + (int)in[1] + (int)in[2] + (int)in[3];
            if (nv > 0) {
                if (wsp + nv - 1 > kWideStack) {
                    flag = true; // cannot stack them all: the reference traversal reruns the query
                    break;
                }
#pragma unroll
                for (int i = 0; i < 3; ++i)
                    if (i < nv - 1) {
                        st[wsp] = ((unsigned long long)__float_as_uint(od[i]) << 32) | (uint32_t)oc[i];
                        ++wsp;
                    }
                cur = nv == 1 ? oc[0] : nv == 2 ? oc[1] : nv == 3 ? oc[2] : oc[3];
            } else {
                have = false;
                while (wsp > 0) {
                    --wsp;
                    const unsigned long long e = st[wsp];
                    if (!(__uint_as_float((uint32_t)(e >> 32)) > kthr)) {
                        cur  = (int)(uint32_t)e;
                        have = true;
                        break;
                    }
                }
            }
        }
        sp = 0;
    }
    if constexpr (VAR == 1) {
        // per-lane walk: own stack, own near-first order (the reference's order)
        int sn[kFastStack];
        sn[0] = 0;
        if (!active) sp = 0;
        while (sp > 0) {
            if (--budget < 0) {
                atomicOr(status, STATUS_TRAVERSAL_LIMIT);
                break;
            }
            --sp;
            const int node = sn[sp];
            const D   d2   = sd[sp];
            if (!needs(d2)) continue;
            ++visits;
            if (node >= n - 1) {
                const int lr = node - (n - 1);
                if ((lr < w0 || lr > w1) && node != self_leaf) insert(d2, lr);
            } else {
                T   lb[6], rb[6];
                int l, r;
                load_rec<T, COH>(t.recs, node, lb, rb, l, r);
                const D ld2 = Metric<T>::template dist<(PER != 0), (PER == 2)>(px, py, pz, lb[0], lb[1], lb[2], lb[3], lb[4], lb[5]);
                const D rd2 = Metric<T>::template dist<(PER != 0), (PER == 2)>(px, py, pz, rb[0], rb[1], rb[2], rb[3], rb[4], rb[5]);
                if (sp + 2 > kFastStack) {
                    atomicOr(status, STATUS_TRAVERSAL_LIMIT);
                    break;
                }
                const bool ln = ld2 <= rd2;
                if (needs(ln ? rd2 : ld2)) {
                    sn[sp] = ln ? r : l;
                    sd[sp] = ln ? rd2 : ld2;
                    ++sp;
                }
                if (needs(ln ? ld2 : rd2)) {
                    sn[sp] = ln ? l : r;
                    sd[sp] = ln ? ld2 : rd2;
                    ++sp;
                }
            }
        }
        sp = 0;
    }
    constexpr bool SHARED = VAR == 0;
    if (SHARED && lane == 0) s_node[warp][0] = 0;
    __syncwarp();
    while (SHARED && sp > 0) {
        if (--budget < 0) {
            if (lane == 0) atomicOr(status, STATUS_TRAVERSAL_LIMIT);
            break;
        }
        --sp;
        const int  node = s_node[warp][sp];
        const D    d2   = sd[sp];
        const bool nd   = needs(d2);
        if (!__any_sync(FULL, nd)) continue;
        ++visits;
        if (node >= n - 1) {
            const int lr = node - (n - 1);
            // window leaves were already offered to the heap during seeding
            if (nd && (lr < w0 || lr > w1) && node != self_leaf) insert(d2, lr);
        } else {
            T   lb[6], rb[6];
            int l, r;
            load_rec<T, COH>(t.recs, node, lb, rb, l, r);
            const D  ld2 = Metric<T>::template dist<(PER != 0), (PER == 2)>(px, py, pz, lb[0], lb[1], lb[2], lb[3], lb[4], lb[5]);
            const D  rd2 = Metric<T>::template dist<(PER != 0), (PER == 2)>(px, py, pz, rb[0], rb[1], rb[2], rb[3], rb[4], rb[5]);
            const bool nl = needs(ld2), nr = needs(rd2);
            const unsigned bl = __ballot_sync(FULL, nl), br = __ballot_sync(FULL, nr);
            if (bl | br) {
                if (sp + 2 > kFastStack) {
                    if (lane == 0) atomicOr(status, STATUS_TRAVERSAL_LIMIT);
                    break;
                }
                const unsigned votes     = __ballot_sync(FULL, (nl || nr) && ld2 <= rd2);
                const bool     left_near = 2 * __popc(votes) >= __popc(bl | br);
                // push the farther child first so the nearer one is walked next
                const int  first = left_near ? r : l, second = left_near ? l : r;
                const D    fd = left_near ? rd2 : ld2, sd2 = left_near ? ld2 : rd2;
                const bool fneed = left_near ? (br != 0) : (bl != 0);
                const bool sneed = left_near ? (bl != 0) : (br != 0);
                if (fneed) {
                    if (lane == 0) s_node[warp][sp] = first;
                    sd[sp] = fd;
                    ++sp;
                }
                if (sneed) {
                    if (lane == 0) s_node[warp][sp] = second;
                    sd[sp] = sd2;
                    ++sp;
                }
                __syncwarp();
            }
        }
    }

    // visit statistics: lane-node evaluations summed per warp
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) visits += __shfl_down_sync(FULL, visits, off);
    if (lane == 0 && visit_count) atomicAdd(visit_count, (unsigned long long)visits);

    // ---- 3. sort, check, write ----
    // a bound that proved too small: the bound may have cut a neighbour, or fewer than k
    // points lie inside it.  With a miss list the query goes to the next launch (the walk
    // without a bound); otherwise the reference traversal reruns it.
    // (k-th key not below the bound's key: the k-th distance may exceed the bound)
    const bool bound_miss =
        active && B != dist_heap_max<D>() && (count < k || !(hk < heap_key<T>(B)));
    if (miss.rows) {
        const uint32_t at = warp_append(miss.count, bound_miss, lane);
        if (bound_miss) {
            if (!ext && !bt.off) miss.ranks[at] = rank;
            miss.rows[at] = q;
            active        = false;
        }
    }
    if (active) {
        if (bound_miss) flag = true;
        // trees of height >= 63: the reference's stack guard may drop part of this query's
        // neighbourhood (fewer than k points found: conservatively so)
        if (!flag && n >= 2 && (int)t.height[0] >= 63 &&
            (count < k || stack_guard_reaches<T, PER, COH>(t, px, py, pz, hmax, lane_stack)))
            flag = true;
        for (int hs = count; hs > 1; --hs) {
            H       last  = HD(hs - 1);
            int32_t lasti = HI(hs - 1);
            HD(hs - 1)    = HD(0);
            HI(hs - 1)    = HI(0);
            const int size = hs - 1;
            int       i    = 0;
            for (;;) {
                int l = 2 * i + 1;
                if (l >= size) break;
                int r  = l + 1;
                int c  = i;
                H   cd = last;
                H   ld = HD(l);
                if (ld > cd) {
                    c  = l;
                    cd = ld;
                }
                if (r < size) {
                    H rd = HD(r);
                    if (rd > cd) {
                        c  = r;
                        cd = rd;
                    }
                }
                if (c == i) break;
                HD(i) = cd;
                HI(i) = HI(c);
                i     = c;
            }
            HD(i) = last;
            HI(i) = lasti;
        }
        if constexpr (heap_keyed<T>()) {
            // runs of equal keys inside the top k: the exact distances order them (the exact
            // order refines the key order); only an exact tie can differ from the reference
            for (int i = 1; i < count; ++i) {
                for (int j = i; j > 0 && HD(j) == HD(j - 1); --j) {
                    const D a = exact(HI(j - 1)), b = exact(HI(j));
                    if (!(b < a)) { // in order, or equal (or not comparable): a tie
                        if (!(a < b)) flag = true;
                        break;
                    }
                    const int32_t tmp = HI(j);
                    HI(j)             = HI(j - 1);
                    HI(j - 1)         = tmp;
                }
            }
        } else {
            // equal distances: their order may differ from the reference's
            for (int i = 1; i < count; ++i)
                if (HD(i) == HD(i - 1)) flag = true;
        }
        const size_t off = (size_t)q * (size_t)k;
        for (int i = 0; i < k; ++i) {
            if (i < count) {
                const int32_t leaf = HI(i);
                const int     s    = leaf + n - 1;
                D             dd;
                if constexpr (heap_keyed<T>()) {
                    // the exact distance, as the walk computed it (a leaf's box is its point)
                    const T x = t.min_x[s], y = t.min_y[s], z = t.min_z[s];
                    dd = Metric<T>::template dist<(PER != 0), (PER == 2)>(px, py, pz, x, x, y, y, z, z);
                } else {
                    dd = (D)HD(i);
                }
                __stcs(out_idx + off + i, (unsigned long long)(long long)(ret_orig ? t.orig_idx[s] : leaf));
                __stcs(out_dist + off + i, dd);
            } else {
                __stcs(out_idx + off + i, ~0ull);
                __stcs(out_dist + off + i, dist_missing<D>());
            }
        }
    }
    const bool to_replay = (active && flag) || force_replay;
    const uint32_t at    = warp_append(replay_count, to_replay, lane);
    if (to_replay) {
        if (!ext) replay_ranks[at] = rank;
        replay_rows[at] = q;
    }
#undef HD
#undef HI
}

// The fast walk over queries [0, num), one warp per 32 queries; or, with a list, a grid-stride
// loop over the list's entries (the count lives on the device: no host synchronisation).
// Resident blocks the 4-wide walk is compiled for (a register budget): its 8-byte heap entries
// leave room for more blocks than the registers it would otherwise take.
template <class T, int KC, int VAR> constexpr int fast_min_blocks() {
    // (VAR 4 with k <= 32 and integer coordinates only: the other shapes keep the registers
    // they take; the float64 walk spills under this budget, 0.52 against 0.40 ms on 100K points)
    return (VAR == 4 && KC <= 32 && !Coord<T>::is_float) ? FT_FAST_MINB : 1;
}
template <class T, int PER, int KC, int VAR, bool XB = false>
__global__ void __launch_bounds__(32 * fast_warps<KC>(), fast_min_blocks<T, KC, VAR>())
    fast_self_knn_kernel(QueryList lst, MissList miss, TreeDev<T> t_all, BatchDev bt, const T *__restrict__ qx,
                         const T *__restrict__ qy, const T *__restrict__ qz, const uint32_t *__restrict__ order,
                         const int32_t *__restrict__ leaf_ids, int num, int k, int half_window, int exclude_self,
                         int ret_orig, const typename Coord<T>::dist_t *__restrict__ bound,
                         unsigned long long *__restrict__ out_idx, typename Coord<T>::dist_t *__restrict__ out_dist,
                         int32_t *__restrict__ replay_ranks, int32_t *__restrict__ replay_rows,
                         uint32_t *replay_count, uint32_t *status, unsigned long long *visit_count) {
    constexpr int W = fast_warps<KC>();
    extern __shared__ __align__(16) unsigned char smem[];
    const int warp = threadIdx.x >> 5;
    const int first = (blockIdx.x * W + warp) * 32;
    if (!lst.count) {
        fast_warp<T, PER, KC, VAR, fast_warps<KC>(), false, XB>(first, lst, miss, smem, t_all, bt, qx, qy, qz, order, leaf_ids, num, k,
                                   half_window, exclude_self, ret_orig, bound, out_idx, out_dist, replay_ranks,
                                   replay_rows, replay_count, status, visit_count);
        return;
    }
    const int cnt = (int)*lst.count;
    for (int base = first; base < cnt; base += gridDim.x * W * 32)
        fast_warp<T, PER, KC, VAR, fast_warps<KC>(), false, XB>(base, lst, miss, smem, t_all, bt, qx, qy, qz, order, leaf_ids, cnt, k,
                                   half_window, exclude_self, ret_orig, bound, out_idx, out_dist, replay_ranks,
                                   replay_rows, replay_count, status, visit_count);
}

// -----------------------------------------------------------------------------------------
// External query points: qx / qy / qz (else self queries) with leaf_ids = their seed ranks.
struct ExtQueries {
    const void     *x = nullptr, *y = nullptr, *z = nullptr;
    const uint32_t *order = nullptr; // walk order (null: input order)
};

// Walk of the fast path: caller's 0 = default, 1 per-lane binary walk, 2 compact per-lane
// binary walk, 3 warp-shared walk, 4 the 4-wide walk, 5 the group walk.  The default is the 4-wide walk, and
// the compact binary walk for k <= 4 (measured on 10M clustered points: k = 32 64.2 against
// 66.8 ms, k = 1 10.2 against 9.2 ms).  Returns the kernel's VAR template value.
static int walk_variant(int v, int k) {
    switch (v) {
    case 1: return 1;
    case 2: return 2;
    case 3: return 0;
    case 4: return 4;
    case 5: return 5;
    default: return k <= 4 ? 2 : 4;
    }
}

template <class T, int PER, int KC>
static void launch_fast_t(const TreeDev<T> &tv, const BatchDev &bt, const ExtQueries &eq, const int32_t *leaf_ids,
                          int num, int k, int half, bool excl, bool ro, const void *bound, uint64_t *idx, void *dist,
                          int32_t *rr, int32_t *rw, uint32_t *rc, uint32_t *status, int variant,
                          unsigned long long *visits, cudaStream_t st, const ListArgs &la) {
    using D     = typename Coord<T>::dist_t;
    constexpr int threads = 32 * fast_warps<KC>();
    size_t        smem    = (size_t)std::max(k, 1) * threads * (sizeof(heap_dist_t<T>) + 4); // heaps of k entries
    // the k-th key settled exactly (XB) for external queries, whose replay is knn_query's heap
    // tier, and for short launches, where one replay's latency outweighs the settling code
    const bool xb = eq.x != nullptr || num <= FT_XB_MAX_QUERIES;
    auto   fn   = variant == 0 ? fast_self_knn_kernel<T, PER, KC, 0>
                  : variant == 1 ? fast_self_knn_kernel<T, PER, KC, 1>
                  : variant == 4 ? (xb ? fast_self_knn_kernel<T, PER, KC, 4, true> : fast_self_knn_kernel<T, PER, KC, 4>)
                  : variant == 5 ? fast_self_knn_kernel<T, PER, KC, 5>
                                 : fast_self_knn_kernel<T, PER, KC, 2>;
    FT_CUDA(cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    // a listed launch (num: the list's capacity) loops over its entries with a grid of a few
    // blocks per SM; otherwise one warp per 32 queries
    int blocks = (num + threads - 1) / threads;
    if (la.lst.count) blocks = std::max(1, std::min(blocks, 148 * 8));
    fn<<<blocks, threads, smem, st>>>(la.lst, la.miss, tv, bt, (const T *)eq.x, (const T *)eq.y, (const T *)eq.z,
                                      eq.order, leaf_ids, num, k, half, excl ? 1 : 0, ro ? 1 : 0, (const D *)bound,
                                      (unsigned long long *)idx, (D *)dist, rr, rw, rc, status, visits);
    FT_CUDA(cudaGetLastError());
}

// Launches the fast walk over `tv` (one tree, or every set of a batch when bt.off is set).
template <class T>
static void launch_fast_view(const TreeDev<T> &tv, const BatchDev &bt, int met, bool ro, const int32_t *leaf_ids,
                             int num, int k, int half, bool excl, const void *bound, uint64_t *idx, void *dist,
                             int32_t *rr, int32_t *rw, uint32_t *rc, uint32_t *status, int variant,
                             unsigned long long *visits, cudaStream_t st, const ExtQueries &eq = {},
                             const ListArgs &la = {}, int kc = 0) {
    met_dispatch<T>(met, [&](auto M) {
        constexpr int PER = decltype(M)::value;
        // heap template: 32 (two-warp blocks) for k <= 32 unless one-warp blocks were chosen
        if (k <= 32 && kc != 64)
            launch_fast_t<T, PER, 32>(tv, bt, eq, leaf_ids, num, k, half, excl, ro, bound, idx, dist, rr, rw, rc,
                                      status, variant, visits, st, la);
        else
            launch_fast_t<T, PER, 64>(tv, bt, eq, leaf_ids, num, k, half, excl, ro, bound, idx, dist, rr, rw, rc,
                                      status, variant, visits, st, la);
    });
}

template <class T>
static void launch_fast(const ft_options &o, const ft_tree &tr, const int32_t *leaf_ids, int num, int k, int half,
                        bool excl, const void *bound, uint64_t *idx, void *dist, int32_t *rr, int32_t *rw,
                        uint32_t *rc, uint32_t *status, int variant, unsigned long long *visits, cudaStream_t st,
                        const ExtQueries &eq = {}, const ListArgs &la = {}, int kc = 0) {
    launch_fast_view<T>(tree_view<T>(tr), BatchDev{}, metric_mode<T>(o, tr), o.return_orig_indices != 0, leaf_ids,
                        num, k, half, excl, bound, idx, dist, rr, rw, rc, status, variant, visits, st, eq, la, kc);
}

// Every coordinate type: launch_fast<T> for the context's type.
static void launch_fast_any(const ft_options &o, const ft_tree &tr, const int32_t *leaf_ids, int num, int k, int half,
                            bool excl, const void *bound, uint64_t *idx, void *dist, int32_t *rr, int32_t *rw,
                            uint32_t *rc, uint32_t *status, int variant, unsigned long long *visits, cudaStream_t st,
                            const ExtQueries &eq = {}, const ListArgs &la = {}, int kc = 0) {
    switch (o.coord_type) {
    case F32: launch_fast<float>(o, tr, leaf_ids, num, k, half, excl, bound, idx, dist, rr, rw, rc, status, variant, visits, st, eq, la, kc); break;
    case F64: launch_fast<double>(o, tr, leaf_ids, num, k, half, excl, bound, idx, dist, rr, rw, rc, status, variant, visits, st, eq, la, kc); break;
    case U32: launch_fast<uint32_t>(o, tr, leaf_ids, num, k, half, excl, bound, idx, dist, rr, rw, rc, status, variant, visits, st, eq, la, kc); break;
    case U64: launch_fast<unsigned long long>(o, tr, leaf_ids, num, k, half, excl, bound, idx, dist, rr, rw, rc, status, variant, visits, st, eq, la, kc); break;
    }
}

// SFC rank of external query points: the point's key (the tree's own encoding and box) and
// its lower bound among the sorted keys; -1 without usable keys.
template <class T, int SFC>
__global__ void __launch_bounds__(256)
    seed_rank_kernel(const T *__restrict__ qx, const T *__restrict__ qy, const T *__restrict__ qz, int nq,
                     const T *__restrict__ bbox, const unsigned long long *__restrict__ klo,
                     const unsigned long long *__restrict__ khi, int n, int32_t *out) {
    __shared__ uint8_t s_rot[48 * 8], s_sub[48 * 8];
    __shared__ T       s_par[6];
    for (int i = threadIdx.x; i < 48 * 8; i += blockDim.x) {
        s_rot[i] = c_rot[i];
        s_sub[i] = c_sub[i];
    }
    if constexpr (Coord<T>::is_float)
        if (threadIdx.x < 3)
            sfc_axis_params(bbox[2 * threadIdx.x], bbox[2 * threadIdx.x + 1], s_par[2 * threadIdx.x],
                            s_par[2 * threadIdx.x + 1]);
    __syncthreads();
    const bool wide = Coord<T>::key_words == 2;
    for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < nq; q += gridDim.x * blockDim.x) {
        unsigned long long hi, lo;
        encode_point<T, SFC>(qx[q], qy[q], qz[q], s_par, s_rot, s_sub, hi, lo);
        int a = 0, b = n; // first j with key[j] >= key
        while (a < b) {
            const int  m    = (a + b) >> 1;
            const bool less = wide ? (khi[m] < hi || (khi[m] == hi && klo[m] < lo)) : (klo[m] < lo);
            if (less) a = m + 1;
            else b = m;
        }
        out[q] = a;
    }
}

template <class T>
static void seed_ranks(const ft_options &o, const TreeImpl &impl, const void *qx, const void *qy, const void *qz,
                       int nq, int n, int32_t *out, cudaStream_t st) {
    const int grid = std::max(1, std::min((nq + 255) / 256, 148 * 16));
    if (o.sfc_type == MORTON)
        seed_rank_kernel<T, MORTON><<<grid, 256, 0, st>>>((const T *)qx, (const T *)qy, (const T *)qz, nq,
                                                          (const T *)impl.bbox, (const unsigned long long *)impl.key_lo,
                                                          (const unsigned long long *)impl.key_hi, n, out);
    else
        seed_rank_kernel<T, PEANO_HILBERT><<<grid, 256, 0, st>>>(
            (const T *)qx, (const T *)qy, (const T *)qz, nq, (const T *)impl.bbox,
            (const unsigned long long *)impl.key_lo, (const unsigned long long *)impl.key_hi, n, out);
    FT_CUDA(cudaGetLastError());
}

// Bound-miss list of the context (queries whose bound proved too small in the first launch).
static void ensure_miss(Context &ctx, size_t num) {
    if (num <= ctx.miss_cap && ctx.miss_ranks) return;
    if (ctx.miss_ranks) cudaFree(ctx.miss_ranks);
    if (ctx.miss_rows) cudaFree(ctx.miss_rows);
    ctx.miss_ranks = ctx.miss_rows = nullptr;
    ctx.miss_cap                   = 0;
    const size_t cap = num + num / 4 + 1024;
    FT_CUDA(cudaMalloc(&ctx.miss_ranks, cap * sizeof(int32_t)));
    FT_CUDA(cudaMalloc(&ctx.miss_rows, cap * sizeof(int32_t)));
    ctx.miss_cap = cap;
}

// The fast walk over num queries (self queries, or external points with eq), its replay, and
// with a per-query bound a second launch of the walk without the bound over the queries
// whose bound proved too small (the walk flags its own ties there, so only those reach the
// reference traversal).  Counters in the context's status words: [1] replayed, [2..3]
// visits, [4] bound misses, [6..7] visits of the second launch.
static void fast_walk_and_replay(Context &ctx, const ft_tree &tr, const int32_t *leaf_ids, size_t num, int k,
                                 bool excl, uint64_t *idx, void *dist, const void *bound, int half_window,
                                 int variant, cudaStream_t st, const ExtQueries &eq = {}, int kc = 0) {
    uint32_t           *rc     = ctx.status + 1;
    unsigned long long *visits = (unsigned long long *)(ctx.status + 2);
    uint32_t           *mc     = ctx.status + 4;
    FT_CUDA(cudaMemsetAsync(rc, 0, 7 * sizeof(uint32_t), st));
    ListArgs la;
    if (bound) {
        ensure_miss(ctx, num);
        la.miss = MissList{ctx.miss_ranks, ctx.miss_rows, mc};
    }
    launch_fast_any(ctx.opts, tr, leaf_ids, (int)num, k, half_window, excl, bound, idx, dist, ctx.replay_ranks,
                    ctx.replay_rows, rc, ctx.status, variant, visits, st, eq, la, kc);
    if (bound) {
        ListArgs again;
        again.lst = QueryList{ctx.miss_ranks, ctx.miss_rows, mc};
        launch_fast_any(ctx.opts, tr, leaf_ids, (int)num, k, half_window, excl, nullptr, idx, dist, ctx.replay_ranks,
                        ctx.replay_rows, rc, ctx.status, variant, (unsigned long long *)(ctx.status + 6), st, eq,
                        again, kc);
    }
}

bool fast_self_knn(Context &ctx, const ft_tree &tr, const int32_t *leaf_ids, size_t num, int k, bool excl,
                   uint64_t *idx, void *dist, const void *bound, int half_window, int variant, cudaStream_t st,
                   int kc) {
    TreeImpl *impl = (TreeImpl *)tr.impl;
    if (k > 64 || tr.num_leaves < 2 || !impl || impl->height_root < 0) return false;
    if (!fast_walk_applies(ctx.opts, *impl)) return false;
    // the autotuner's choice for this shape; it was made on every leaf in SFC order, so a
    // subset (whose warps hold unrelated leaves) keeps the defaults
    if (half_window <= 0 && variant <= 0 && kc <= 0 && !leaf_ids) {
        auto it = ctx.tuned.find(tune_key(TUNE_SELF_KNN, k, tr.num_leaves));
        if (it != ctx.tuned.end()) {
            half_window = it->second.half;
            variant     = it->second.variant;
            kc          = it->second.kc;
        }
    }
    if (half_window <= 0) half_window = k;
    variant = walk_variant(variant, k);
    ensure_replay(ctx, num);
    fast_walk_and_replay(ctx, tr, leaf_ids, num, k, excl, idx, dist, bound, half_window, variant, st, {}, kc);
    replay_exact(ctx, tr, ctx.replay_ranks, ctx.replay_rows, ctx.status + 1, k, excl, idx, dist, st);
    return true;
}

// (seed rank, query index) pairs for the query sort.
__global__ void rank_pairs_kernel(const int32_t *__restrict__ seeds, int nq, unsigned long long *key, uint32_t *perm) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < nq; i += gridDim.x * blockDim.x) {
        key[i]  = (unsigned long long)(uint32_t)seeds[i];
        perm[i] = (uint32_t)i;
    }
}

// Sort scratch for external queries (one key word, nq pairs); status words go to the context.
static void ensure_query_sort(Context &ctx, size_t nq) {
    TreeImpl &s = ctx.qsort;
    if (nq <= s.cap && s.key_lo) return;
    void *ptrs[] = {s.key_lo, s.tmp_lo, s.perm, s.tmp_perm, s.hist, s.lookback, s.tile_counter};
    for (void *p : ptrs)
        if (p) cudaFree(p);
    s            = TreeImpl{};
    const size_t cap = nq + nq / 4 + 1024;
    auto alloc = [&](size_t bytes) {
        void       *p = nullptr;
        cudaError_t e = cudaMalloc(&p, bytes);
        if (e != cudaSuccess) {
            cudaGetLastError();
            fail(FT_ERR_OUT_OF_MEMORY, "cudaMalloc of the query sort scratch failed");
        }
        return p;
    };
    s.key_lo         = (uint64_t *)alloc(cap * 8);
    s.tmp_lo         = (uint64_t *)alloc(cap * 8);
    s.perm           = (uint32_t *)alloc(cap * 4);
    s.tmp_perm       = (uint32_t *)alloc(cap * 4);
    s.hist           = (uint32_t *)alloc((16 * 256 + 16) * 4);
    s.lookback_words = sort_lookback_words(cap, 1);
    s.lookback       = (uint32_t *)alloc(s.lookback_words * 4);
    s.tile_counter   = (uint32_t *)alloc(16 * 4);
    s.cap            = cap;
}

void free_query_sort(Context &ctx) {
    TreeImpl &s      = ctx.qsort;
    void     *ptrs[] = {s.key_lo, s.tmp_lo, s.perm, s.tmp_perm, s.hist, s.lookback, s.tile_counter};
    for (void *p : ptrs)
        if (p) cudaFree(p);
    s = TreeImpl{};
}

// SFC rank of each external query in ctx.seed_ranks (-1 without usable keys).
static bool compute_seed_ranks(Context &ctx, const ft_tree &tr, const void *qx, const void *qy, const void *qz,
                               size_t nq, cudaStream_t st) {
    TreeImpl *impl = (TreeImpl *)tr.impl;
    ensure_replay(ctx, nq);
    const int n = (int)tr.num_leaves;
    if (!(impl->own_keys && impl->key_lo)) {
        FT_CUDA(cudaMemsetAsync(ctx.seed_ranks, 0xFF, nq * sizeof(int32_t), st)); // -1: no seeding window
        return false;
    }
    switch (ctx.opts.coord_type) {
    case F32: seed_ranks<float>(ctx.opts, *impl, qx, qy, qz, (int)nq, n, ctx.seed_ranks, st); break;
    case F64: seed_ranks<double>(ctx.opts, *impl, qx, qy, qz, (int)nq, n, ctx.seed_ranks, st); break;
    case U32: seed_ranks<uint32_t>(ctx.opts, *impl, qx, qy, qz, (int)nq, n, ctx.seed_ranks, st); break;
    case U64: seed_ranks<unsigned long long>(ctx.opts, *impl, qx, qy, qz, (int)nq, n, ctx.seed_ranks, st); break;
    }
    return true;
}

void query_seed_ranks(Context &ctx, const ft_tree &tr, const void *qx, const void *qy, const void *qz, size_t nq,
                      cudaStream_t st) {
    compute_seed_ranks(ctx, tr, qx, qy, qz, nq, st);
}

// Query order by SFC rank (ctx.seed_ranks must hold the ranks): sorts (rank, index) pairs.
static const uint32_t *order_by_rank(Context &ctx, size_t nq, int n, cudaStream_t st) {
    ensure_query_sort(ctx, nq);
    TreeImpl &qs = ctx.qsort;
    qs.status    = ctx.status;
    rank_pairs_kernel<<<std::max(1, std::min((int)((nq + 255) / 256), 148 * 16)), 256, 0, st>>>(
        ctx.seed_ranks, (int)nq, (unsigned long long *)qs.key_lo, qs.perm);
    FT_CUDA(cudaGetLastError());
    int bytes = 1;
    while (bytes < 4 && ((unsigned long long)n >> (8 * bytes)) != 0) ++bytes;
    static const int digits[4] = {0, 1, 2, 3};
    sort_pairs_fixed(qs, nq, 1, bytes, digits, st);
    return qs.perm;
}

const uint32_t *sfc_query_order(Context &ctx, const ft_tree &tr, const void *qx, const void *qy, const void *qz,
                                size_t nq, cudaStream_t st) {
    if (nq < 2 || tr.num_leaves < 2 || !tr.impl) return nullptr;
    if (!compute_seed_ranks(ctx, tr, qx, qy, qz, nq, st)) return nullptr;
    return order_by_rank(ctx, nq, (int)tr.num_leaves, st);
}

bool fast_knn(Context &ctx, const ft_tree &tr, const void *qx, const void *qy, const void *qz, size_t nq, int k,
              int max_k, uint64_t *idx, void *dist, int half_window, cudaStream_t st, const void *bound,
              int walk) {
    TreeImpl *impl = (TreeImpl *)tr.impl;
    if (k > 64 || tr.num_leaves < 2 || !impl || impl->height_root < 0) return false;
    if (!fast_walk_applies(ctx.opts, *impl)) return false;
    // SortedMergeHeap with k equal to its capacity keeps the first k leaves it meets, not the
    // nearest: only the reference traversal reproduces that
    int cap = 1;
    while (cap < max_k) cap <<= 1;
    if (k > 32 && max_k > 32 && k >= cap) return false;
    if (half_window <= 0) half_window = k;
    const int  n      = (int)tr.num_leaves;
    const bool ranked = compute_seed_ranks(ctx, tr, qx, qy, qz, nq, st);
    ExtQueries eq;
    eq.x = qx;
    eq.y = qy;
    eq.z = qz;
    if (ranked && nq > 1) eq.order = order_by_rank(ctx, nq, n, st); // walk the queries in SFC order
    const int variant = walk_variant(walk, k);
    fast_walk_and_replay(ctx, tr, ctx.seed_ranks, nq, k, false, idx, dist, bound, half_window, variant, st, eq);
    replay_external(ctx, tr, qx, qy, qz, ctx.replay_rows, ctx.status + 1, k, max_k, idx, dist, st);
    return true;
}

void batch_self_knn(Context &ctx, const ft_tree &all, const BatchDev &bt, size_t num, int k, bool excl, uint64_t *idx,
                    void *dist, bool fast, int half_window, int variant, int32_t *rr, int32_t *rw, uint32_t *counters,
                    cudaStream_t st, const void *bound, int32_t *mw, int kc) {
    if (num == 0 || k <= 0) return;
    if (!fast || k > 64) {
        batch_self_knn_exact(ctx, all, bt, num, k, excl, idx, dist, st);
        return;
    }
    if (half_window <= 0 && variant <= 0 && kc <= 0) { // the autotuner's choice for this shape
        auto it = ctx.tuned.find(tune_key(TUNE_BATCH, k, num));
        if (it != ctx.tuned.end()) {
            half_window = it->second.half;
            variant     = it->second.variant;
            kc          = it->second.kc;
        }
    }
    if (half_window <= 0) half_window = k;
    variant                        = walk_variant(variant, k);
    unsigned long long *visits     = (unsigned long long *)(counters + 2);
    const bool          ro         = ctx.opts.return_orig_indices != 0;
    const int           n          = (int)num;
    FT_CUDA(cudaMemsetAsync(counters, 0, 8 * sizeof(uint32_t), st));
    ListArgs first, again;
    if (bound) { // bound misses: leaf ranks follow from the rows inside a batch, so rows suffice
        first.miss = MissList{nullptr, mw, counters + 4};
        again.lst  = QueryList{nullptr, mw, counters + 4};
    }
#define FT_BF(T, B, LA)                                                                                            \
    launch_fast_view<T>(tree_view<T>(all), bt, metric_mode<T>(ctx.opts, all), ro, nullptr, n, k, half_window, excl, \
                        B, idx, dist, rr, rw, counters, ctx.status, variant, visits, st, ExtQueries{}, LA, kc)
    for (int pass = 0; pass < (bound ? 2 : 1); ++pass) {
        const void     *b  = pass == 0 ? bound : nullptr;
        const ListArgs &la = pass == 0 ? first : again;
        if (pass == 1) visits = (unsigned long long *)(counters + 6); // the rerun's visits apart
        switch (ctx.opts.coord_type) {
        case F32: FT_BF(float, b, la); break;
        case F64: FT_BF(double, b, la); break;
        case U32: FT_BF(uint32_t, b, la); break;
        case U64: FT_BF(unsigned long long, b, la); break;
        }
    }
#undef FT_BF
    replay_exact(ctx, all, rr, rw, counters, k, excl, idx, dist, st, bt);
}

void ensure_replay(Context &ctx, size_t num) {
    if (num <= ctx.replay_cap && ctx.replay_ranks) return;
    if (ctx.replay_ranks) cudaFree(ctx.replay_ranks);
    if (ctx.replay_rows) cudaFree(ctx.replay_rows);
    if (ctx.seed_ranks) cudaFree(ctx.seed_ranks);
    ctx.replay_ranks = ctx.replay_rows = ctx.seed_ranks = nullptr;
    ctx.replay_cap                                       = 0;
    size_t cap = num + num / 4 + 1024;
    FT_CUDA(cudaMalloc(&ctx.replay_ranks, cap * sizeof(int32_t)));
    FT_CUDA(cudaMalloc(&ctx.replay_rows, cap * sizeof(int32_t)));
    FT_CUDA(cudaMalloc(&ctx.seed_ranks, cap * sizeof(int32_t)));
    ctx.replay_cap = cap;
}

// =========================================================================================
// Self-kNN without any device allocation (ft_self_knn_noalloc).
//
// Some callers cannot let a library allocate device memory in the middle of their work: a
// simulation that hands the whole GPU to its own memory pool at start-up (a cudaMalloc then
// fails), or a time step that must not stall every stream (cudaMalloc / cudaFree
// synchronise the device).  This variant runs the fast self-kNN walk with its only scratch
// -- the list of queries handed to the exact replay and its counter -- in the fixed array
// below, instead of the context's growable buffers.
//
// * The array lives in every GPU that loads the library, for the life of the process:
//   kNoAllocMaxQueries (2^20) queries per call, 8 MiB + a small header.  Larger calls are
//   rejected with FT_ERR_INVALID_ARGUMENT.
// * Host code needs the array's device address: the first call on a device looks it up
//   with cudaGetSymbolAddress (with that device current) and keeps it; make that first call
//   before any stream capture.  The symbol itself is only a host-side stand-in, never a
//   device pointer.
// * All calls share the array.  Each call clears the counter it needs on its stream first;
//   calls whose work overlaps on the GPU (different streams, or threads racing on one
//   device) race on the array and must be serialised by the caller.
// =========================================================================================
static constexpr size_t kNoAllocMaxQueries = size_t(1) << 20;
static constexpr size_t kNoAllocHeader     = 64; // words: [0] replay count, [2..3] visit counter
static __device__ __align__(256) uint32_t g_noalloc_scratch[kNoAllocHeader + 2 * kNoAllocMaxQueries];

static constexpr int kNoAllocMaxDevices = 64;
static std::mutex    g_noalloc_mutex;
static uint32_t     *g_noalloc_addr[kNoAllocMaxDevices] = {};
static CUcontext     g_noalloc_owner[kNoAllocMaxDevices] = {}; // the context the address belongs to

// The current driver context, read through the runtime's driver entry point (the library
// links no driver library); null when it cannot be read.
static CUcontext current_context() {
    using GetCurrent = CUresult (*)(CUcontext *);
    static GetCurrent fn = [] {
        void                           *p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &p, cudaEnableDefault, &q) != cudaSuccess ||
            q != cudaDriverEntryPointSuccess) {
            cudaGetLastError();
            p = nullptr;
        }
        return reinterpret_cast<GetCurrent>(p);
    }();
    CUcontext c = nullptr;
    if (!fn || fn(&c) != CUDA_SUCCESS) return nullptr;
    return c;
}

// Device address of g_noalloc_scratch on `device` (device must be current).  Looked up on
// the first call on a device and again whenever the device's context has changed since (a
// cudaDeviceReset makes a new primary context, which holds its own copy of the array).
static uint32_t *noalloc_scratch(int device) {
    if (device < 0 || device >= kNoAllocMaxDevices) fail(FT_ERR_INVALID_ARGUMENT, "device ordinal out of range");
    std::lock_guard<std::mutex> lock(g_noalloc_mutex);
    const CUcontext cur = current_context();
    if (!g_noalloc_addr[device] || cur == nullptr || cur != g_noalloc_owner[device]) {
        void       *p = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess || p == nullptr) {
            cudaGetLastError();
            fail(FT_ERR_CUDA, std::string("cudaGetSymbolAddress of the no-allocation scratch failed: ") +
                                  cudaGetErrorString(e));
        }
        g_noalloc_addr[device]  = static_cast<uint32_t *>(p);
        g_noalloc_owner[device] = cur;
    }
    return g_noalloc_addr[device];
}

size_t noalloc_max_queries() { return kNoAllocMaxQueries; }

// Returns false when the fast walk does not apply (k > 64); the
// caller then runs the reference traversal, which needs no scratch.
bool fast_self_knn_noalloc(Context &ctx, const ft_tree &tr, const int32_t *leaf_ids, size_t num, int k, bool excl,
                           uint64_t *idx, void *dist, cudaStream_t st) {
    if (num > kNoAllocMaxQueries)
        fail(FT_ERR_INVALID_ARGUMENT, "ft_self_knn_noalloc: more than 1048576 queries in one call (the fixed "
                                      "scratch holds 2^20); split the call");
    TreeImpl *impl = (TreeImpl *)tr.impl;
    if (k > 64 || tr.num_leaves < 2 || !impl || impl->height_root < 0) return false;
    if (!fast_walk_applies(ctx.opts, *impl)) return false;
    uint32_t           *s      = noalloc_scratch(ctx.device);
    uint32_t           *rc     = s;
    unsigned long long *visits = reinterpret_cast<unsigned long long *>(s + 2);
    int32_t            *ranks  = reinterpret_cast<int32_t *>(s + kNoAllocHeader);
    int32_t            *rows   = ranks + kNoAllocMaxQueries;
    FT_CUDA(cudaMemsetAsync(s, 0, 4 * sizeof(uint32_t), st)); // the replay count must start at zero
    const int half = k, variant = walk_variant(0, k);
    switch (ctx.opts.coord_type) {
    case F32: launch_fast<float>(ctx.opts, tr, leaf_ids, (int)num, k, half, excl, nullptr, idx, dist, ranks, rows, rc, ctx.status, variant, visits, st); break;
    case F64: launch_fast<double>(ctx.opts, tr, leaf_ids, (int)num, k, half, excl, nullptr, idx, dist, ranks, rows, rc, ctx.status, variant, visits, st); break;
    case U32: launch_fast<uint32_t>(ctx.opts, tr, leaf_ids, (int)num, k, half, excl, nullptr, idx, dist, ranks, rows, rc, ctx.status, variant, visits, st); break;
    case U64: launch_fast<unsigned long long>(ctx.opts, tr, leaf_ids, (int)num, k, half, excl, nullptr, idx, dist, ranks, rows, rc, ctx.status, variant, visits, st); break;
    }
    replay_exact(ctx, tr, ranks, rows, rc, k, excl, idx, dist, st);
    // query statistics as ft_self_knn keeps them: the replay count and visits move into the
    // context's status words (a device-to-device copy on the stream; nothing is allocated)
    // (scratch words: [0] replay count, [2..3] visits; context words: [1] and [2..3])
    FT_CUDA(cudaMemcpyAsync(ctx.status + 1, rc, sizeof(uint32_t), cudaMemcpyDeviceToDevice, st));
    FT_CUDA(cudaMemcpyAsync(ctx.status + 2, visits, sizeof(unsigned long long), cudaMemcpyDeviceToDevice, st));
    FT_CUDA(cudaMemsetAsync(ctx.status + 4, 0, 4 * sizeof(uint32_t), st)); // no bound, no bound misses
    ctx.stats.queries  = (int64_t)num;
    ctx.stats.replayed = 0;
    ctx.last_fast      = true;
    ctx.last_rows      = false; // the replayed rows stay in the fixed array
    return true;
}

// =========================================================================================
// Persistent batched launch: build every set and answer its self-kNN queries in one kernel.
//
// Phase 1 -- builds.  Blocks take sets by ticket in the order `order` (largest first, so the
// longest builds start first) and build each whole set (cta_build_set).  A finished set is
// published: after a fence, its id goes to the next slot of `ready` with a release store.
// Phase 2 -- queries.  Each warp takes 32 queries of the set at the cursor of `ready` (one
// atomic per chunk on the set's chunk counter); when that set has no chunk left the cursor
// moves on.  The warp runs the fast walk on its 32 queries, reading the set's
// tree through L2 (the records were written by another block of this launch, so the
// read-only path cannot be used for them); tied queries go to the replay list as in every
// other fast walk.
// A block waits only for a set whose build another running block has claimed (every build is
// claimed before any block queries), so the waits end; they are bounded all the same (30 s of
// global time), after which the block sets STATUS_SPIN_LIMIT and stops.
// =========================================================================================
// Block shape: blocks as large as the SM's room for them allows, because a block builds a
// whole set and the largest sets' builds (latency-bound climbs and searches) set the launch's
// tail: for float coordinates 4 warps a block, 7 blocks (28 warps) with k <= 32 heaps; other
// types take more registers a thread (the exact 64-bit distances), 8 warps a block, 2 blocks.
template <class T> constexpr int persist_warps() { return std::is_same<T, float>::value ? 4 : 8; }
template <class T, int KC> constexpr int persist_blocks_per_sm() {
    return std::is_same<T, float>::value ? (KC > 32 ? 3 : 7) : (KC > 32 ? 1 : 2);
}
static constexpr int kPersistItems = 4; // keys per thread of a sort tile

template <class T> struct PersistDev {
    const long long *off, *node_off, *rec_off;
    int              S;
    const T         *x, *y, *z;
    const uint32_t  *id;
    const int8_t    *ghost;
    T               *mnx, *mxx, *mny, *mxy, *mnz, *mxz;
    int32_t         *left, *right, *parent;
    uint32_t        *tid_out;
    int8_t          *ghost_out;
    int32_t         *orig;
    NodeRec<T>      *recs;
    WideRec<T>      *wide;
    uint8_t         *height;
    int32_t         *counters, *leaves;
    unsigned long long *klo, *khi, *tlo, *thi;
    uint32_t        *perm, *tperm;
    T               *bbox;
    uint8_t         *set_height;
    const int32_t   *order;
    int32_t         *ready, *chunk_next;
    uint32_t        *ctl;
    int              query;
};

FT_D unsigned long long global_ns() {
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}
FT_D int ld_acquire_gpu(const int32_t *p) {
    int v;
    asm volatile("ld.acquire.gpu.global.b32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}
FT_D void st_release_gpu(int32_t *p, int v) {
    asm volatile("st.release.gpu.global.b32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}
FT_D int ld_relaxed_gpu_i(const int32_t *p) {
    int v;
    asm volatile("ld.relaxed.gpu.global.b32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}
FT_D uint32_t ld_relaxed_gpu(const uint32_t *p) {
    uint32_t v;
    asm volatile("ld.relaxed.gpu.global.b32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}

template <class T, int PER, int KC, int SFC, int KIND>
__global__ void __launch_bounds__(32 * persist_warps<T>(), persist_blocks_per_sm<T, KC>())
    batch_persistent_kernel(PersistDev<T> a, TreeDev<T> t_all, BatchDev bt, int k, int half_window,
                            int exclude_self, int ret_orig, unsigned long long *out_idx,
                            typename Coord<T>::dist_t *out_dist, int32_t *replay_ranks, int32_t *replay_rows,
                            uint32_t *replay_count, uint32_t *status, unsigned long long *visit_count) {
    constexpr int NW = persist_warps<T>(), PT = 32 * NW;
    extern __shared__ __align__(16) unsigned char smem[];
    __shared__ int s_item;
    const int      tid = threadIdx.x;

    // ---- 1. builds ----
    for (;;) {
        if (tid == 0) s_item = (int)atomicAdd(&a.ctl[0], 1u);
        __syncthreads();
        const int i = s_item;
        __syncthreads();
        if (i >= a.S) break; // block-uniform
        const int       s = a.order[i];
        const long long o = a.off[s];
        const int       n = (int)(a.off[s + 1] - o);
        if (n > 0) {
            const long long no = a.node_off[s], ro = a.rec_off[s];
            CtaTreeOut<T>   out;
            out.mnx      = a.mnx + no;
            out.mxx      = a.mxx + no;
            out.mny      = a.mny + no;
            out.mxy      = a.mxy + no;
            out.mnz      = a.mnz + no;
            out.mxz      = a.mxz + no;
            out.left     = a.left + ro;
            out.right    = a.right + ro;
            out.parent   = a.parent + no;
            out.id       = a.tid_out + no;
            out.ghost    = a.ghost_out + no;
            out.orig     = a.orig + no;
            out.recs     = a.recs + ro;
            out.wide     = a.wide + ro;
            out.height   = a.height + ro;
            out.counters = a.counters + ro;
            out.leaves   = a.leaves + ro;
            cta_build_set<T, SFC, KIND, PT, kPersistItems>(
                n, a.x + o, a.y + o, a.z + o, a.id ? a.id + o : nullptr, a.ghost ? a.ghost + o : nullptr, a.klo + o,
                a.khi ? a.khi + o : nullptr, a.perm + o, a.tlo + o, a.thi ? a.thi + o : nullptr, a.tperm + o, out,
                a.bbox + 6 * (size_t)s, a.set_height + s, smem);
        } else if (tid == 0) {
            // an empty set: the box the atomic min / max build leaves (no point folded in)
            using O = typename Ord<T>::type;
#pragma unroll
            for (int d = 0; d < 3; ++d) {
                a.bbox[6 * (size_t)s + 2 * d]     = Ord<T>::value((O)~(O)0);
                a.bbox[6 * (size_t)s + 2 * d + 1] = Ord<T>::value((O)0);
            }
            a.set_height[s] = 0;
        }
        if (tid == 0) { // publish the set: its tree is complete
            __threadfence();
            const uint32_t p = atomicAdd(&a.ctl[1], 1u);
            st_release_gpu(&a.ready[p], s);
        }
    }
    if (!a.query) return;

    // ---- 2. queries: each warp takes 32 queries at a time ----
    // A warp acquires a set's publication before it first reads the set's tree; the warp
    // barrier after the broadcast orders the other lanes' reads after it.
    const int lane     = tid & 31;
    int       acquired = -1; // the last set this warp acquired (lane 0)
    for (;;) {
        int s = -1, j = 0;
        if (lane == 0) {
            const unsigned long long t0 = global_ns();
            for (;;) {
                const uint32_t c = ld_relaxed_gpu(&a.ctl[2]);
                if (c >= (uint32_t)a.S) break;
                int r = ld_relaxed_gpu_i(&a.ready[c]);
                if (r >= 0 && r != acquired) {
                    r        = ld_acquire_gpu(&a.ready[c]);
                    acquired = r;
                }
                if (r < 0) { // a build another block holds is still running
                    if (global_ns() - t0 > 30000000000ull) {
                        atomicOr(status, STATUS_SPIN_LIMIT);
                        break;
                    }
                    __nanosleep(256);
                    continue;
                }
                const int n   = (int)(a.off[r + 1] - a.off[r]);
                const int nch = (n + 31) >> 5;
                if (nch > 0) {
                    const int jj = (int)atomicAdd(reinterpret_cast<uint32_t *>(&a.chunk_next[r]), 1u);
                    if (jj < nch) {
                        s = r;
                        j = jj;
                        break;
                    }
                }
                atomicCAS(&a.ctl[2], c, c + 1u); // this set has no chunk left
            }
        }
        s = __shfl_sync(0xffffffffu, s, 0);
        j = __shfl_sync(0xffffffffu, j, 0);
        __syncwarp();
        if (s < 0) break; // warp-uniform
        const int qbase = (int)a.off[s] + j * 32;
        const int end   = (int)a.off[s + 1];
        fast_warp<T, PER, KC, 4, NW, true>(qbase, QueryList{}, MissList{}, smem, t_all, bt, nullptr, nullptr, nullptr,
                                           nullptr, nullptr, end, k, half_window, exclude_self, ret_orig, nullptr,
                                           out_idx, out_dist, replay_ranks, replay_rows, replay_count, status,
                                           visit_count);
    }
}

template <class T, int PER, int KC, int SFC, int KIND>
static void launch_persistent_t(Context &ctx, const PersistLaunch &p, const PersistDev<T> &a, const TreeDev<T> &tv,
                                const BatchDev &bt, cudaStream_t st) {
    using D               = typename Coord<T>::dist_t;
    constexpr int NW      = persist_warps<T>(), PT = 32 * NW;
    const size_t  heaps   = p.query ? (size_t)std::max(p.k, 1) * PT * (sizeof(heap_dist_t<T>) + 4) : 0;
    const size_t  sorting = cta_sort_smem<Coord<T>::key_words, PT, kPersistItems>();
    const size_t  smem    = std::max(heaps, sorting);
    auto          fn      = batch_persistent_kernel<T, PER, KC, SFC, KIND>;
    FT_CUDA(cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    int per_sm = 0;
    FT_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fn, PT, smem));
    const int blocks = std::max(1, per_sm) * ctx.num_sms;
    const int half   = p.k; // the seeding window of the fast walk's default
    fn<<<blocks, PT, smem, st>>>(a, tv, bt, p.k, half, p.excl ? 1 : 0, ctx.opts.return_orig_indices ? 1 : 0,
                                 (unsigned long long *)p.idx, (D *)p.dist, p.rr, p.rw, p.counters, ctx.status,
                                 (unsigned long long *)(p.counters + 2));
    FT_CUDA(cudaGetLastError());
}

template <class T, int SFC, int KIND>
static void persistent_typed(Context &ctx, const PersistLaunch &p, cudaStream_t st) {
    PersistDev<T> a;
    a.off = p.off; a.node_off = p.node_off; a.rec_off = p.rec_off; a.S = p.S;
    a.x = (const T *)p.x; a.y = (const T *)p.y; a.z = (const T *)p.z; a.id = p.id; a.ghost = p.ghost;
    a.mnx = (T *)p.all.min_x; a.mxx = (T *)p.all.max_x; a.mny = (T *)p.all.min_y;
    a.mxy = (T *)p.all.max_y; a.mnz = (T *)p.all.min_z; a.mxz = (T *)p.all.max_z;
    a.left = p.all.left_child; a.right = p.all.right_child; a.parent = p.all.parent;
    a.tid_out = p.all.id; a.ghost_out = p.all.is_ghost; a.orig = p.all.orig_idx;
    a.recs = (NodeRec<T> *)p.scr->recs; a.wide = (WideRec<T> *)p.scr->wide; a.height = p.scr->height;
    a.counters = p.scr->counters; a.leaves = p.scr->leafcount;
    a.klo = (unsigned long long *)p.scr->key_lo; a.khi = (unsigned long long *)p.scr->key_hi;
    a.tlo = (unsigned long long *)p.scr->tmp_lo; a.thi = (unsigned long long *)p.scr->tmp_hi;
    a.perm = p.scr->perm; a.tperm = p.scr->tmp_perm;
    a.bbox = (T *)p.bbox; a.set_height = p.set_height;
    a.order = p.order; a.ready = p.ready; a.chunk_next = p.chunk_next; a.ctl = p.ctl;
    a.query = p.query ? 1 : 0;
    BatchDev bt;
    bt.off = p.off; bt.node_off = p.node_off; bt.rec_off = p.rec_off; bt.height = p.set_height; bt.S = p.S;
    const TreeDev<T> tv = tree_view<T>(p.all);
    if (!p.query) { // builds only: the smallest block shape's instance
        launch_persistent_t<T, 0, 32, SFC, KIND>(ctx, p, a, tv, bt, st);
        return;
    }
    met_dispatch<T>(metric_mode<T>(ctx.opts, p.all), [&](auto M) {
        constexpr int PER = decltype(M)::value;
        if (p.k <= 32) launch_persistent_t<T, PER, 32, SFC, KIND>(ctx, p, a, tv, bt, st);
        else launch_persistent_t<T, PER, 64, SFC, KIND>(ctx, p, a, tv, bt, st);
    });
}

void batch_persistent(Context &ctx, const PersistLaunch &p, cudaStream_t st) {
    if (p.query && (p.k < 1 || p.k > 64)) fail(FT_ERR_INVALID_ARGUMENT, "the persistent batched launch serves k <= 64");
    const bool morton = ctx.opts.sfc_type == MORTON;
    switch (ctx.opts.coord_type) {
    case F32:
        if (morton) persistent_typed<float, MORTON, 0>(ctx, p, st);
        else persistent_typed<float, PEANO_HILBERT, 1>(ctx, p, st);
        break;
    case F64:
        if (morton) persistent_typed<double, MORTON, 0>(ctx, p, st);
        else persistent_typed<double, PEANO_HILBERT, 1>(ctx, p, st);
        break;
    case U32: // integer positions always take Peano-Hilbert keys; the delta follows build_bvh's
        if (morton) persistent_typed<uint32_t, MORTON, 0>(ctx, p, st);
        else persistent_typed<uint32_t, PEANO_HILBERT, 1>(ctx, p, st);
        break;
    case U64:
        if (morton) persistent_typed<unsigned long long, MORTON, 0>(ctx, p, st);
        else persistent_typed<unsigned long long, PEANO_HILBERT, 2>(ctx, p, st);
        break;
    }
}

} // namespace ft
