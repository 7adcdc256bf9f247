// ft_common.cuh -- shared device definitions: coordinate traits, SFC cells and keys, the
// point-to-box distance, node records and small helpers.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <cfloat>
#include <type_traits>

#include "ft_internal.h"

#define FT_HD __host__ __device__ __forceinline__
#define FT_D __device__ __forceinline__

namespace ft {

enum CoordType : int32_t { F32 = 0, F64 = 1, U32 = 2, U64 = 3 };
enum SfcType : int32_t { MORTON = 0, PEANO_HILBERT = 1 };

// ---------------------------------------------------------------------------------------
// Coordinate traits.  The constants are those of the reference's configurations:
//   float/double with Peano-Hilbert: 32-bit position words, 21 bits per axis
//     (src/sfc.peano_hilbert.hpp:123-129, 168-172); Morton: 21 bits (src/sfc.morton.hpp:11)
//   uint32: 21 bits, SHIFT_BITS 11, _DIST_SHIFT 0   (src/sfc.peano_hilbert.hpp:169-172, 188)
//   uint64: 42 bits, SHIFT_BITS 22, _DIST_SHIFT 11  (src/sfc.peano_hilbert.hpp:173-176, 188)
// ---------------------------------------------------------------------------------------
template <class T> struct Coord {
    static constexpr bool is_float  = std::is_floating_point<T>::value;
    using dist_t                    = typename std::conditional<is_float, double, unsigned long long>::type;
    static constexpr int bits       = (!is_float && sizeof(T) == 8) ? 42 : 21;
    static constexpr int shift_bits = (sizeof(T) == 8) ? 22 : 11;
    static constexpr int dist_shift = (!is_float && bits > 31) ? bits - 31 : 0;
    static constexpr int key_words  = (!is_float && sizeof(T) == 8) ? 2 : 1; // 126- or 63-bit
};

// heap sentinel DIST_MAX (src/maxheap.hpp:45) and the "missing" output distance
// type_identity_max<dist_t>() (src/hlbvh.hpp:59-69)
template <class D> FT_HD D dist_heap_max();
template <> FT_HD double dist_heap_max<double>() { return DBL_MAX; }
template <> FT_HD unsigned long long dist_heap_max<unsigned long long>() { return ~0ull; }
template <class D> FT_HD D dist_missing();
template <> FT_HD double dist_missing<double>() { return -DBL_MAX; }
template <> FT_HD unsigned long long dist_missing<unsigned long long>() { return 0ull; }

// fmin / fmax with the C library's generic semantics: equality returns the first
// argument, a NaN argument yields the other one.  Written as compares so the sign of a
// zero result is defined (hardware min/max may pick either).
template <class T> FT_HD T c_fmin(T a, T b) { return (a <= b || b != b) ? a : b; }
template <class T> FT_HD T c_fmax(T a, T b) { return (a >= b || b != b) ? a : b; }

// sfc_min / sfc_max (src/hlbvh.hpp:580-594)
template <class T> FT_HD T box_min(T a, T b) {
    if constexpr (std::is_floating_point<T>::value) return c_fmin(a, b);
    else return (a < b) ? a : b;
}
template <class T> FT_HD T box_max(T a, T b) {
    if constexpr (std::is_floating_point<T>::value) return c_fmax(a, b);
    else return (a < b) ? b : a;
}

// IEEE round-to-nearest arithmetic with no contraction.
FT_D float add_rn(float a, float b) { return __fadd_rn(a, b); }
FT_D double add_rn(double a, double b) { return __dadd_rn(a, b); }
FT_D float sub_rn(float a, float b) { return __fsub_rn(a, b); }
FT_D double sub_rn(double a, double b) { return __dsub_rn(a, b); }
FT_D float mul_rn(float a, float b) { return __fmul_rn(a, b); }
FT_D double mul_rn(double a, double b) { return __dmul_rn(a, b); }

// ---------------------------------------------------------------------------------------
// Point-to-box squared distance (node_distance_sq, src/hlbvh.hpp:998-1055).
// ---------------------------------------------------------------------------------------
template <class T> struct Metric {
    using C      = Coord<T>;
    using dist_t = typename C::dist_t;

    // open integer axis: gap to the nearer face, low word shifted (1043-1047)
    static FT_D unsigned long long open_axis(T v, T lo, T hi) {
        if (v < lo) return (unsigned long long)(T)(lo - v) >> C::dist_shift;
        if (v > hi) return (unsigned long long)(T)(v - hi) >> C::dist_shift;
        return 0ull;
    }
    // shortest_periodic_distance in T's width (src/sfc.peano_hilbert.hpp:532-538)
    static FT_D long long spd(T a, T b) {
        if constexpr (sizeof(T) == 8) {
            return (long long)((unsigned long long)(T)(a - b) << C::shift_bits) >> C::shift_bits;
        } else {
            return (long long)((int32_t)((uint32_t)(a - b) << C::shift_bits) >> C::shift_bits);
        }
    }
    // periodic integer axis (1021-1033): inside [lo, hi] -> 0, else the smaller of the two
    // wrapped gaps, shifted.  Same value as the reference's formulation, fewer operations:
    //  * inside test: for lo <= hi, lo <= v <= hi  <=>  (v - lo) <= (hi - lo) as unsigned;
    //    for lo > hi the reference's test is false and so is the fallback compare used here;
    //  * a wrapped gap is x = sext_B(v - b); y = (v - b) << SHIFT_BITS holds x << SHIFT_BITS
    //    exactly, so |x| >> DIST_SHIFT == |y| >> (SHIFT_BITS + DIST_SHIFT) with |y| taken as
    //    an unsigned 64-bit value (covers |x| = 2^(B-1)).
    static FT_D unsigned long long periodic_axis(T v, T lo, T hi) {
        if constexpr (sizeof(T) == 8) {
            v &= (T)((T(1) << C::bits) - T(1));
            const unsigned long long dl = (unsigned long long)(v - lo), dh = (unsigned long long)(v - hi);
            const bool inside = (lo <= hi) ? (dl <= (unsigned long long)(hi - lo)) : false;
            const long long  yl = (long long)(dl << C::shift_bits), yh = (long long)(dh << C::shift_bits);
            const unsigned long long al = yl < 0 ? 0ull - (unsigned long long)yl : (unsigned long long)yl;
            const unsigned long long ah = yh < 0 ? 0ull - (unsigned long long)yh : (unsigned long long)yh;
            constexpr int s  = C::shift_bits + C::dist_shift; // 33 for 42-bit positions
            const uint32_t gl = (uint32_t)(al >> s), gh = (uint32_t)(ah >> s);
            return inside ? 0ull : (unsigned long long)min(gl, gh);
        } else {
            if (v >= lo && v <= hi) return 0ull;
            long long          dl = spd(v, lo), dh = spd(v, hi);
            unsigned long long al = (unsigned long long)(dl < 0 ? -dl : dl);
            unsigned long long ah = (unsigned long long)(dh < 0 ? -dh : dh);
            return ((al < ah) ? al : ah) >> C::dist_shift;
        }
    }
    // periodic 42-bit axis for trees whose coordinates are all below 2^42 (checked at build
    // time from the bounding box).  With v masked and lo <= hi < 2^42:
    //   a = (lo - v) mod 2^42 (up from v to lo),  b = (v - hi) mod 2^42 (down from v to hi);
    //   v strictly inside (lo, hi)  <=>  a + b > 2^42  (a + b = 2^43 - (hi - lo) there and
    //   2^42 - (hi - lo) outside), an endpoint gives a or b = 0, and outside the interval
    //   the reference's min(|sext(v - lo)|, |sext(v - hi)|) equals min(a, b).
    static FT_D unsigned long long periodic_axis_clean(T v, T lo, T hi) {
        static_assert(sizeof(T) == 8, "42-bit positions only");
        constexpr unsigned long long M = (1ull << C::bits) - 1ull;
        const unsigned long long     vv = (unsigned long long)v & M;
        const unsigned long long     a  = ((unsigned long long)lo - vv) & M;
        const unsigned long long     b  = (vv - (unsigned long long)hi) & M;
        const unsigned long long     g  = a < b ? a : b;
        return (a + b > M + 1ull) ? 0ull : (unsigned long long)(uint32_t)(g >> C::dist_shift);
    }
    static FT_D unsigned long long sq(unsigned long long g) {
        // gaps are < 2^32 for every configuration, so a 32x32->64 multiply is exact
        return (g >> 32) ? g * g : (unsigned long long)(uint32_t)g * (uint32_t)g;
    }

    // CLEAN: the tree's coordinates are all below 2^bits (42-bit periodic fast form).
    template <bool PERIODIC, bool CLEAN = false>
    static FT_D dist_t dist(T px, T py, T pz, T x0, T x1, T y0, T y1, T z0, T z1) {
        if constexpr (C::is_float) {
            T dx = c_fmax(sub_rn(x0, px), c_fmax(T(0), sub_rn(px, x1)));
            T dy = c_fmax(sub_rn(y0, py), c_fmax(T(0), sub_rn(py, y1)));
            T dz = c_fmax(sub_rn(z0, pz), c_fmax(T(0), sub_rn(pz, z1)));
            T s  = add_rn(add_rn(mul_rn(dx, dx), mul_rn(dy, dy)), mul_rn(dz, dz));
            return (double)s;
        } else {
            unsigned long long ax, ay, az;
            if constexpr (PERIODIC && CLEAN && sizeof(T) == 8) {
                ax = periodic_axis_clean(px, x0, x1);
                ay = periodic_axis_clean(py, y0, y1);
                az = periodic_axis_clean(pz, z0, z1);
            } else if constexpr (PERIODIC) {
                ax = periodic_axis(px, x0, x1);
                ay = periodic_axis(py, y0, y1);
                az = periodic_axis(pz, z0, z1);
            } else {
                ax = open_axis(px, x0, x1);
                ay = open_axis(py, y0, y1);
                az = open_axis(pz, z0, z1);
            }
            return sq(ax) + sq(ay) + sq(az);
        }
    }
};

// ---------------------------------------------------------------------------------------
// Internal node record used by the traversals: both child boxes and child indices in one
// 16-word line (64 B for 4-byte coordinates, 128 B for 8-byte ones), fetched with 16-byte
// vector loads.  Words 0-5: left box (minx,maxx,miny,maxy,minz,maxz); 6-11: right box;
// then the child indices (Karras encoding: index >= n-1 is a leaf slot), then one word per
// child with its leaf count and subtree height (rec_child_info), read in the same vector load.
// ---------------------------------------------------------------------------------------
template <class T> struct alignas(16 * sizeof(T)) NodeRec {
    T       lb[6];
    T       rb[6];
    int32_t l, r;
    int32_t pad[(16 * sizeof(T) - 12 * sizeof(T) - 8) / 4]; // [0] left, [1] right: rec_child_info
};

// A child's leaf count (25 bits, saturated) and subtree height (7 bits, saturated) in one
// word; saturated values are never used as exact (the range walk descends instead).
static constexpr uint32_t kInfoCountMax = (1u << 25) - 1u, kInfoHeightMax = 127u;
FT_HD uint32_t rec_child_info(uint32_t leaves, uint32_t height) {
    return (leaves < kInfoCountMax ? leaves : kInfoCountMax) | ((height < kInfoHeightMax ? height : kInfoHeightMax) << 25);
}
FT_HD uint32_t info_leaves(uint32_t w) { return w & kInfoCountMax; }
FT_HD uint32_t info_height(uint32_t w) { return w >> 25; }
static_assert(sizeof(NodeRec<float>) == 64, "record size");
static_assert(sizeof(NodeRec<double>) == 128, "record size");

// 4-wide record of an internal node for the fast walk: the node's grandchildren (a child
// that is a leaf stands for itself), up to four boxes and their node indices (-1: absent).
template <class T> struct alignas(16) WideRec {
    T       box[4][6];
    int32_t child[4];
};
static_assert(sizeof(WideRec<float>) == 112, "wide record size");
static_assert(sizeof(WideRec<double>) == 208, "wide record size");

// Record loads: through the read-only path by default.  COH: an ordinary (weak, L1-cached)
// global load instead, for kernels that read records other blocks wrote earlier in the same
// launch -- the read-only path is only valid for data that stays unchanged while the kernel
// runs, while an ordinary load that follows an acquire of the writer's release (and a warp
// barrier, for the other lanes) sees the written values.
template <bool COH> FT_D uint4 ld_rec16(const uint4 *p) {
    if constexpr (COH) {
        uint4 v;
        asm("ld.global.v4.u32 {%0, %1, %2, %3}, [%4];" : "=r"(v.x), "=r"(v.y), "=r"(v.z), "=r"(v.w) : "l"(p));
        return v;
    } else {
        return __ldg(p);
    }
}

template <class T, bool COH = false> FT_D void load_wide(const WideRec<T> *w, int node, T b[4][6], int c[4]) {
    constexpr int NW = (int)(sizeof(WideRec<T>) / 16);
    const uint4  *p  = reinterpret_cast<const uint4 *>(w + node);
    uint4         v[NW];
#pragma unroll
    for (int i = 0; i < NW; ++i) v[i] = ld_rec16<COH>(p + i);
    const T *f = reinterpret_cast<const T *>(v);
#pragma unroll
    for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int d = 0; d < 6; ++d) b[i][d] = f[6 * i + d];
    const int32_t *ci = reinterpret_cast<const int32_t *>(f + 24);
#pragma unroll
    for (int i = 0; i < 4; ++i) c[i] = ci[i];
}

// load_rec plus the two children's info words (rec_child_info).
template <class T, bool COH = false>
FT_D void load_rec_info(const NodeRec<T> *recs, int node, T lb[6], T rb[6], int &l, int &r, uint32_t &il,
                        uint32_t &ir) {
    const uint4 *p = reinterpret_cast<const uint4 *>(recs + node);
    if constexpr (sizeof(T) == 8) {
        uint4 w[7];
#pragma unroll
        for (int i = 0; i < 7; ++i) w[i] = ld_rec16<COH>(p + i);
        const T *v = reinterpret_cast<const T *>(w);
#pragma unroll
        for (int i = 0; i < 6; ++i) {
            lb[i] = v[i];
            rb[i] = v[6 + i];
        }
        l  = (int)w[6].x;
        r  = (int)w[6].y;
        il = w[6].z;
        ir = w[6].w;
    } else {
        uint4 w[4];
#pragma unroll
        for (int i = 0; i < 4; ++i) w[i] = ld_rec16<COH>(p + i);
        const T *v = reinterpret_cast<const T *>(w);
#pragma unroll
        for (int i = 0; i < 6; ++i) {
            lb[i] = v[i];
            rb[i] = v[6 + i];
        }
        l  = (int)w[3].x;
        r  = (int)w[3].y;
        il = w[3].z;
        ir = w[3].w;
    }
}

template <class T, bool COH = false>
FT_D void load_rec(const NodeRec<T> *recs, int node, T lb[6], T rb[6], int &l, int &r) {
    const uint4 *p = reinterpret_cast<const uint4 *>(recs + node);
    if constexpr (sizeof(T) == 8) {
        uint4 w[7];
#pragma unroll
        for (int i = 0; i < 7; ++i) w[i] = ld_rec16<COH>(p + i);
        const T *v = reinterpret_cast<const T *>(w);
#pragma unroll
        for (int i = 0; i < 6; ++i) {
            lb[i] = v[i];
            rb[i] = v[6 + i];
        }
        l = (int)w[6].x;
        r = (int)w[6].y;
    } else {
        uint4 w[4];
#pragma unroll
        for (int i = 0; i < 4; ++i) w[i] = ld_rec16<COH>(p + i);
        const T *v = reinterpret_cast<const T *>(w);
#pragma unroll
        for (int i = 0; i < 6; ++i) {
            lb[i] = v[i];
            rb[i] = v[6 + i];
        }
        l = (int)w[3].x;
        r = (int)w[3].y;
    }
}

// Distance mode of a query launch: 0 open box, 1 periodic, 2 periodic with every tree
// coordinate below 2^bits (the cheaper exact form of Metric::periodic_axis_clean).
// met_dispatch calls f(std::integral_constant<int, mode>) for the modes a type can have.
template <class T, class F> inline void met_dispatch(int met, F &&f) {
    if constexpr (Coord<T>::is_float) {
        f(std::integral_constant<int, 0>{});
    } else if constexpr (sizeof(T) == 4) {
        if (met) f(std::integral_constant<int, 1>{});
        else f(std::integral_constant<int, 0>{});
    } else {
        if (met == 2) f(std::integral_constant<int, 2>{});
        else if (met == 1) f(std::integral_constant<int, 1>{});
        else f(std::integral_constant<int, 0>{});
    }
}

// Device view of a built tree.
template <class T> struct TreeDev {
    const T *min_x, *max_x, *min_y, *max_y, *min_z, *max_z;
    const int32_t    *orig_idx;
    const NodeRec<T> *recs;
    const uint8_t    *height; // subtree height of each internal node
    const int32_t    *leaves; // leaf count of each internal node
    const WideRec<T> *wide;   // 4-wide record of each internal node
    int               n;      // leaves
};

// Device view of a built tree.
template <class T> inline TreeDev<T> tree_view(const ft_tree &tr) {
    TreeDev<T> v;
    v.min_x    = (const T *)tr.min_x;
    v.max_x    = (const T *)tr.max_x;
    v.min_y    = (const T *)tr.min_y;
    v.max_y    = (const T *)tr.max_y;
    v.min_z    = (const T *)tr.min_z;
    v.max_z    = (const T *)tr.max_z;
    v.orig_idx = tr.orig_idx;
    v.recs     = (const NodeRec<T> *)((TreeImpl *)tr.impl)->recs;
    v.height   = ((TreeImpl *)tr.impl)->height;
    v.leaves   = ((TreeImpl *)tr.impl)->leafcount;
    v.wide     = (const WideRec<T> *)((TreeImpl *)tr.impl)->wide;
    v.n        = (int)tr.num_leaves;
    return v;
}

// ---------------------------------------------------------------------------------------
// Batched trees (BatchDev, ft_internal.h): locating a leaf's set and viewing one set.
// ---------------------------------------------------------------------------------------
// Set holding global leaf q (the largest s with off[s] <= q; empty sets are skipped).
FT_D int find_set(const long long *off, int S, long long q) {
    int lo = 0, hi = S;
    while (hi - lo > 1) {
        int mid = (lo + hi) >> 1;
        if (off[mid] <= q) lo = mid;
        else hi = mid;
    }
    return lo;
}

template <class T> FT_D TreeDev<T> set_view(const TreeDev<T> &all, const BatchDev &b, int s) {
    const long long nb = b.node_off[s], rb = b.rec_off[s];
    TreeDev<T>      t;
    t.min_x    = all.min_x + nb;
    t.max_x    = all.max_x + nb;
    t.min_y    = all.min_y + nb;
    t.max_y    = all.max_y + nb;
    t.min_z    = all.min_z + nb;
    t.max_z    = all.max_z + nb;
    t.orig_idx = all.orig_idx + nb;
    t.recs     = all.recs + rb;
    t.height   = all.height + rb;
    t.leaves   = all.leaves + rb;
    t.wide     = all.wide + rb;
    t.n        = (int)(b.off[s + 1] - b.off[s]);
    return t;
}

// ---------------------------------------------------------------------------------------
// Bit tricks
// ---------------------------------------------------------------------------------------
FT_D int clz64(unsigned long long x) { return __clzll((long long)x); }

} // namespace ft
