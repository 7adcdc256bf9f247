// ft_oracle.cpp -- CPU restatement of FastTree's HLBVH build and neighbour queries.
//
// TEST INFRASTRUCTURE ONLY.  This file is the checker that the CUDA library is compared
// against; the library never calls it and has no CPU fallback.  Only tests/, the smoke
// check and bench.py's CPU-baseline leg load it.
//
// Every function restates the algorithm of the reference (sparxastronomy/fasttree) and
// cites the file:line it follows.  Semantics that the reference leaves to a library or
// to the platform are fixed here and marked "FIXED":
//   * equal SFC keys sort stably by original index (the reference uses oneDPL's device
//     sort, src/hlbvh.hpp:2215-2231, whose order among equal keys is unspecified);
//   * fmin/fmax follow the C library's generic definition (equality returns the first
//     argument, a NaN argument yields the other one);
//   * no floating-point contraction: build with -ffp-contract=off.
//   * Morton trees use KEY_TOTAL_BITS = 63 in the Karras tie-break (the Morton header
//     does not define it); any value >= 31 yields the same topology.
//   * for n == 1 the single leaf's parent is -1 (the reference leaves it unset).
//   * internal-node slots of id / is_ghost / orig_idx are zero (unset in the reference).
//
// Build: see oracle/Makefile (g++ -O2 -fopenmp -ffp-contract=off -shared -fPIC).

#include <algorithm>
#include <atomic>
#include <cfloat>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <limits>
#include <numeric>
#include <stdexcept>
#include <type_traits>
#include <vector>

#ifdef _OPENMP
#include <omp.h>
#endif

namespace ora {

// ----------------------------------------------------------------------------------------
// Options shared with the C ABI of the CUDA library (same numbering).
// ----------------------------------------------------------------------------------------
enum CoordType : int32_t { F32 = 0, F64 = 1, U32 = 2, U64 = 3 };
enum SfcType : int32_t { MORTON = 0, PEANO_HILBERT = 1 };

struct Options {
    int32_t coord_type;
    int32_t sfc_type;
    int32_t periodic;            // PERIODIC_BC (integer coordinates only)
    int32_t return_orig_indices; // RETURN_ORIG_INDICES
};

// Flat tree, same index layout as TreeSoA (src/hlbvh.hpp:596-673): internal nodes
// [0, n-2] with the root at 0, leaves [n-1, 2n-2].
struct Tree {
    void     *min_x, *max_x, *min_y, *max_y, *min_z, *max_z; // 2n-1 coords each
    int32_t  *left_child, *right_child;                      // n-1
    int32_t  *parent;                                        // 2n-1
    uint32_t *id;                                            // 2n-1
    int8_t   *is_ghost;                                      // 2n-1
    int32_t  *orig_idx;                                      // 2n-1
    int64_t   num_leaves;
};

// 126-bit (or 63-bit, hi == 0) SFC key.
struct Key {
    uint64_t hi, lo;
    bool operator<(const Key &o) const { return hi != o.hi ? hi < o.hi : lo < o.lo; }
    bool operator==(const Key &o) const { return hi == o.hi && lo == o.lo; }
    bool operator!=(const Key &o) const { return !(*this == o); }
};

static inline int clz64(uint64_t x) { return x ? __builtin_clzll(x) : 64; }

// FIXED fmin/fmax: C library generic semantics (see header note).
template <class T> static inline T c_fmin(T a, T b) { return (a <= b || b != b) ? a : b; }
template <class T> static inline T c_fmax(T a, T b) { return (a >= b || b != b) ? a : b; }

// sfc_min / sfc_max (src/hlbvh.hpp:580-594).
template <class T> static inline T sfc_min(T a, T b) {
    if constexpr (std::is_floating_point_v<T>) return c_fmin(a, b);
    else return (a < b) ? a : b;
}
template <class T> static inline T sfc_max(T a, T b) {
    if constexpr (std::is_floating_point_v<T>) return c_fmax(a, b);
    else return (a < b) ? b : a;
}

// ----------------------------------------------------------------------------------------
// Per-coordinate-type constants.
//   float/double + PH  : POSITIONS_IN_32BIT default, BITS_PER_DIMENSION = 21
//                        (src/sfc.peano_hilbert.hpp:123-129, 168-172)
//   float/double + Morton: BITS_PER_DIMENSION = 21 (src/sfc.morton.hpp:11-13)
//   uint32 : B = 21, SHIFT_BITS = 11, _DIST_SHIFT = 0   (sfc.peano_hilbert.hpp:169-172, 188)
//   uint64 : B = 42, SHIFT_BITS = 22, _DIST_SHIFT = 11  (sfc.peano_hilbert.hpp:173-176, 188)
// ----------------------------------------------------------------------------------------
template <class T> struct CT {
    static constexpr bool is_float = std::is_floating_point_v<T>;
    using dist_t                   = std::conditional_t<is_float, double, uint64_t>;
    static constexpr int bits      = (!is_float && sizeof(T) == 8) ? 42 : 21;
    static constexpr int shift_bits = (sizeof(T) == 8) ? 22 : 11;
    static constexpr int dist_shift = (!is_float && bits > 31) ? bits - 31 : 0;
    static constexpr int key_bits   = 3 * bits;
    // heap_dist_t sentinel DIST_MAX (src/maxheap.hpp:45, 488-492)
    static constexpr dist_t heap_max() { return std::numeric_limits<dist_t>::max(); }
    // type_identity_max<dist_t>() -- the "missing neighbour" distance written to the
    // output (src/hlbvh.hpp:59-69, 1178-1179)
    static constexpr dist_t missing() {
        if constexpr (is_float) return -std::numeric_limits<double>::max();
        else return 0;
    }
};

// ----------------------------------------------------------------------------------------
// Morton bit spreading (src/sfc.morton.hpp:26-41).
// ----------------------------------------------------------------------------------------
static inline uint64_t spread3(uint64_t x) {
    x &= 0x1FFFFFull;
    x = (x | (x << 32)) & 0x1F00000000FFFFull;
    x = (x | (x << 16)) & 0x1F0000FF0000FFull;
    x = (x | (x << 8)) & 0x100F00F00F00F00Full;
    x = (x | (x << 4)) & 0x10C30C30C30C30C3ull;
    x = (x | (x << 2)) & 0x1249249249249249ull;
    return x;
}

// ----------------------------------------------------------------------------------------
// AREPO Peano-Hilbert state tables (src/sfc.peano_hilbert.hpp:332-376).  These are data
// (a published table of the AREPO/GADGET curve), reproduced value for value because the
// curve is defined by them.
// ----------------------------------------------------------------------------------------
static const uint8_t kRot[48][8] = {
    {36, 28, 25, 27, 10, 10, 25, 27}, {29, 11, 24, 24, 37, 11, 26, 26}, {8, 8, 25, 27, 30, 38, 25, 27},
    {9, 39, 24, 24, 9, 31, 26, 26},   {40, 24, 44, 32, 40, 6, 44, 6},   {25, 7, 33, 7, 41, 41, 45, 45},
    {4, 42, 4, 46, 26, 42, 34, 46},   {43, 43, 47, 47, 5, 27, 5, 35},   {33, 35, 36, 28, 33, 35, 2, 2},
    {32, 32, 29, 3, 34, 34, 37, 3},   {33, 35, 0, 0, 33, 35, 30, 38},   {32, 32, 1, 39, 34, 34, 1, 31},
    {24, 42, 32, 46, 14, 42, 14, 46}, {43, 43, 47, 47, 25, 15, 33, 15}, {40, 12, 44, 12, 40, 26, 44, 34},
    {13, 27, 13, 35, 41, 41, 45, 45}, {28, 41, 28, 22, 38, 43, 38, 22}, {42, 40, 23, 23, 29, 39, 29, 39},
    {41, 36, 20, 36, 43, 30, 20, 30}, {37, 31, 37, 31, 42, 40, 21, 21}, {28, 18, 28, 45, 38, 18, 38, 47},
    {19, 19, 46, 44, 29, 39, 29, 39}, {16, 36, 45, 36, 16, 30, 47, 30}, {37, 31, 37, 31, 17, 17, 46, 44},
    {12, 4, 1, 3, 34, 34, 1, 3},      {5, 35, 0, 0, 13, 35, 2, 2},      {32, 32, 1, 3, 6, 14, 1, 3},
    {33, 15, 0, 0, 33, 7, 2, 2},      {16, 0, 20, 8, 16, 30, 20, 30},   {1, 31, 9, 31, 17, 17, 21, 21},
    {28, 18, 28, 22, 2, 18, 10, 22},  {19, 19, 23, 23, 29, 3, 29, 11},  {9, 11, 12, 4, 9, 11, 26, 26},
    {8, 8, 5, 27, 10, 10, 13, 27},    {9, 11, 24, 24, 9, 11, 6, 14},    {8, 8, 25, 15, 10, 10, 25, 7},
    {0, 18, 8, 22, 38, 18, 38, 22},   {19, 19, 23, 23, 1, 39, 9, 39},   {16, 36, 20, 36, 16, 2, 20, 10},
    {37, 3, 37, 11, 17, 17, 21, 21},  {4, 17, 4, 46, 14, 19, 14, 46},   {18, 16, 47, 47, 5, 15, 5, 15},
    {17, 12, 44, 12, 19, 6, 44, 6},   {13, 7, 13, 7, 18, 16, 45, 45},   {4, 42, 4, 21, 14, 42, 14, 23},
    {43, 43, 22, 20, 5, 15, 5, 15},   {40, 12, 21, 12, 40, 6, 23, 6},   {13, 7, 13, 7, 41, 41, 22, 20}};
static const uint8_t kSub[48][8] = {
    {0, 7, 1, 6, 3, 4, 2, 5}, {7, 4, 6, 5, 0, 3, 1, 2}, {4, 3, 5, 2, 7, 0, 6, 1}, {3, 0, 2, 1, 4, 7, 5, 6},
    {1, 0, 6, 7, 2, 3, 5, 4}, {0, 3, 7, 4, 1, 2, 6, 5}, {3, 2, 4, 5, 0, 1, 7, 6}, {2, 1, 5, 6, 3, 0, 4, 7},
    {6, 1, 7, 0, 5, 2, 4, 3}, {1, 2, 0, 3, 6, 5, 7, 4}, {2, 5, 3, 4, 1, 6, 0, 7}, {5, 6, 4, 7, 2, 1, 3, 0},
    {7, 6, 0, 1, 4, 5, 3, 2}, {6, 5, 1, 2, 7, 4, 0, 3}, {5, 4, 2, 3, 6, 7, 1, 0}, {4, 7, 3, 0, 5, 6, 2, 1},
    {6, 7, 5, 4, 1, 0, 2, 3}, {7, 0, 4, 3, 6, 1, 5, 2}, {0, 1, 3, 2, 7, 6, 4, 5}, {1, 6, 2, 5, 0, 7, 3, 4},
    {2, 3, 1, 0, 5, 4, 6, 7}, {3, 4, 0, 7, 2, 5, 1, 6}, {4, 5, 7, 6, 3, 2, 0, 1}, {5, 2, 6, 1, 4, 3, 7, 0},
    {7, 0, 6, 1, 4, 3, 5, 2}, {0, 3, 1, 2, 7, 4, 6, 5}, {3, 4, 2, 5, 0, 7, 1, 6}, {4, 7, 5, 6, 3, 0, 2, 1},
    {6, 7, 1, 0, 5, 4, 2, 3}, {7, 4, 0, 3, 6, 5, 1, 2}, {4, 5, 3, 2, 7, 6, 0, 1}, {5, 6, 2, 1, 4, 7, 3, 0},
    {1, 6, 0, 7, 2, 5, 3, 4}, {6, 5, 7, 4, 1, 2, 0, 3}, {5, 2, 4, 3, 6, 1, 7, 0}, {2, 1, 3, 0, 5, 6, 4, 7},
    {0, 1, 7, 6, 3, 2, 4, 5}, {1, 2, 6, 5, 0, 3, 7, 4}, {2, 3, 5, 4, 1, 0, 6, 7}, {3, 0, 4, 7, 2, 1, 5, 6},
    {1, 0, 2, 3, 6, 7, 5, 4}, {0, 7, 3, 4, 1, 6, 2, 5}, {7, 6, 4, 5, 0, 1, 3, 2}, {6, 1, 5, 2, 7, 0, 4, 3},
    {5, 4, 6, 7, 2, 3, 1, 0}, {4, 3, 7, 0, 5, 2, 6, 1}, {3, 2, 0, 1, 4, 5, 7, 6}, {2, 5, 1, 6, 3, 4, 0, 7}};

// Peano-Hilbert key of three B-bit integers (src/sfc.peano_hilbert.hpp:569-600 with the
// shift register of 396-405).  The reference's {hs,is,ls} word triple holds at most 126
// bits for the configurations built here, so a (hi, lo) pair is the same register.
static inline Key ph_encode(uint64_t px, uint64_t py, uint64_t pz, int bits) {
    Key     k{0, 0};
    uint8_t rot = 0;
    for (int b = bits - 1; b >= 0; --b) {
        unsigned pix = (unsigned)(((px >> b) & 1u) << 2 | ((py >> b) & 1u) << 1 | ((pz >> b) & 1u));
        k.hi         = (k.hi << 3) | (k.lo >> 61);
        k.lo         = (k.lo << 3) | kSub[rot][pix];
        rot          = kRot[rot][pix];
    }
    return k;
}

// Float -> 21-bit cell for Morton (encode_to_sfc1d, src/hlbvh.hpp:246-271): mantissa of
// (1 + nx) evaluated in T, top 21 bits.
template <class T> static inline uint64_t morton_cell(T nx) {
    T v = T(1) + nx;
    if constexpr (std::is_same_v<T, float>) {
        uint32_t bits;
        std::memcpy(&bits, &v, 4);
        return (bits & 0x007FFFFFu) >> (23 - 21);
    } else {
        uint64_t bits;
        std::memcpy(&bits, &v, 8);
        return (bits & 0x000FFFFFFFFFFFFFull) >> (52 - 21);
    }
}

// Float -> 21-bit cell for Peano-Hilbert (quantize_coord + convert_to_sfc1d_impl for a
// 32-bit position word, src/sfc.peano_hilbert.hpp:417-425, 472-476): evaluated in double,
// clamped below 2.
template <class T> static inline uint64_t ph_cell(T nx) {
    const double upper = 0x1.fffffffffffffp+0;
    double       b     = c_fmin(1.0 + static_cast<double>(nx), upper);
    uint64_t     bits;
    std::memcpy(&bits, &b, 8);
    return ((bits & 0x000FFFFFFFFFFFFFull) >> (52 - 21)) & 0x1FFFFFull;
}

// ----------------------------------------------------------------------------------------
// compute_bbox (src/hlbvh.hpp:462-572): per-axis minimum / maximum.  Empty input returns
// the identities (max, -max) for floats and (~0, 0) for integers.
// ----------------------------------------------------------------------------------------
template <class T> static void compute_bbox(const T *x, const T *y, const T *z, size_t n, T out[6]) {
    T lo, hi;
    if constexpr (std::is_floating_point_v<T>) {
        lo = std::numeric_limits<T>::max();
        hi = -std::numeric_limits<T>::max();
    } else {
        lo = std::numeric_limits<T>::max();
        hi = 0;
    }
    T r[6] = {lo, hi, lo, hi, lo, hi};
    const T *a[3] = {x, y, z};
    for (int d = 0; d < 3; ++d)
        for (size_t i = 0; i < n; ++i) {
            T v = a[d][i];
            if (v < r[2 * d]) r[2 * d] = v;          // sycl::minimum
            if (r[2 * d + 1] < v) r[2 * d + 1] = v;  // sycl::maximum
        }
    std::memcpy(out, r, sizeof(r));
}

// ----------------------------------------------------------------------------------------
// sfc_encode (src/hlbvh.hpp:357-423).  bbox = {min_x, max_x, min_y, max_y, min_z, max_z}.
// ----------------------------------------------------------------------------------------
template <class T>
static void sfc_encode(const Options &o, const T *x, const T *y, const T *z, size_t n,
                       const T bbox[6], Key *keys) {
    using C = CT<T>;
    if constexpr (!C::is_float) {
        // Integer coordinates: mask to B bits, bbox ignored (375-387).
        const uint64_t mask = (1ull << C::bits) - 1ull;
#pragma omp parallel for schedule(static)
        for (int64_t i = 0; i < (int64_t)n; ++i)
            keys[i] = ph_encode((uint64_t)x[i] & mask, (uint64_t)y[i] & mask, (uint64_t)z[i] & mask,
                                C::bits);
    } else {
        // Floating-point coordinates: normalise with host-computed reciprocals (389-396).
        T dx = bbox[1] - bbox[0], dy = bbox[3] - bbox[2], dz = bbox[5] - bbox[4];
        T inv[3] = {(dx == 0) ? T(0) : T(1) / dx, (dy == 0) ? T(0) : T(1) / dy,
                    (dz == 0) ? T(0) : T(1) / dz};
        T upper  = std::nextafter(T(1), T(0));
        const T *src[3] = {x, y, z};
#pragma omp parallel for schedule(static)
        for (int64_t i = 0; i < (int64_t)n; ++i) {
            uint64_t c[3];
            for (int d = 0; d < 3; ++d) {
                // sycl::clamp(v, lo, hi) == fmin(fmax(v, lo), hi)  (401-403)
                T nx = c_fmin(c_fmax((src[d][i] - bbox[2 * d]) * inv[d], T(0)), upper);
                c[d] = (o.sfc_type == MORTON) ? morton_cell(nx) : ph_cell(nx);
            }
            if (o.sfc_type == MORTON)
                keys[i] = Key{0, spread3(c[0]) | (spread3(c[1]) << 1) | (spread3(c[2]) << 2)};
            else
                keys[i] = ph_encode(c[0], c[1], c[2], 21);
        }
    }
}

// ----------------------------------------------------------------------------------------
// Karras delta (src/hlbvh.hpp:283-340, 852-859).
// ----------------------------------------------------------------------------------------
struct DeltaFn {
    const Key *k;
    int64_t    n;
    int        kind; // 0 = Morton (clz64), 1 = 63-bit PH (clz64 - 1), 2 = 126-bit PH
    int operator()(int i, int j) const {
        if (j < 0 || (int64_t)j >= n) return -1;
        const Key &a = k[i], &b = k[j];
        if (a != b) {
            if (kind == 0) return clz64(a.lo ^ b.lo);
            if (kind == 1) return clz64(a.lo ^ b.lo) - 1;
            if (a.hi != b.hi) return clz64(a.hi ^ b.hi) - 2;
            return 62 + clz64(a.lo ^ b.lo);
        }
        int ktb = (kind == 2) ? 126 : 63;
        return ktb + clz64((uint64_t)(int64_t)i ^ (uint64_t)(int64_t)j);
    }
};

static inline int sgn(int v) { return (v > 0) - (v < 0); }

static int delta_kind(const Options &o) {
    if (o.sfc_type == MORTON) return 0;
    return (o.coord_type == U64) ? 2 : 1;
}

// ----------------------------------------------------------------------------------------
// build_tree (src/hlbvh.hpp:773-982): Karras topology + optional leaf init + refit.
// ----------------------------------------------------------------------------------------
template <class T>
static void build_tree(const Options &o, Tree &t, const Key *keys, const T *sx, const T *sy,
                       const T *sz, const uint32_t *sid, const int8_t *sghost, const int32_t *sorig) {
    const int64_t n = t.num_leaves;
    if (n == 0) return;
    T *mnx = (T *)t.min_x, *mxx = (T *)t.max_x, *mny = (T *)t.min_y, *mxy = (T *)t.max_y,
      *mnz = (T *)t.min_z, *mxz = (T *)t.max_z;
    if (n == 1) { // single leaf (801-828)
        if (sx) {
            mnx[0] = mxx[0] = sx[0];
            mny[0] = mxy[0] = sy[0];
            mnz[0] = mxz[0] = sz[0];
        }
        if (sid) t.id[0] = sid[0];
        if (sghost) t.is_ghost[0] = sghost[0];
        if (sorig) t.orig_idx[0] = sorig[0];
        t.parent[0] = -1; // FIXED (unset in the reference)
        return;
    }
    for (int64_t i = 0; i < 2 * n - 1; ++i) t.parent[i] = -1; // 849
    DeltaFn delta{keys, n, delta_kind(o)};
    const int nn = (int)n;
#pragma omp parallel for schedule(static)
    for (int i = 0; i < nn - 1; ++i) { // 861-903
        int d         = sgn(delta(i, i + 1) - delta(i, i - 1));
        int delta_min = delta(i, i - d);
        int l_max     = 2;
        while (delta(i, i + l_max * d) > delta_min) l_max *= 2;
        int l = 0;
        for (int s = l_max / 2; s >= 1; s /= 2)
            if (delta(i, i + (l + s) * d) > delta_min) l += s;
        int j          = i + l * d;
        int delta_node = delta(i, j);
        int s          = 0;
        int step       = 1;
        while (step <= l) step *= 2;
        step /= 2;
        for (int tt = step; tt >= 1; tt /= 2)
            if (s + tt < l && delta(i, i + (s + tt) * d) > delta_node) s += tt;
        int split = i + s * d + std::min(d, 0);
        int left  = (std::min(i, j) == split) ? split + nn - 1 : split;
        int right = (std::max(i, j) == split + 1) ? split + 1 + nn - 1 : split + 1;
        t.left_child[i]  = left;
        t.right_child[i] = right;
        t.parent[left]   = i;
        t.parent[right]  = i;
    }
    if (sx && sy && sz) { // leaf init (906-923)
        for (int64_t i = 0; i < n; ++i) {
            int64_t leaf = i + n - 1;
            mnx[leaf] = mxx[leaf] = sx[i];
            mny[leaf] = mxy[leaf] = sy[i];
            mnz[leaf] = mxz[leaf] = sz[i];
            if (t.id && sid) t.id[leaf] = sid[i];
            if (t.is_ghost && sghost) t.is_ghost[leaf] = sghost[i];
            if (t.orig_idx && sorig) t.orig_idx[leaf] = sorig[i];
        }
    }
    // Bottom-up refit (925-969).  The second child to arrive at a parent merges the two
    // child boxes; the result does not depend on arrival order, so a sequential climb
    // reproduces it.
    std::vector<uint8_t> counter(n - 1, 0);
    for (int64_t leaf = 0; leaf < n; ++leaf) {
        int curr = (int)(leaf + n - 1);
        while (curr != 0) {
            int p = t.parent[curr];
            if (p < 0 || p >= nn - 1) break;
            if (counter[p]++ == 0) break;
            int l = t.left_child[p], r = t.right_child[p];
            mnx[p] = sfc_min(mnx[l], mnx[r]);
            mxx[p] = sfc_max(mxx[l], mxx[r]);
            mny[p] = sfc_min(mny[l], mny[r]);
            mxy[p] = sfc_max(mxy[l], mxy[r]);
            mnz[p] = sfc_min(mnz[l], mnz[r]);
            mxz[p] = sfc_max(mxz[l], mxz[r]);
            curr   = p;
        }
    }
}

// ----------------------------------------------------------------------------------------
// build_bvh (src/hlbvh.hpp:2165-2290).  keys_io (optional) are the caller's keys, which
// the reference sorts in place (2198-2200); sorted_keys_out (optional) receives the sorted
// keys either way.
// ----------------------------------------------------------------------------------------
template <class T>
static void build_bvh(const Options &o, const T *x, const T *y, const T *z, size_t n,
                      const uint32_t *id, const int8_t *ghost, const T *bbox_in, Key *keys_io,
                      Tree &t, Key *sorted_keys_out, T *bbox_out) {
    if (n == 0) return;
    if (n > (size_t)(std::numeric_limits<int>::max() / 2))
        throw std::runtime_error("Particle count n exceeds maximum supported tree size (INT_MAX / 2).");
    T bb[6];
    if (bbox_in) std::memcpy(bb, bbox_in, sizeof(bb));
    else compute_bbox(x, y, z, n, bb);
    if (bbox_out) std::memcpy(bbox_out, bb, sizeof(bb));
    std::vector<Key> own;
    Key             *keys = keys_io;
    if (!keys) {
        own.resize(n);
        keys = own.data();
        sfc_encode<T>(o, x, y, z, n, bb, keys);
    }
    // Sort (2202-2232), FIXED stable by original index.
    std::vector<int32_t> idx(n);
    std::iota(idx.begin(), idx.end(), 0);
    std::stable_sort(idx.begin(), idx.end(), [&](int32_t a, int32_t b) { return keys[a] < keys[b]; });
    std::vector<Key> sorted(n);
    for (size_t i = 0; i < n; ++i) sorted[i] = keys[idx[i]];
    if (keys_io) std::copy(sorted.begin(), sorted.end(), keys_io);
    if (sorted_keys_out) std::copy(sorted.begin(), sorted.end(), sorted_keys_out);
    // Gather into leaf slots (2235-2279).
    T *mnx = (T *)t.min_x, *mxx = (T *)t.max_x, *mny = (T *)t.min_y, *mxy = (T *)t.max_y,
      *mnz = (T *)t.min_z, *mxz = (T *)t.max_z;
    t.num_leaves = (int64_t)n;
    for (int64_t i = 0; i < (int64_t)(2 * n - 1); ++i) {
        if (t.id) t.id[i] = 0;
        if (t.is_ghost) t.is_ghost[i] = 0;
        if (t.orig_idx) t.orig_idx[i] = 0;
    }
    for (size_t i = 0; i < n; ++i) {
        size_t src  = (size_t)idx[i];
        size_t leaf = i + n - 1;
        mnx[leaf] = mxx[leaf] = x[src];
        mny[leaf] = mxy[leaf] = y[src];
        mnz[leaf] = mxz[leaf] = z[src];
        if (t.id) t.id[leaf] = id ? id[src] : (uint32_t)src;
        if (t.is_ghost) t.is_ghost[leaf] = ghost ? ghost[src] : 0;
        if (t.orig_idx) t.orig_idx[leaf] = (int32_t)src;
    }
    build_tree<T>(o, t, sorted.data(), nullptr, nullptr, nullptr, nullptr, nullptr, nullptr);
}

// ----------------------------------------------------------------------------------------
// node_distance_sq (src/hlbvh.hpp:998-1055).
// ----------------------------------------------------------------------------------------
template <class T> struct Dist {
    using C      = CT<T>;
    using dist_t = typename C::dist_t;
    bool periodic;

    static inline uint64_t open_axis(T v, T lo, T hi) {
        if (v < lo) return (uint64_t)(lo - v) >> C::dist_shift;
        if (v > hi) return (uint64_t)(v - hi) >> C::dist_shift;
        return 0;
    }
    // shortest_periodic_distance (src/sfc.peano_hilbert.hpp:532-538) in T's width.
    static inline int64_t spd(T a, T b) {
        if constexpr (sizeof(T) == 8) {
            return (int64_t)((uint64_t)(a - b) << C::shift_bits) >> C::shift_bits;
        } else {
            return (int64_t)((int32_t)((uint32_t)(a - b) << C::shift_bits) >> C::shift_bits);
        }
    }
    static inline uint64_t periodic_axis(T v, T lo, T hi) {
        if constexpr (sizeof(T) >= 8) v &= (T)((T(1) << C::bits) - T(1));
        if (v >= lo && v <= hi) return 0;
        int64_t  dl = spd(v, lo), dh = spd(v, hi);
        uint64_t al = (uint64_t)(dl < 0 ? -dl : dl), ah = (uint64_t)(dh < 0 ? -dh : dh);
        uint64_t g  = (al < ah) ? al : ah;
        return g >> C::dist_shift;
    }
    inline dist_t operator()(T px, T py, T pz, T x0, T x1, T y0, T y1, T z0, T z1) const {
        if constexpr (C::is_float) {
            T dx = c_fmax(x0 - px, c_fmax(T(0), px - x1));
            T dy = c_fmax(y0 - py, c_fmax(T(0), py - y1));
            T dz = c_fmax(z0 - pz, c_fmax(T(0), pz - z1));
            T s  = dx * dx;
            s    = s + dy * dy;
            s    = s + dz * dz;
            return static_cast<double>(s);
        } else {
            uint64_t ax, ay, az;
            if (periodic) {
                ax = periodic_axis(px, x0, x1);
                ay = periodic_axis(py, y0, y1);
                az = periodic_axis(pz, z0, z1);
            } else {
                ax = open_axis(px, x0, x1);
                ay = open_axis(py, y0, y1);
                az = open_axis(pz, z0, z1);
            }
            return ax * ax + ay * ay + az * az;
        }
    }
};

// ----------------------------------------------------------------------------------------
// RegisterMaxHeap / LocalMaxHeap (src/maxheap.hpp:33-144, 340-478): the same binary
// max-heap; LocalMaxHeap only moves the storage.  Capacity k.
// ----------------------------------------------------------------------------------------
template <class D> struct MaxHeap {
    std::vector<D>       dist;
    std::vector<int32_t> idx;
    int                  count = 0, k = 0;
    explicit MaxHeap(int k_) : dist(std::max(k_, 1), std::numeric_limits<D>::max()), idx(std::max(k_, 1), -1), k(k_) {}
    bool should_prune(D d) const { return count >= k && d >= dist[0]; }
    void swap_e(int a, int b) {
        std::swap(dist[a], dist[b]);
        std::swap(idx[a], idx[b]);
    }
    void sift_up(int i) {
        while (i > 0) {
            int p = (i - 1) >> 1;
            if (dist[i] <= dist[p]) break;
            swap_e(i, p);
            i = p;
        }
    }
    void sift_down(int i, int size) {
        for (;;) {
            int big = i, l = 2 * i + 1, r = 2 * i + 2;
            if (l < size && dist[l] > dist[big]) big = l;
            if (r < size && dist[r] > dist[big]) big = r;
            if (big == i) break;
            swap_e(i, big);
            i = big;
        }
    }
    void push(D d, int32_t i) {
        if (count < k) {
            dist[count] = d;
            idx[count]  = i;
            sift_up(count);
            ++count;
        } else if (d < dist[0]) {
            dist[0] = d;
            idx[0]  = i;
            sift_down(0, k);
        }
    }
    // extract_sorted / sort_in_place: in-place heapsort, ascending.
    void sort_in_place() {
        for (int hs = count; hs > 1;) {
            swap_e(0, hs - 1);
            --hs;
            sift_down(0, hs);
        }
    }
};

static constexpr int kMaxStack = 64; // MAX_STACK_DEPTH (src/hlbvh.hpp:984)

template <class T> struct TreeView {
    const T *mnx, *mxx, *mny, *mxy, *mnz, *mxz;
    const int32_t *l, *r, *orig;
    int64_t        n;
    explicit TreeView(const Tree &t)
        : mnx((const T *)t.min_x), mxx((const T *)t.max_x), mny((const T *)t.min_y),
          mxy((const T *)t.max_y), mnz((const T *)t.min_z), mxz((const T *)t.max_z),
          l(t.left_child), r(t.right_child), orig(t.orig_idx), n(t.num_leaves) {}
};

// One depth-first kNN traversal with the register/local max-heap, shared by knn_query's
// small-k kernel (src/hlbvh.hpp:1079-1182) and both grouped self-kNN kernels
// (1520-1647, 1690-1818).  The grouped kernels give each lane the same result as this
// independent traversal: a lane that follows a node only because another lane needs it
// pushes nothing from that subtree (its boxes are no nearer than the pruned ancestor),
// and the shared stack height bounds the same guard.  self_leaf < 0 disables
// exclude_self.
template <class T>
static void knn_dfs(const TreeView<T> &tv, const Dist<T> &dist, T px, T py, T pz, int k,
                    int64_t self_leaf, bool ret_orig, MaxHeap<typename CT<T>::dist_t> &heap,
                    bool self_mode, bool exclude_self) {
    const int64_t n = tv.n;
    int           stack[kMaxStack];
    int           sp = 0;
    stack[sp++]      = 0;
    while (sp > 0) {
        int  node = stack[--sp];
        auto d2   = dist(px, py, pz, tv.mnx[node], tv.mxx[node], tv.mny[node], tv.mxy[node],
                         tv.mnz[node], tv.mxz[node]);
        if (heap.should_prune(d2)) continue;
        if (node >= n - 1 && n > 1) {
            if (self_mode && exclude_self && node == self_leaf) continue;
            heap.push(d2, ret_orig ? tv.orig[node] : (int32_t)(node - (n - 1)));
        } else if (n == 1) {
            if (self_mode && exclude_self) continue;
            heap.push(d2, ret_orig ? tv.orig[0] : 0);
        } else {
            int  l   = tv.l[node], r = tv.r[node];
            auto ld2 = dist(px, py, pz, tv.mnx[l], tv.mxx[l], tv.mny[l], tv.mxy[l], tv.mnz[l], tv.mxz[l]);
            auto rd2 = dist(px, py, pz, tv.mnx[r], tv.mxx[r], tv.mny[r], tv.mxy[r], tv.mnz[r], tv.mxz[r]);
            if (sp < kMaxStack - 2) {
                if (ld2 <= rd2) {
                    stack[sp++] = r;
                    stack[sp++] = l;
                } else {
                    stack[sp++] = l;
                    stack[sp++] = r;
                }
            }
        }
    }
    (void)k;
}

template <class T>
static void write_heap(MaxHeap<typename CT<T>::dist_t> &heap, int k, uint64_t *out_idx,
                       typename CT<T>::dist_t *out_dist) {
    heap.sort_in_place();
    for (int i = 0; i < k; ++i) {
        if (i < heap.count && heap.idx[i] >= 0) {
            out_idx[i]  = (uint64_t)(int64_t)heap.idx[i];
            out_dist[i] = heap.dist[i];
        } else {
            out_idx[i]  = ~0ull;            // static_cast<size_t>(-1)
            out_dist[i] = CT<T>::missing(); // type_identity_max<dist_t>()
        }
    }
}

// self_knn_query / self_knn_query_subset (src/hlbvh.hpp:1929-1983).
template <class T>
static void self_knn(const Options &o, const Tree &t, const int32_t *leaf_ids, int64_t num, int k,
                     bool exclude_self, uint64_t *out_idx, void *out_dist_v) {
    using D = typename CT<T>::dist_t;
    D         *out_dist = (D *)out_dist_v;
    TreeView<T> tv(t);
    Dist<T>     dist{o.periodic != 0};
    const int64_t ni = tv.n - 1;
#pragma omp parallel for schedule(dynamic, 256)
    for (int64_t q = 0; q < num; ++q) {
        int64_t rank = leaf_ids ? leaf_ids[q] : q;
        T       px = tv.mnx[ni + rank], py = tv.mny[ni + rank], pz = tv.mnz[ni + rank];
        MaxHeap<D> heap(k);
        knn_dfs<T>(tv, dist, px, py, pz, k, rank + ni, o.return_orig_indices != 0, heap, true,
                   exclude_self);
        write_heap<T>(heap, k, out_idx + q * k, out_dist + q * k);
    }
}

// SortedMergeHeap and local_bitonic_sort (src/maxheap.hpp:193-324), single work-group
// emulated sequentially.  Each (k, j) stage of the bitonic network is a set of disjoint
// compare-exchanges, so a sequential sweep gives the work-group's result.
template <class D> struct MergeHeap {
    std::vector<D>       d;
    std::vector<int32_t> ix;
    int                  count = 0, cap, k;
    MergeHeap(int cap_, int k_) : d(cap_, std::numeric_limits<D>::max()), ix(cap_, -1), cap(cap_), k(k_) {}
    static void bitonic(D *dd, int32_t *ii, int n) {
        for (int kk = 2; kk <= n; kk <<= 1)
            for (int j = kk >> 1; j > 0; j >>= 1)
                for (int i = 0; i < n; ++i) {
                    int  l   = i ^ j;
                    bool asc = (i & kk) == 0;
                    if (l > i && l < n && ((dd[i] > dd[l]) == asc)) {
                        std::swap(dd[i], dd[l]);
                        std::swap(ii[i], ii[l]);
                    }
                }
    }
    bool should_prune(D v) const { return count >= k && v >= d[k - 1]; }
    // merge_batch with one real candidate (lane 0) and 31 empty lanes.
    void merge_one(D v, int32_t i) {
        D       sd[32];
        int32_t si[32];
        for (int a = 0; a < 32; ++a) {
            sd[a] = std::numeric_limits<D>::max();
            si[a] = -1;
        }
        sd[0] = v;
        si[0] = i;
        bitonic(sd, si, 32);
        for (int a = 0; a < 32; ++a) {
            int dst = count + a;
            if (dst < cap) {
                d[dst]  = sd[a];
                ix[dst] = si[a];
            }
        }
        int nc   = std::min(count + 32, cap);
        int pow2 = 1;
        while (pow2 < nc) pow2 <<= 1;
        for (int a = nc; a < pow2 && a < cap; ++a) {
            d[a]  = std::numeric_limits<D>::max();
            ix[a] = -1;
        }
        bitonic(d.data(), ix.data(), pow2);
        count = std::min(nc, cap);
        count = std::min(count, k);
    }
};

// knn_query (src/hlbvh.hpp:1405-1472): k <= 32 -> knn_query_small_k<32> (1057-1183);
// otherwise knn_query_large_k<max_k> (1185-1388) with HEAP_CAP = nextpow2(max_k).
template <class T>
static void knn(const Options &o, const Tree &t, const T *qx, const T *qy, const T *qz, int64_t nq,
                int k, int max_k, uint64_t *out_idx, void *out_dist_v) {
    using D = typename CT<T>::dist_t;
    D          *out_dist = (D *)out_dist_v;
    TreeView<T> tv(t);
    Dist<T>     dist{o.periodic != 0};
    const bool  ro = o.return_orig_indices != 0;
    if (k <= 32 || max_k <= 32) {
#pragma omp parallel for schedule(dynamic, 256)
        for (int64_t q = 0; q < nq; ++q) {
            MaxHeap<D> heap(k);
            knn_dfs<T>(tv, dist, qx[q], qy[q], qz[q], k, -1, ro, heap, false, false);
            write_heap<T>(heap, k, out_idx + q * k, out_dist + q * k);
        }
        return;
    }
    int cap = 1;
    while (cap < max_k) cap <<= 1;
    const int64_t n = tv.n;
#pragma omp parallel for schedule(dynamic, 64)
    for (int64_t q = 0; q < nq; ++q) {
        MergeHeap<D> h(cap, k);
        int          stack[kMaxStack];
        int          sp = 0;
        stack[sp++]     = 0;
        T px = qx[q], py = qy[q], pz = qz[q];
        while (sp > 0) {
            int  node = stack[--sp];
            auto d2   = dist(px, py, pz, tv.mnx[node], tv.mxx[node], tv.mny[node], tv.mxy[node],
                             tv.mnz[node], tv.mxz[node]);
            if (h.should_prune(d2)) continue;
            if (node >= n - 1 && n > 1) {
                h.merge_one(d2, ro ? tv.orig[node] : (int32_t)(node - (n - 1)));
            } else if (n == 1) {
                h.merge_one(d2, ro ? tv.orig[0] : 0);
            } else {
                int  l   = tv.l[node], r = tv.r[node];
                auto ld2 = dist(px, py, pz, tv.mnx[l], tv.mxx[l], tv.mny[l], tv.mxy[l], tv.mnz[l], tv.mxz[l]);
                auto rd2 = dist(px, py, pz, tv.mnx[r], tv.mxx[r], tv.mny[r], tv.mxy[r], tv.mnz[r], tv.mxz[r]);
                if (sp < kMaxStack - 2) {
                    if (ld2 <= rd2) {
                        stack[sp++] = r;
                        stack[sp++] = l;
                    } else {
                        stack[sp++] = l;
                        stack[sp++] = r;
                    }
                }
            }
        }
        for (int i = 0; i < k; ++i) {
            if (h.ix[i] >= 0) {
                out_idx[q * k + i]  = (uint64_t)(int64_t)h.ix[i];
                out_dist[q * k + i] = h.d[i];
            } else {
                out_idx[q * k + i]  = ~0ull;
                out_dist[q * k + i] = CT<T>::missing();
            }
        }
    }
}

// range_query (src/hlbvh.hpp:2006-2136).
template <class T>
static void range(const Options &o, const Tree &t, const T *qx, const T *qy, const T *qz,
                  const T *rmin, const T *rmax, int64_t nq, int32_t *results, int32_t *counts,
                  int max_per_q) {
    using D = typename CT<T>::dist_t;
    TreeView<T> tv(t);
    Dist<T>     dist{o.periodic != 0};
    const bool  ro = o.return_orig_indices != 0;
    const int64_t n = tv.n;
#pragma omp parallel for schedule(dynamic, 256)
    for (int64_t q = 0; q < nq; ++q) {
        D rm2, RM2;
        if constexpr (CT<T>::is_float) {
            double a = (double)rmin[q], b = (double)rmax[q];
            rm2 = a * a;
            RM2 = b * b;
        } else {
            uint64_t a = (uint64_t)rmin[q] >> CT<T>::dist_shift, b = (uint64_t)rmax[q] >> CT<T>::dist_shift;
            rm2 = a * a;
            RM2 = b * b;
        }
        int stack[kMaxStack];
        int sp = 0;
        stack[sp++] = 0;
        int     count = 0;
        int64_t off   = q * (int64_t)max_per_q;
        while (sp > 0) {
            int  node = stack[--sp];
            auto d2   = dist(qx[q], qy[q], qz[q], tv.mnx[node], tv.mxx[node], tv.mny[node],
                             tv.mxy[node], tv.mnz[node], tv.mxz[node]);
            if (!(d2 <= RM2)) continue;
            if (node >= n - 1 && n > 1) {
                if (d2 >= rm2) {
                    if (count < max_per_q) results[off + count] = ro ? tv.orig[node] : (int32_t)(node - (n - 1));
                    ++count;
                }
            } else if (n == 1) {
                if (d2 >= rm2) {
                    if (count < max_per_q) results[off + count] = ro ? tv.orig[0] : 0;
                    ++count;
                }
            } else if (sp < kMaxStack - 2) {
                stack[sp++] = tv.r[node];
                stack[sp++] = tv.l[node];
            }
        }
        counts[q] = count;
    }
}

} // namespace ora

// ========================================================================================
// C entry points (ctypes).  Keys cross the boundary as two uint64 arrays (hi, lo).
// Return 0 on success, 1 on invalid argument, 2 on runtime error.
// ========================================================================================
using namespace ora;

#define ORA_DISPATCH(o, FN, ...)                                            \
    switch ((o).coord_type) {                                               \
    case F32: FN<float>(__VA_ARGS__); break;                                \
    case F64: FN<double>(__VA_ARGS__); break;                               \
    case U32: FN<uint32_t>(__VA_ARGS__); break;                             \
    case U64: FN<uint64_t>(__VA_ARGS__); break;                             \
    default: return 1;                                                      \
    }

static bool valid(const Options &o) {
    if (o.coord_type < 0 || o.coord_type > 3) return false;
    if (o.sfc_type != MORTON && o.sfc_type != PEANO_HILBERT) return false;
    if (o.sfc_type == MORTON && (o.coord_type == U32 || o.coord_type == U64)) return false;
    return true;
}

static void split_keys(const Key *k, size_t n, uint64_t *hi, uint64_t *lo) {
    for (size_t i = 0; i < n; ++i) {
        if (hi) hi[i] = k[i].hi;
        if (lo) lo[i] = k[i].lo;
    }
}

extern "C" {

int ora_set_threads(int n) {
#ifdef _OPENMP
    if (n > 0) omp_set_num_threads(n);
    return omp_get_max_threads();
#else
    (void)n;
    return 1;
#endif
}

int ora_compute_bbox(const Options *o, const void *x, const void *y, const void *z, int64_t n, void *out6) {
    if (!valid(*o)) return 1;
    switch (o->coord_type) {
    case F32: compute_bbox<float>((const float *)x, (const float *)y, (const float *)z, n, (float *)out6); break;
    case F64: compute_bbox<double>((const double *)x, (const double *)y, (const double *)z, n, (double *)out6); break;
    case U32: compute_bbox<uint32_t>((const uint32_t *)x, (const uint32_t *)y, (const uint32_t *)z, n, (uint32_t *)out6); break;
    case U64: compute_bbox<uint64_t>((const uint64_t *)x, (const uint64_t *)y, (const uint64_t *)z, n, (uint64_t *)out6); break;
    }
    return 0;
}

int ora_sfc_encode(const Options *o, const void *x, const void *y, const void *z, int64_t n,
                   const void *bbox6, uint64_t *hi, uint64_t *lo) {
    if (!valid(*o)) return 1;
    std::vector<Key> k(n);
    switch (o->coord_type) {
    case F32: sfc_encode<float>(*o, (const float *)x, (const float *)y, (const float *)z, n, (const float *)bbox6, k.data()); break;
    case F64: sfc_encode<double>(*o, (const double *)x, (const double *)y, (const double *)z, n, (const double *)bbox6, k.data()); break;
    case U32: sfc_encode<uint32_t>(*o, (const uint32_t *)x, (const uint32_t *)y, (const uint32_t *)z, n, nullptr, k.data()); break;
    case U64: sfc_encode<uint64_t>(*o, (const uint64_t *)x, (const uint64_t *)y, (const uint64_t *)z, n, nullptr, k.data()); break;
    }
    split_keys(k.data(), n, hi, lo);
    return 0;
}

// keys_hi/keys_lo: optional caller keys (sorted in place, as the reference does).
// sorted_hi/sorted_lo: optional sorted-key outputs.  bbox_out: optional 6 coords.
int ora_build_bvh(const Options *o, const void *x, const void *y, const void *z, int64_t n,
                  const uint32_t *id, const int8_t *ghost, const void *bbox_in, uint64_t *keys_hi,
                  uint64_t *keys_lo, Tree *t, uint64_t *sorted_hi, uint64_t *sorted_lo, void *bbox_out) {
    if (!valid(*o)) return 1;
    try {
        std::vector<Key> caller, sorted(n > 0 ? n : 1);
        Key             *kio = nullptr;
        if (keys_lo) {
            caller.resize(n);
            for (int64_t i = 0; i < n; ++i) caller[i] = Key{keys_hi ? keys_hi[i] : 0, keys_lo[i]};
            kio = caller.data();
        }
        switch (o->coord_type) {
        case F32: build_bvh<float>(*o, (const float *)x, (const float *)y, (const float *)z, n, id, ghost, (const float *)bbox_in, kio, *t, sorted.data(), (float *)bbox_out); break;
        case F64: build_bvh<double>(*o, (const double *)x, (const double *)y, (const double *)z, n, id, ghost, (const double *)bbox_in, kio, *t, sorted.data(), (double *)bbox_out); break;
        case U32: build_bvh<uint32_t>(*o, (const uint32_t *)x, (const uint32_t *)y, (const uint32_t *)z, n, id, ghost, (const uint32_t *)bbox_in, kio, *t, sorted.data(), (uint32_t *)bbox_out); break;
        case U64: build_bvh<uint64_t>(*o, (const uint64_t *)x, (const uint64_t *)y, (const uint64_t *)z, n, id, ghost, (const uint64_t *)bbox_in, kio, *t, sorted.data(), (uint64_t *)bbox_out); break;
        }
        if (kio) split_keys(kio, n, keys_hi, keys_lo);
        if (n > 0) split_keys(sorted.data(), n, sorted_hi, sorted_lo);
    } catch (const std::runtime_error &) {
        return 2;
    }
    return 0;
}

// build_tree with caller-sorted keys and optional sorted leaf attributes.
int ora_build_tree(const Options *o, Tree *t, const uint64_t *keys_hi, const uint64_t *keys_lo,
                   const void *sx, const void *sy, const void *sz, const uint32_t *sid,
                   const int8_t *sghost, const int32_t *sorig) {
    if (!valid(*o)) return 1;
    int64_t          n = t->num_leaves;
    std::vector<Key> k(n > 0 ? n : 1);
    for (int64_t i = 0; i < n; ++i) k[i] = Key{keys_hi ? keys_hi[i] : 0, keys_lo[i]};
    switch (o->coord_type) {
    case F32: build_tree<float>(*o, *t, k.data(), (const float *)sx, (const float *)sy, (const float *)sz, sid, sghost, sorig); break;
    case F64: build_tree<double>(*o, *t, k.data(), (const double *)sx, (const double *)sy, (const double *)sz, sid, sghost, sorig); break;
    case U32: build_tree<uint32_t>(*o, *t, k.data(), (const uint32_t *)sx, (const uint32_t *)sy, (const uint32_t *)sz, sid, sghost, sorig); break;
    case U64: build_tree<uint64_t>(*o, *t, k.data(), (const uint64_t *)sx, (const uint64_t *)sy, (const uint64_t *)sz, sid, sghost, sorig); break;
    }
    return 0;
}

int ora_self_knn(const Options *o, const Tree *t, const int32_t *leaf_ids, int64_t num, int k,
                 int exclude_self, uint64_t *out_idx, void *out_dist) {
    if (!valid(*o)) return 1;
    if (t->num_leaves == 0 || num == 0 || k <= 0) return 0;
    ORA_DISPATCH(*o, self_knn, *o, *t, leaf_ids, num, k, exclude_self != 0, out_idx, out_dist);
    return 0;
}

int ora_knn(const Options *o, const Tree *t, const void *qx, const void *qy, const void *qz, int64_t nq,
            int k, int max_k, uint64_t *out_idx, void *out_dist) {
    if (!valid(*o)) return 1;
    if (t->num_leaves == 0 || nq == 0 || k <= 0) return 0;
    if (max_k > 32 && k > max_k) return 1; // std::invalid_argument (1443-1447)
    switch (o->coord_type) {
    case F32: knn<float>(*o, *t, (const float *)qx, (const float *)qy, (const float *)qz, nq, k, max_k, out_idx, out_dist); break;
    case F64: knn<double>(*o, *t, (const double *)qx, (const double *)qy, (const double *)qz, nq, k, max_k, out_idx, out_dist); break;
    case U32: knn<uint32_t>(*o, *t, (const uint32_t *)qx, (const uint32_t *)qy, (const uint32_t *)qz, nq, k, max_k, out_idx, out_dist); break;
    case U64: knn<uint64_t>(*o, *t, (const uint64_t *)qx, (const uint64_t *)qy, (const uint64_t *)qz, nq, k, max_k, out_idx, out_dist); break;
    }
    return 0;
}

int ora_range(const Options *o, const Tree *t, const void *qx, const void *qy, const void *qz,
              const void *rmin, const void *rmax, int64_t nq, int32_t *results, int32_t *counts,
              int max_per_q) {
    if (!valid(*o)) return 1;
    if (t->num_leaves == 0 || nq == 0) return 0;
    switch (o->coord_type) {
    case F32: range<float>(*o, *t, (const float *)qx, (const float *)qy, (const float *)qz, (const float *)rmin, (const float *)rmax, nq, results, counts, max_per_q); break;
    case F64: range<double>(*o, *t, (const double *)qx, (const double *)qy, (const double *)qz, (const double *)rmin, (const double *)rmax, nq, results, counts, max_per_q); break;
    case U32: range<uint32_t>(*o, *t, (const uint32_t *)qx, (const uint32_t *)qy, (const uint32_t *)qz, (const uint32_t *)rmin, (const uint32_t *)rmax, nq, results, counts, max_per_q); break;
    case U64: range<uint64_t>(*o, *t, (const uint64_t *)qx, (const uint64_t *)qy, (const uint64_t *)qz, (const uint64_t *)rmin, (const uint64_t *)rmax, nq, results, counts, max_per_q); break;
    }
    return 0;
}

// Point-to-box distance as the queries compute it (for brute-force checks in tests).
int ora_point_dist(const Options *o, const void *p3, const void *box6, void *out) {
    if (!valid(*o)) return 1;
    switch (o->coord_type) {
    case F32: { const float *p = (const float *)p3, *b = (const float *)box6; *(double *)out = Dist<float>{o->periodic != 0}(p[0], p[1], p[2], b[0], b[1], b[2], b[3], b[4], b[5]); break; }
    case F64: { const double *p = (const double *)p3, *b = (const double *)box6; *(double *)out = Dist<double>{o->periodic != 0}(p[0], p[1], p[2], b[0], b[1], b[2], b[3], b[4], b[5]); break; }
    case U32: { const uint32_t *p = (const uint32_t *)p3, *b = (const uint32_t *)box6; *(uint64_t *)out = Dist<uint32_t>{o->periodic != 0}(p[0], p[1], p[2], b[0], b[1], b[2], b[3], b[4], b[5]); break; }
    case U64: { const uint64_t *p = (const uint64_t *)p3, *b = (const uint64_t *)box6; *(uint64_t *)out = Dist<uint64_t>{o->periodic != 0}(p[0], p[1], p[2], b[0], b[1], b[2], b[3], b[4], b[5]); break; }
    }
    return 0;
}

// Isolated heap runs mirroring the reference's heap unit tests
// (test/test_self_knn.cpp:374-562): push a sequence through the max-heap (with its
// prune check) or through SortedMergeHeap rounds; outputs are the final arrays.
int ora_maxheap_run(int k, const double *d, const int32_t *ix, int m, int use_prune, double *out_d,
                    int32_t *out_i, int *out_count) {
    MaxHeap<double> h(k);
    for (int a = 0; a < m; ++a) {
        if (use_prune && h.should_prune(d[a])) continue;
        h.push(d[a], ix[a]);
    }
    h.sort_in_place();
    for (int a = 0; a < k; ++a) {
        out_d[a] = h.dist[a];
        out_i[a] = h.idx[a];
    }
    *out_count = h.count;
    return 0;
}

// rounds x 32 lanes of (d, i); each round is one merge_batch of all 32 lanes.
int ora_mergeheap_run(int k, int cap, const double *d, const int32_t *ix, int rounds, double *out_d,
                      int32_t *out_i) {
    MergeHeap<double> h(cap, k);
    for (int r = 0; r < rounds; ++r) {
        double  sd[32];
        int32_t si[32];
        for (int a = 0; a < 32; ++a) {
            sd[a] = d[r * 32 + a];
            si[a] = ix[r * 32 + a];
        }
        MergeHeap<double>::bitonic(sd, si, 32);
        for (int a = 0; a < 32; ++a) {
            int dst = h.count + a;
            if (dst < cap) {
                h.d[dst]  = sd[a];
                h.ix[dst] = si[a];
            }
        }
        int nc   = std::min(h.count + 32, cap);
        int pow2 = 1;
        while (pow2 < nc) pow2 <<= 1;
        for (int a = nc; a < pow2 && a < cap; ++a) {
            h.d[a]  = std::numeric_limits<double>::max();
            h.ix[a] = -1;
        }
        MergeHeap<double>::bitonic(h.d.data(), h.ix.data(), pow2);
        h.count = std::min(std::min(nc, cap), k);
    }
    for (int a = 0; a < cap; ++a) {
        out_d[a] = h.d[a];
        out_i[a] = h.ix[a];
    }
    return 0;
}

} // extern "C"
