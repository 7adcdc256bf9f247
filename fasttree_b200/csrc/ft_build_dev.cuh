// ft_build_dev.cuh -- device helpers shared by the single-tree build (ft_build.cu) and the
// batched build (ft_batch.cu): SFC cells and keys, the Karras delta.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "ft_common.cuh"

namespace ft {

// =========================================================================================
// Peano-Hilbert state tables (AREPO's rottable3 / subpix3, reproduced in
// src/sfc.peano_hilbert.hpp:332-376).  The curve is defined by these values.
// =========================================================================================
static __constant__ uint8_t c_rot[48 * 8] = {
    36, 28, 25, 27, 10, 10, 25, 27, 29, 11, 24, 24, 37, 11, 26, 26, 8,  8,  25, 27, 30, 38, 25, 27,
    9,  39, 24, 24, 9,  31, 26, 26, 40, 24, 44, 32, 40, 6,  44, 6,  25, 7,  33, 7,  41, 41, 45, 45,
    4,  42, 4,  46, 26, 42, 34, 46, 43, 43, 47, 47, 5,  27, 5,  35, 33, 35, 36, 28, 33, 35, 2,  2,
    32, 32, 29, 3,  34, 34, 37, 3,  33, 35, 0,  0,  33, 35, 30, 38, 32, 32, 1,  39, 34, 34, 1,  31,
    24, 42, 32, 46, 14, 42, 14, 46, 43, 43, 47, 47, 25, 15, 33, 15, 40, 12, 44, 12, 40, 26, 44, 34,
    13, 27, 13, 35, 41, 41, 45, 45, 28, 41, 28, 22, 38, 43, 38, 22, 42, 40, 23, 23, 29, 39, 29, 39,
    41, 36, 20, 36, 43, 30, 20, 30, 37, 31, 37, 31, 42, 40, 21, 21, 28, 18, 28, 45, 38, 18, 38, 47,
    19, 19, 46, 44, 29, 39, 29, 39, 16, 36, 45, 36, 16, 30, 47, 30, 37, 31, 37, 31, 17, 17, 46, 44,
    12, 4,  1,  3,  34, 34, 1,  3,  5,  35, 0,  0,  13, 35, 2,  2,  32, 32, 1,  3,  6,  14, 1,  3,
    33, 15, 0,  0,  33, 7,  2,  2,  16, 0,  20, 8,  16, 30, 20, 30, 1,  31, 9,  31, 17, 17, 21, 21,
    28, 18, 28, 22, 2,  18, 10, 22, 19, 19, 23, 23, 29, 3,  29, 11, 9,  11, 12, 4,  9,  11, 26, 26,
    8,  8,  5,  27, 10, 10, 13, 27, 9,  11, 24, 24, 9,  11, 6,  14, 8,  8,  25, 15, 10, 10, 25, 7,
    0,  18, 8,  22, 38, 18, 38, 22, 19, 19, 23, 23, 1,  39, 9,  39, 16, 36, 20, 36, 16, 2,  20, 10,
    37, 3,  37, 11, 17, 17, 21, 21, 4,  17, 4,  46, 14, 19, 14, 46, 18, 16, 47, 47, 5,  15, 5,  15,
    17, 12, 44, 12, 19, 6,  44, 6,  13, 7,  13, 7,  18, 16, 45, 45, 4,  42, 4,  21, 14, 42, 14, 23,
    43, 43, 22, 20, 5,  15, 5,  15, 40, 12, 21, 12, 40, 6,  23, 6,  13, 7,  13, 7,  41, 41, 22, 20};
static __constant__ uint8_t c_sub[48 * 8] = {
    0, 7, 1, 6, 3, 4, 2, 5, 7, 4, 6, 5, 0, 3, 1, 2, 4, 3, 5, 2, 7, 0, 6, 1, 3, 0, 2, 1, 4, 7, 5, 6,
    1, 0, 6, 7, 2, 3, 5, 4, 0, 3, 7, 4, 1, 2, 6, 5, 3, 2, 4, 5, 0, 1, 7, 6, 2, 1, 5, 6, 3, 0, 4, 7,
    6, 1, 7, 0, 5, 2, 4, 3, 1, 2, 0, 3, 6, 5, 7, 4, 2, 5, 3, 4, 1, 6, 0, 7, 5, 6, 4, 7, 2, 1, 3, 0,
    7, 6, 0, 1, 4, 5, 3, 2, 6, 5, 1, 2, 7, 4, 0, 3, 5, 4, 2, 3, 6, 7, 1, 0, 4, 7, 3, 0, 5, 6, 2, 1,
    6, 7, 5, 4, 1, 0, 2, 3, 7, 0, 4, 3, 6, 1, 5, 2, 0, 1, 3, 2, 7, 6, 4, 5, 1, 6, 2, 5, 0, 7, 3, 4,
    2, 3, 1, 0, 5, 4, 6, 7, 3, 4, 0, 7, 2, 5, 1, 6, 4, 5, 7, 6, 3, 2, 0, 1, 5, 2, 6, 1, 4, 3, 7, 0,
    7, 0, 6, 1, 4, 3, 5, 2, 0, 3, 1, 2, 7, 4, 6, 5, 3, 4, 2, 5, 0, 7, 1, 6, 4, 7, 5, 6, 3, 0, 2, 1,
    6, 7, 1, 0, 5, 4, 2, 3, 7, 4, 0, 3, 6, 5, 1, 2, 4, 5, 3, 2, 7, 6, 0, 1, 5, 6, 2, 1, 4, 7, 3, 0,
    1, 6, 0, 7, 2, 5, 3, 4, 6, 5, 7, 4, 1, 2, 0, 3, 5, 2, 4, 3, 6, 1, 7, 0, 2, 1, 3, 0, 5, 6, 4, 7,
    0, 1, 7, 6, 3, 2, 4, 5, 1, 2, 6, 5, 0, 3, 7, 4, 2, 3, 5, 4, 1, 0, 6, 7, 3, 0, 4, 7, 2, 1, 5, 6,
    1, 0, 2, 3, 6, 7, 5, 4, 0, 7, 3, 4, 1, 6, 2, 5, 7, 6, 4, 5, 0, 1, 3, 2, 6, 1, 5, 2, 7, 0, 4, 3,
    5, 4, 6, 7, 2, 3, 1, 0, 4, 3, 7, 0, 5, 2, 6, 1, 3, 2, 0, 1, 4, 5, 7, 6, 2, 5, 1, 6, 3, 4, 0, 7};

FT_D unsigned long long spread3(unsigned long long x) { // src/sfc.morton.hpp:33-41
    x &= 0x1FFFFFull;
    x = (x | (x << 32)) & 0x1F00000000FFFFull;
    x = (x | (x << 16)) & 0x1F0000FF0000FFull;
    x = (x | (x << 8)) & 0x100F00F00F00F00Full;
    x = (x | (x << 4)) & 0x10C30C30C30C30C3ull;
    x = (x | (x << 2)) & 0x1249249249249249ull;
    return x;
}

// Peano-Hilbert key: B rounds of octant index -> table lookup (src/sfc.peano_hilbert.hpp:569-600);
// the key register is shifted 3 bits per round (396-405).
template <int B>
FT_D void ph_key(unsigned long long px, unsigned long long py, unsigned long long pz, const uint8_t *rot_t,
                 const uint8_t *sub_t, unsigned long long &hi, unsigned long long &lo) {
    unsigned long long h = 0, l = 0;
    unsigned           rot = 0;
#pragma unroll 6
    for (int b = B - 1; b >= 0; --b) {
        unsigned pix = (unsigned)((((px >> b) & 1ull) << 2) | (((py >> b) & 1ull) << 1) | ((pz >> b) & 1ull));
        unsigned e   = rot * 8u + pix;
        h            = (h << 3) | (l >> 61);
        l            = (l << 3) | sub_t[e];
        rot          = rot_t[e];
    }
    hi = h;
    lo = l;
}

template <class T> FT_D unsigned long long morton_cell(T nx) { // encode_to_sfc1d (src/hlbvh.hpp:246-271)
    T v = add_rn(T(1), nx);
    if constexpr (sizeof(T) == 4) return (unsigned long long)((__float_as_uint(v) & 0x007FFFFFu) >> 2);
    else return ((unsigned long long)__double_as_longlong(v) & 0x000FFFFFFFFFFFFFull) >> 31;
}
template <class T> FT_D unsigned long long ph_cell(T nx) { // quantize_coord (src/sfc.peano_hilbert.hpp:472-476)
    double b = c_fmin(__dadd_rn(1.0, (double)nx), 0x1.fffffffffffffp+0);
    return (((unsigned long long)__double_as_longlong(b) & 0x000FFFFFFFFFFFFFull) >> 31) & 0x1FFFFFull;
}

template <int KIND> struct Delta {
    const unsigned long long *lo, *hi;
    int                       n;
    unsigned long long        ilo, ihi;
    int                       i;
    FT_D int operator()(int j) const {
        if (j < 0 || j >= n) return -1;
        unsigned long long jlo = lo[j];
        if (KIND == 2) {
            unsigned long long jhi = hi[j];
            if (jhi != ihi) return clz64(jhi ^ ihi) - 2;
            if (jlo != ilo) return 62 + clz64(jlo ^ ilo);
        } else {
            if (jlo != ilo) return clz64(jlo ^ ilo) - (KIND == 1 ? 1 : 0);
        }
        return (KIND == 2 ? 126 : 63) + clz64((unsigned long long)(long long)i ^ (unsigned long long)(long long)j);
    }
};

FT_D int sgn(int v) { return (v > 0) - (v < 0); }

// =========================================================================================
// Bounding-box folding: min: (v < m) ? v : m; max: (m < v) ? v : m, as sycl::minimum /
// sycl::maximum.  bb_block_reduce folds a block of kBboxThreads threads into thread 0.
// =========================================================================================
static constexpr int kBboxThreads = 256;

template <class T> FT_D void bb_fold(T *m, const T *v) {
#pragma unroll
    for (int d = 0; d < 3; ++d) {
        if (v[2 * d] < m[2 * d]) m[2 * d] = v[2 * d];
        if (m[2 * d + 1] < v[2 * d + 1]) m[2 * d + 1] = v[2 * d + 1];
    }
}
template <class T> FT_HD void bb_identity(T *m) {
    T lo, hi;
    if constexpr (std::is_floating_point<T>::value) {
        lo = std::is_same<T, float>::value ? (T)FLT_MAX : (T)DBL_MAX;
        hi = -lo;
    } else {
        lo = (T)~T(0);
        hi = 0;
    }
    m[0] = m[2] = m[4] = lo;
    m[1] = m[3] = m[5] = hi;
}

template <class T> FT_D void bb_block_reduce(T *m) {
    __shared__ T s[kBboxThreads / 32][6];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) {
        T o[6];
#pragma unroll
        for (int d = 0; d < 6; ++d) o[d] = __shfl_down_sync(0xffffffffu, m[d], off);
        bb_fold(m, o);
    }
    if (lane == 0)
#pragma unroll
        for (int d = 0; d < 6; ++d) s[w][d] = m[d];
    __syncthreads();
    if (w == 0) {
        if (lane < kBboxThreads / 32)
#pragma unroll
            for (int d = 0; d < 6; ++d) m[d] = s[lane][d];
        else
            bb_identity(m);
#pragma unroll
        for (int off = 16; off > 0; off >>= 1) {
            T o[6];
#pragma unroll
            for (int d = 0; d < 6; ++d) o[d] = __shfl_down_sync(0xffffffffu, m[d], off);
            bb_fold(m, o);
        }
    }
}

// Quantisation parameters of one axis from the box (src/hlbvh.hpp:389-394): the lower
// bound and 1 / (hi - lo), 0 for a flat axis.
template <class T> FT_D void sfc_axis_params(T lo, T hi, T &p_lo, T &p_inv) {
    T dd = sub_rn(hi, lo);
    if constexpr (sizeof(T) == 4) p_inv = (dd == 0.0f) ? 0.0f : __fdiv_rn(1.0f, dd);
    else p_inv = (dd == 0.0) ? 0.0 : __ddiv_rn(1.0, dd);
    p_lo = lo;
}

// SFC key of one point (sfc_encode, src/hlbvh.hpp:357-423).  par = {lo, inv} per axis (float
// coordinates only); integer coordinates are masked to their position bits (375-387).
template <class T, int SFC>
FT_D void encode_point(T x, T y, T z, const T *par, const uint8_t *s_rot, const uint8_t *s_sub,
                       unsigned long long &hi, unsigned long long &lo) {
    using C = Coord<T>;
    hi      = 0;
    lo      = 0;
    if constexpr (!C::is_float) {
        const unsigned long long mask = (1ull << C::bits) - 1ull;
        ph_key<C::bits>((unsigned long long)x & mask, (unsigned long long)y & mask, (unsigned long long)z & mask,
                        s_rot, s_sub, hi, lo);
    } else {
        // nx = clamp((p - min) * inv, 0, nextafter(1, 0)) in T (389-403)
        const T upper = (sizeof(T) == 4) ? (T)0x1.fffffep-1f : (T)0x1.fffffffffffffp-1;
        T       p[3]  = {x, y, z};
        unsigned long long c[3];
#pragma unroll
        for (int d = 0; d < 3; ++d) {
            T nx = c_fmin(c_fmax(mul_rn(sub_rn(p[d], par[2 * d]), par[2 * d + 1]), T(0)), upper);
            c[d] = (SFC == MORTON) ? morton_cell(nx) : ph_cell(nx);
        }
        if (SFC == MORTON) lo = spread3(c[0]) | (spread3(c[1]) << 1) | (spread3(c[2]) << 2);
        else ph_key<21>(c[0], c[1], c[2], s_rot, s_sub, hi, lo);
    }
}

// =========================================================================================
// Karras 2012 topology of internal node i of an n-leaf tree over sorted keys (src/hlbvh.hpp:
// 852-903): direction, range end by exponential + binary search, split by binary search.
// Child indices >= n-1 are leaves; leaves[i] receives the node's leaf count.
// =========================================================================================
template <int KIND>
FT_D void karras_node(const unsigned long long *klo, const unsigned long long *khi, int n, int i, int32_t *left,
                      int32_t *right, int32_t *parent, int32_t *leaves) {
    Delta<KIND> delta{klo, khi, n, klo[i], KIND == 2 ? khi[i] : 0ull, i};
    int d         = sgn(delta(i + 1) - delta(i - 1));
    int delta_min = delta(i - d);
    int l_max     = 2;
    while (delta(i + l_max * d) > delta_min) l_max *= 2;
    int l = 0;
    for (int t = l_max / 2; t >= 1; t /= 2)
        if (delta(i + (l + t) * d) > delta_min) l += t;
    int j          = i + l * d;
    int delta_node = delta(j);
    int s          = 0;
    int t_split    = 1;
    while (t_split <= l) t_split *= 2;
    t_split /= 2;
    for (int t = t_split; t >= 1; t /= 2)
        if (s + t < l && delta(i + (s + t) * d) > delta_node) s += t;
    int split  = i + s * d + min(d, 0);
    int lc     = (min(i, j) == split) ? split + n - 1 : split;
    int rc     = (max(i, j) == split + 1) ? split + 1 + n - 1 : split + 1;
    left[i]    = lc;
    right[i]   = rc;
    parent[lc] = i;
    parent[rc] = i;
    leaves[i]  = l + 1; // node i covers leaves i .. j
}

// =========================================================================================
// Bottom-up refit from one leaf (src/hlbvh.hpp:925-969): the thread climbs; at each parent
// the first arrival stops and the second merges both child boxes.  The merge also writes
// the traversal record (both child boxes + indices) and the subtree height.  Child boxes
// that other threads wrote in this launch are read through L2 (ld.cg) after the acquiring
// arrival.  A valid tree is climbed in fewer than n steps; a bad parent ends the climb.
// =========================================================================================
FT_D int atomic_add_acq_rel(int32_t *p, int v) {
    int old;
    asm volatile("atom.acq_rel.gpu.global.add.u32 %0, [%1], %2;" : "=r"(old) : "l"(p), "r"(v) : "memory");
    return old;
}

// The merge at internal node p (both children's boxes are final): p's box, its traversal
// record (both child boxes and indices, leaf counts and heights) and its height.
template <class T>
FT_D void refit_merge(int p, int n, const int32_t *__restrict__ left, const int32_t *__restrict__ right,
                      T *const *soa, NodeRec<T> *recs, uint8_t *height, const int32_t *__restrict__ leaves) {
    int l = left[p], r = right[p];
    T   lb[6], rb[6];
#pragma unroll
    for (int d = 0; d < 6; ++d) {
        lb[d] = __ldcg(soa[d] + l);
        rb[d] = __ldcg(soa[d] + r);
    }
    int hl = (l >= n - 1) ? 0 : (int)__ldcg(height + l);
    int hr = (r >= n - 1) ? 0 : (int)__ldcg(height + r);
    T   pb[6];
#pragma unroll
    for (int d = 0; d < 3; ++d) {
        pb[2 * d]     = box_min(lb[2 * d], rb[2 * d]);
        pb[2 * d + 1] = box_max(lb[2 * d + 1], rb[2 * d + 1]);
    }
#pragma unroll
    for (int d = 0; d < 6; ++d) __stcg(soa[d] + p, pb[d]);
    NodeRec<T> rec;
#pragma unroll
    for (int d = 0; d < 6; ++d) {
        rec.lb[d] = lb[d];
        rec.rb[d] = rb[d];
    }
    rec.l = l;
    rec.r = r;
#pragma unroll
    for (int d = 0; d < (int)(sizeof(rec.pad) / 4); ++d) rec.pad[d] = 0;
    // leaf counts (the Karras ranges) and heights of both children
    rec.pad[0] = (int32_t)rec_child_info(l >= n - 1 ? 1u : (uint32_t)leaves[l], (uint32_t)hl);
    rec.pad[1] = (int32_t)rec_child_info(r >= n - 1 ? 1u : (uint32_t)leaves[r], (uint32_t)hr);
    recs[p] = rec;
    int h   = 1 + max(hl, hr);
    __stcg(height + p, (uint8_t)min(h, 255));
}

// One step of a climb at node curr: the arrival at its parent.  Returns the parent when this
// arrival is the second (the merge is done, the climb goes on), else -1 (first arrival, the
// root, or a bad parent: the climb ends).
template <class T>
FT_D int refit_step(int curr, int n, const int32_t *__restrict__ left, const int32_t *__restrict__ right,
                    const int32_t *__restrict__ parent, T *const *soa, NodeRec<T> *recs, uint8_t *height,
                    int32_t *counters, const int32_t *__restrict__ leaves) {
    if (curr == 0) return -1;
    const int p = parent[curr];
    if (p < 0 || p >= n - 1) return -1;
    // one acquire-release arrival: this thread's writes of curr are released to the sibling
    // that arrives second, and the second arrival acquires the first's writes
    if (atomic_add_acq_rel(&counters[p], 1) == 0) return -1;
    refit_merge<T>(p, n, left, right, soa, recs, height, leaves);
    return p;
}

template <class T>
FT_D void refit_leaf(int leaf, int n, const int32_t *__restrict__ left, const int32_t *__restrict__ right,
                     const int32_t *__restrict__ parent, T *const *soa, NodeRec<T> *recs, uint8_t *height,
                     int32_t *counters, const int32_t *__restrict__ leaves) {
    int curr  = leaf + n - 1;
    int steps = 0;
    while (curr >= 0 && ++steps < n)
        curr = refit_step<T>(curr, n, left, right, parent, soa, recs, height, counters, leaves);
}


// =========================================================================================
// 4-wide record of internal node v (the fast walk's node format): its grandchildren, where
// a child that is a leaf stands for itself; boxes from the SoA arrays of the built tree.
// =========================================================================================
template <class T>
FT_D void collapse_node(int v, int n, const int32_t *__restrict__ left, const int32_t *__restrict__ right,
                        const T *const *soa, WideRec<T> *out) {
    int       ch[4] = {-1, -1, -1, -1};
    int       c     = 0;
    const int l = left[v], r = right[v];
    if (l >= n - 1) ch[c++] = l;
    else {
        ch[c++] = left[l];
        ch[c++] = right[l];
    }
    if (r >= n - 1) ch[c++] = r;
    else {
        ch[c++] = left[r];
        ch[c++] = right[r];
    }
    WideRec<T> w;
#pragma unroll
    for (int i = 0; i < 4; ++i) {
#pragma unroll
        for (int d = 0; d < 6; ++d) w.box[i][d] = ch[i] >= 0 ? soa[d][ch[i]] : T(0);
        w.child[i] = ch[i];
    }
    out[v] = w;
}

} // namespace ft
