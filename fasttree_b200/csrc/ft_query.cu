// ft_query.cu -- neighbour queries on sm_100a with the reference's exact semantics.
//
// Traversal (src/hlbvh.hpp:1079-1182, 1520-1647, 1690-1818): depth-first from the root with a
// 64-entry stack that drops both children when 62 entries are in use; a popped node is pruned
// when the heap holds k entries and its distance is >= the heap maximum; leaves are pushed
// into a binary max-heap (RegisterMaxHeap / LocalMaxHeap, src/maxheap.hpp:33-144, 340-478);
// internal nodes push the farther child first (ld2 <= rd2 -> push right, then left).  Results
// leave through an in-place heapsort.  Ties among equal distances therefore come out exactly
// as the reference orders them.
//
// B200 layout: one thread per query (queries in SFC leaf order, so a warp walks neighbouring
// regions), the child boxes of a node arrive in one 64/128-byte record, the stack keeps the
// distance computed at push time (the same value the reference recomputes at pop), and the
// heap lives in shared memory as [slot][thread] so that heap operations of a warp hit
// distinct banks.
#include <cuda_runtime.h>

#include <algorithm>

#include "ft_common.cuh"
#include "ft_internal.h"

namespace ft {

static constexpr int kStack = 64; // MAX_STACK_DEPTH (src/hlbvh.hpp:984)

template <class T, int PER, class D = typename Coord<T>::dist_t>
FT_D D box_dist(T px, T py, T pz, const T *b) {
    return Metric<T>::template dist<(PER != 0), (PER == 2)>(px, py, pz, b[0], b[1], b[2], b[3], b[4], b[5]);
}
template <class T, int PER, class D = typename Coord<T>::dist_t>
FT_D D node_dist_soa(const TreeDev<T> &t, int node, T px, T py, T pz) {
    return Metric<T>::template dist<(PER != 0), (PER == 2)>(px, py, pz, t.min_x[node], t.max_x[node], t.min_y[node], t.max_y[node],
                                         t.min_z[node], t.max_z[node]);
}

// -----------------------------------------------------------------------------------------
// Exact kNN: SELF = self_knn_query[_subset] (query = sorted leaf), else knn_query small-k.
// -----------------------------------------------------------------------------------------
// One query with the reference's traversal and heap; the heap rows live in shared memory
// at hd[slot * QT + tid] / hix[slot * QT + tid].  Writes the k results of row `row`.
template <class T, int CAP, int QT, int PER>
FT_D void exact_query(const TreeDev<T> &t, T px, T py, T pz, int self_leaf, int k, int ret_orig,
                      typename Coord<T>::dist_t *hd, int32_t *hix, int tid, size_t row,
                      unsigned long long *__restrict__ out_idx, typename Coord<T>::dist_t *__restrict__ out_dist,
                      uint32_t *status) {
    using D     = typename Coord<T>::dist_t;
    const int n = t.n;
#define HD(s) hd[(s) * QT + tid]
#define HI(s) hix[(s) * QT + tid]
    int sn[kStack];
    D   sd[kStack];
    int sp = 1;
    sn[0]  = 0;
    sd[0]  = node_dist_soa<T, PER>(t, 0, px, py, pz);
    int count = 0;
    D   hmax  = D(0);
    // each node is pushed once by its parent in a valid tree: 2n-1 pops at most
    long long budget = 2ll * n + 64;

    while (sp > 0) {
        if (--budget < 0) {
            atomicOr(status, STATUS_TRAVERSAL_LIMIT);
            break;
        }
        --sp;
        const int node = sn[sp];
        const D   d2   = sd[sp];
        if (count >= k && d2 >= hmax) continue; // should_prune
        if (node >= n - 1) {                    // leaf (the n == 1 root included)
            if (node == self_leaf) continue;
            const int32_t id = ret_orig ? t.orig_idx[node] : node - (n - 1);
            if (count < k) { // append + sift_up
                int i = count;
                while (i > 0) {
                    int p  = (i - 1) >> 1;
                    D   pd = HD(p);
                    if (d2 <= pd) break;
                    HD(i) = pd;
                    HI(i) = HI(p);
                    i     = p;
                }
                HD(i) = d2;
                HI(i) = id;
                ++count;
            } else if (d2 < HD(0)) { // replace root + sift_down
                int i = 0;
                for (;;) {
                    int l = 2 * i + 1;
                    if (l >= k) break;
                    int r  = l + 1;
                    int c  = i;
                    D   cd = d2;
                    D   ld = HD(l);
                    if (ld > cd) {
                        c  = l;
                        cd = ld;
                    }
                    if (r < k) {
                        D rd = HD(r);
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
                HD(i) = d2;
                HI(i) = id;
            }
            if (count >= k) hmax = HD(0);
        } else {
            T   lb[6], rb[6];
            int l, r;
            load_rec(t.recs, node, lb, rb, l, r);
            const D ld2 = box_dist<T, PER>(px, py, pz, lb);
            const D rd2 = box_dist<T, PER>(px, py, pz, rb);
            if (sp < kStack - 2) {
                if (ld2 <= rd2) {
                    sn[sp] = r;
                    sd[sp] = rd2;
                    sn[sp + 1] = l;
                    sd[sp + 1] = ld2;
                } else {
                    sn[sp] = l;
                    sd[sp] = ld2;
                    sn[sp + 1] = r;
                    sd[sp + 1] = rd2;
                }
                sp += 2;
            }
        }
    }

    // extract_sorted / sort_in_place: heapsort in place
    for (int hs = count; hs > 1; --hs) {
        D       last  = HD(hs - 1);
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
            D   cd = last;
            D   ld = HD(l);
            if (ld > cd) {
                c  = l;
                cd = ld;
            }
            if (r < size) {
                D rd = HD(r);
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
    const size_t off = row * (size_t)k;
    for (int i = 0; i < k; ++i) {
        if (i < count) {
            __stcs(out_idx + off + i, (unsigned long long)(long long)HI(i));
            __stcs(out_dist + off + i, HD(i));
        } else {
            __stcs(out_idx + off + i, ~0ull);
            __stcs(out_dist + off + i, dist_missing<D>());
        }
    }
#undef HD
#undef HI
}

// Query point of a self query (sorted leaf `rank`); false (and an empty row) for a bad id.
template <class T>
FT_D bool self_point(const TreeDev<T> &t, int rank, int k, size_t row, unsigned long long *out_idx,
                     typename Coord<T>::dist_t *out_dist, uint32_t *status, T &px, T &py, T &pz) {
    using D = typename Coord<T>::dist_t;
    if (rank < 0 || rank >= t.n) { // invalid caller leaf id: empty row, flag the call
        atomicOr(status, STATUS_BAD_INPUT);
        for (int i = 0; i < k; ++i) {
            out_idx[row * k + i]  = ~0ull;
            out_dist[row * k + i] = dist_missing<D>();
        }
        return false;
    }
    int slot = rank + t.n - 1;
    px       = t.min_x[slot];
    py       = t.min_y[slot];
    pz       = t.min_z[slot];
    return true;
}

template <class T, int CAP, int QT, bool SELF, int PER>
__global__ void __launch_bounds__(QT) exact_knn_kernel(TreeDev<T> t_all, BatchDev bt, const T *__restrict__ qx,
                                                       const T *__restrict__ qy, const T *__restrict__ qz,
                                                       const int32_t *__restrict__ leaf_ids, int num, int k,
                                                       int exclude_self, int ret_orig,
                                                       unsigned long long *__restrict__ out_idx,
                                                       typename Coord<T>::dist_t *__restrict__ out_dist,
                                                       uint32_t *status) {
    using D = typename Coord<T>::dist_t;
    extern __shared__ __align__(16) unsigned char smem[];
    D       *hd  = reinterpret_cast<D *>(smem);
    int32_t *hix = reinterpret_cast<int32_t *>(hd + CAP * QT);
    const int tid = threadIdx.x;
    const int q   = blockIdx.x * QT + tid;
    if (q >= num) return;
    T          px, py, pz;
    int        self_leaf = -1;
    TreeDev<T> t         = t_all;
    if (SELF) {
        int rank;
        if (bt.off) { // batched sets: row q is leaf q - off[s] of set s
            const int s = find_set(bt.off, bt.S, q);
            t           = set_view(t_all, bt, s);
            rank        = q - (int)bt.off[s];
        } else {
            rank = leaf_ids ? leaf_ids[q] : q;
        }
        if (!self_point(t, rank, k, (size_t)q, out_idx, out_dist, status, px, py, pz)) return;
        if (exclude_self) self_leaf = rank + t.n - 1;
    } else {
        px = qx[q];
        py = qy[q];
        pz = qz[q];
    }
    exact_query<T, CAP, QT, PER>(t, px, py, pz, self_leaf, k, ret_orig, hd, hix, tid, (size_t)q, out_idx, out_dist,
                                 status);
}

// Replays the self queries listed by the fast traversal (ranks[i] -> output row rows[i]) with
// the reference traversal; grid-stride over a count that lives on the device, so no host
// synchronisation is needed between the two launches.  For batched sets the row names the
// set and the rank is local to it.
template <class T, int CAP, int QT, int PER>
__global__ void __launch_bounds__(QT) exact_replay_kernel(TreeDev<T> t_all, BatchDev bt,
                                                          const int32_t *__restrict__ ranks,
                                                          const int32_t *__restrict__ rows,
                                                          const uint32_t *__restrict__ count_dev, int k,
                                                          int exclude_self, int ret_orig,
                                                          unsigned long long *__restrict__ out_idx,
                                                          typename Coord<T>::dist_t *__restrict__ out_dist,
                                                          uint32_t *status) {
    using D = typename Coord<T>::dist_t;
    extern __shared__ __align__(16) unsigned char smem[];
    D       *hd    = reinterpret_cast<D *>(smem);
    int32_t *hix   = reinterpret_cast<int32_t *>(hd + CAP * QT);
    const int tid  = threadIdx.x;
    const int cnt  = (int)*count_dev;
    for (int i = blockIdx.x * QT + tid; i < cnt; i += gridDim.x * QT) {
        const int  rank = ranks[i];
        const int  row  = rows[i];
        TreeDev<T> t    = bt.off ? set_view(t_all, bt, find_set(bt.off, bt.S, row)) : t_all;
        T          px, py, pz;
        if (!self_point(t, rank, k, (size_t)row, out_idx, out_dist, status, px, py, pz)) continue;
        exact_query<T, CAP, QT, PER>(t, px, py, pz, exclude_self ? rank + t.n - 1 : -1, k, ret_orig, hd, hix, tid,
                                     (size_t)row, out_idx, out_dist, status);
    }
}

// -----------------------------------------------------------------------------------------
// knn_query_large_k (src/hlbvh.hpp:1185-1388) with SortedMergeHeap (src/maxheap.hpp:193-324):
// one warp per query; every lane walks the same traversal, each leaf is merged as a 32-wide
// batch holding one real candidate, and the list is re-sorted with the reference's bitonic
// network so equal distances land where the reference puts them.
// -----------------------------------------------------------------------------------------
template <class D> FT_D void warp_bitonic(D *d, int32_t *ix, int n, int lane) {
    for (int kk = 2; kk <= n; kk <<= 1)
        for (int j = kk >> 1; j > 0; j >>= 1) {
            for (int i = lane; i < n; i += 32) {
                int l = i ^ j;
                if (l > i && l < n) {
                    bool asc = (i & kk) == 0;
                    D    a = d[i], b = d[l];
                    if ((a > b) == asc) {
                        d[i] = b;
                        d[l] = a;
                        int32_t t = ix[i];
                        ix[i]     = ix[l];
                        ix[l]     = t;
                    }
                }
            }
            __syncwarp();
        }
}

static constexpr int kMergeWarps = 4;

// One warp runs the SortedMergeHeap traversal of one query point and writes row `row`.
template <class T, int PER>
FT_D void merge_query(const TreeDev<T> &t, T px, T py, T pz, int k, int cap, int ret_orig, size_t row,
                      typename Coord<T>::dist_t *hd, int32_t *hix, typename Coord<T>::dist_t *sgd, int32_t *sgi,
                      int lane, unsigned long long *__restrict__ out_idx,
                      typename Coord<T>::dist_t *__restrict__ out_dist, uint32_t *status) {
    using D      = typename Coord<T>::dist_t;
    const D DMAX = dist_heap_max<D>();
    for (int i = lane; i < cap; i += 32) {
        hd[i]  = DMAX;
        hix[i] = -1;
    }
    int count = 0;
    __syncwarp();
    const int n = t.n;
    int       sn[kStack];
    D         sd[kStack];
    int       sp = 1;
    sn[0]        = 0;
    sd[0]        = node_dist_soa<T, PER>(t, 0, px, py, pz);
    long long budget = 2ll * n + 64;
    while (sp > 0) {
        if (--budget < 0) {
            if (lane == 0) atomicOr(status, STATUS_TRAVERSAL_LIMIT);
            break;
        }
        --sp;
        const int node = sn[sp];
        const D   d2   = sd[sp];
        if (count >= k && d2 >= hd[k - 1]) continue;
        if (node >= n - 1) {
            const int32_t id = ret_orig ? t.orig_idx[node] : node - (n - 1);
            // merge_batch: stage [candidate, 31 empty lanes], bitonic-sort it (32)
            sgd[lane] = (lane == 0) ? d2 : DMAX;
            sgi[lane] = (lane == 0) ? id : -1;
            __syncwarp();
            if (d2 == DMAX) warp_bitonic(sgd, sgi, 32, lane); // otherwise already sorted
            // append at [count, count + 32) within cap
            int dst = count + lane;
            D   vd  = sgd[lane];
            int vi  = sgi[lane];
            __syncwarp();
            if (dst < cap) {
                hd[dst]  = vd;
                hix[dst] = vi;
            }
            const int nc = min(count + 32, cap);
            int       p2 = 1;
            while (p2 < nc) p2 <<= 1;
            for (int i = nc + lane; i < p2 && i < cap; i += 32) {
                hd[i]  = DMAX;
                hix[i] = -1;
            }
            __syncwarp();
            warp_bitonic(hd, hix, p2, lane);
            count = min(nc, k);
        } else {
            T   lb[6], rb[6];
            int l, r;
            load_rec(t.recs, node, lb, rb, l, r);
            const D ld2 = box_dist<T, PER>(px, py, pz, lb);
            const D rd2 = box_dist<T, PER>(px, py, pz, rb);
            if (sp < kStack - 2) {
                if (ld2 <= rd2) {
                    sn[sp] = r;
                    sd[sp] = rd2;
                    sn[sp + 1] = l;
                    sd[sp + 1] = ld2;
                } else {
                    sn[sp] = l;
                    sd[sp] = ld2;
                    sn[sp + 1] = r;
                    sd[sp + 1] = rd2;
                }
                sp += 2;
            }
        }
    }
    const size_t off = row * (size_t)k;
    for (int i = lane; i < k; i += 32) {
        if (hix[i] >= 0) {
            out_idx[off + i]  = (unsigned long long)(long long)hix[i];
            out_dist[off + i] = hd[i];
        } else {
            out_idx[off + i]  = ~0ull;
            out_dist[off + i] = dist_missing<D>();
        }
    }
    __syncwarp();
}

template <class T, int PER>
__global__ void __launch_bounds__(32 * kMergeWarps)
    merge_knn_kernel(TreeDev<T> t, const T *__restrict__ qx, const T *__restrict__ qy, const T *__restrict__ qz,
                     int nq, int k, int cap, int ret_orig, unsigned long long *__restrict__ out_idx,
                     typename Coord<T>::dist_t *__restrict__ out_dist, uint32_t *status) {
    using D = typename Coord<T>::dist_t;
    extern __shared__ __align__(16) unsigned char smem[];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const int q    = blockIdx.x * kMergeWarps + w;
    if (q >= nq) return;
    D       *hd  = reinterpret_cast<D *>(smem) + (size_t)w * (cap + 32);
    int32_t *hix = reinterpret_cast<int32_t *>(reinterpret_cast<D *>(smem) + (size_t)kMergeWarps * (cap + 32)) +
                   (size_t)w * (cap + 32);
    merge_query<T, PER>(t, qx[q], qy[q], qz[q], k, cap, ret_orig, (size_t)q, hd, hix, hd + cap, hix + cap, lane,
                        out_idx, out_dist, status);
}

// Reruns the external queries listed by the fast walk (rows[i], *count_dev of them) with the
// SortedMergeHeap traversal: one warp per listed row, grid-stride over the device count.
template <class T, int PER>
__global__ void __launch_bounds__(32 * kMergeWarps)
    merge_replay_kernel(TreeDev<T> t, const T *__restrict__ qx, const T *__restrict__ qy, const T *__restrict__ qz,
                        const int32_t *__restrict__ rows, const uint32_t *__restrict__ count_dev, int k, int cap,
                        int ret_orig, unsigned long long *__restrict__ out_idx,
                        typename Coord<T>::dist_t *__restrict__ out_dist, uint32_t *status) {
    using D = typename Coord<T>::dist_t;
    extern __shared__ __align__(16) unsigned char smem[];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    D        *hd   = reinterpret_cast<D *>(smem) + (size_t)w * (cap + 32);
    int32_t  *hix  = reinterpret_cast<int32_t *>(reinterpret_cast<D *>(smem) + (size_t)kMergeWarps * (cap + 32)) +
                   (size_t)w * (cap + 32);
    const int cnt  = (int)*count_dev;
    for (int i = blockIdx.x * kMergeWarps + w; i < cnt; i += gridDim.x * kMergeWarps) {
        const int row = rows[i];
        merge_query<T, PER>(t, qx[row], qy[row], qz[row], k, cap, ret_orig, (size_t)row, hd, hix, hd + cap,
                            hix + cap, lane, out_idx, out_dist, status);
    }
}

// The same for the register / local heap tier (knn_query with k <= 32 or MAXK <= 32).
template <class T, int CAP, int QT, int PER>
__global__ void __launch_bounds__(QT)
    exact_replay_ext_kernel(TreeDev<T> t, const T *__restrict__ qx, const T *__restrict__ qy,
                            const T *__restrict__ qz, const int32_t *__restrict__ rows,
                            const uint32_t *__restrict__ count_dev, int k, int ret_orig,
                            unsigned long long *__restrict__ out_idx, typename Coord<T>::dist_t *__restrict__ out_dist,
                            uint32_t *status) {
    using D = typename Coord<T>::dist_t;
    extern __shared__ __align__(16) unsigned char smem[];
    D       *hd   = reinterpret_cast<D *>(smem);
    int32_t *hix  = reinterpret_cast<int32_t *>(hd + CAP * QT);
    const int tid = threadIdx.x;
    const int cnt = (int)*count_dev;
    for (int i = blockIdx.x * QT + tid; i < cnt; i += gridDim.x * QT) {
        const int row = rows[i];
        exact_query<T, CAP, QT, PER>(t, qx[row], qy[row], qz[row], -1, k, ret_orig, hd, hix, tid, (size_t)row,
                                     out_idx, out_dist, status);
    }
}

// -----------------------------------------------------------------------------------------
// range_query (src/hlbvh.hpp:2046-2119): left-first DFS, descend while d2 <= rmax^2, count
// leaves with d2 >= rmin^2, store while the row has room; subtrees inside the shell are
// counted whole once the row is full (same counts, far fewer visits for large radii).
// -----------------------------------------------------------------------------------------
// Squared distance from the query to the farthest point of a box, never below the distance
// node_distance_sq gives any point inside it: the same operations per axis on the farther
// face (rounding and the shift are monotone).  42-bit periodic trees (PER 2): the wrapped
// gap over [lo, hi] peaks at the query's antipode when the interval holds it, else at an
// end.  false when no such bound is provided (general periodic form).
template <class T, int PER>
FT_D bool far_dist(T px, T py, T pz, const TreeDev<T> &t, int node, typename Coord<T>::dist_t &out) {
    using C      = Coord<T>;
    const T p[3] = {px, py, pz};
    const T lo[3] = {t.min_x[node], t.min_y[node], t.min_z[node]};
    const T hi[3] = {t.max_x[node], t.max_y[node], t.max_z[node]};
    if constexpr (C::is_float) {
        T f[3];
#pragma unroll
        for (int d = 0; d < 3; ++d) f[d] = c_fmax(sub_rn(hi[d], p[d]), sub_rn(p[d], lo[d]));
        out = (double)add_rn(add_rn(mul_rn(f[0], f[0]), mul_rn(f[1], f[1])), mul_rn(f[2], f[2]));
        return true;
    } else if constexpr (PER == 0) {
        unsigned long long s = 0;
#pragma unroll
        for (int d = 0; d < 3; ++d) {
            const unsigned long long a = p[d] > lo[d] ? (unsigned long long)(T)(p[d] - lo[d]) : 0ull;
            const unsigned long long b = hi[d] > p[d] ? (unsigned long long)(T)(hi[d] - p[d]) : 0ull;
            s += Metric<T>::sq((a > b ? a : b) >> C::dist_shift);
        }
        out = s;
        return true;
    } else if constexpr (PER == 2 && sizeof(T) == 8) {
        constexpr unsigned long long M = (1ull << C::bits) - 1ull, H = 1ull << (C::bits - 1);
        unsigned long long           s = 0;
#pragma unroll
        for (int d = 0; d < 3; ++d) {
            const unsigned long long v = (unsigned long long)p[d] & M, l = lo[d], h = hi[d];
            const unsigned long long a = (v + H) & M; // antipode
            auto w = [&](unsigned long long x) {
                const unsigned long long u = (x - v) & M, e = (v - x) & M;
                return u < e ? u : e;
            };
            const unsigned long long wl = w(l), wh = w(h);
            const unsigned long long g  = (a >= l && a <= h) ? H : (wl > wh ? wl : wh);
            s += Metric<T>::sq((unsigned long long)(uint32_t)(g >> C::dist_shift));
        }
        out = s;
        return true;
    } else {
        return false;
    }
}

// far_dist for a box held in registers (minx, maxx, miny, maxy, minz, maxz).
template <class T, int PER>
FT_D bool far_dist_box(T px, T py, T pz, const T b[6], typename Coord<T>::dist_t &out) {
    using C      = Coord<T>;
    const T p[3] = {px, py, pz};
    if constexpr (C::is_float) {
        T f[3];
#pragma unroll
        for (int d = 0; d < 3; ++d) f[d] = c_fmax(sub_rn(b[2 * d + 1], p[d]), sub_rn(p[d], b[2 * d]));
        out = (double)add_rn(add_rn(mul_rn(f[0], f[0]), mul_rn(f[1], f[1])), mul_rn(f[2], f[2]));
        return true;
    } else if constexpr (PER == 0) {
        unsigned long long s = 0;
#pragma unroll
        for (int d = 0; d < 3; ++d) {
            const T                  lo = b[2 * d], hi = b[2 * d + 1];
            const unsigned long long a  = p[d] > lo ? (unsigned long long)(T)(p[d] - lo) : 0ull;
            const unsigned long long c  = hi > p[d] ? (unsigned long long)(T)(hi - p[d]) : 0ull;
            s += Metric<T>::sq((a > c ? a : c) >> C::dist_shift);
        }
        out = s;
        return true;
    } else if constexpr (PER == 2 && sizeof(T) == 8) {
        constexpr unsigned long long M = (1ull << C::bits) - 1ull, H = 1ull << (C::bits - 1);
        unsigned long long           s = 0;
#pragma unroll
        for (int d = 0; d < 3; ++d) {
            const unsigned long long v = (unsigned long long)p[d] & M, l = b[2 * d], h = b[2 * d + 1];
            const unsigned long long a = (v + H) & M; // antipode
            auto w = [&](unsigned long long x) {
                const unsigned long long u = (x - v) & M, e = (v - x) & M;
                return u < e ? u : e;
            };
            const unsigned long long wl = w(l), wh = w(h);
            const unsigned long long g  = (a >= l && a <= h) ? H : (wl > wh ? wl : wh);
            s += Metric<T>::sq((unsigned long long)(uint32_t)(g >> C::dist_shift));
        }
        out = s;
        return true;
    } else {
        return false;
    }
}

// range_query on trees of height <= 62, where the reference's stack guard (which drops both
// children of a node popped with 62 entries below it) cannot fire: the stack then only
// orders the walk, so a child can be judged when its parent is expanded.  A child beyond
// r_max is not pushed; once the row is full a child inside the shell is counted from its leaf
// count (kept in the parent's record) instead of being walked.  Results are still written in
// the reference's depth-first, left-first order.
// The query's squared shell radii in the walk's distance units (src/hlbvh.hpp:2032-2043).
template <class T>
FT_D void range_radii(const T *__restrict__ rmin, const T *__restrict__ rmax, int q, typename Coord<T>::dist_t &rm2,
                      typename Coord<T>::dist_t &RM2) {
    using C = Coord<T>;
    if constexpr (C::is_float) {
        const double a = (double)rmin[q], b = (double)rmax[q];
        rm2            = __dmul_rn(a, a);
        RM2            = __dmul_rn(b, b);
    } else {
        const unsigned long long a = (unsigned long long)rmin[q] >> C::dist_shift;
        const unsigned long long b = (unsigned long long)rmax[q] >> C::dist_shift;
        rm2                        = a * a;
        RM2                        = b * b;
    }
}

// One query's range walk on a tree of height <= 62; returns its full count.
template <class T, int PER>
FT_D int range_one(const TreeDev<T> &t, T px, T py, T pz, typename Coord<T>::dist_t rm2,
                   typename Coord<T>::dist_t RM2, int32_t *__restrict__ results, size_t off, int max_per, int ret_orig,
                   uint32_t *status) {
    using D     = typename Coord<T>::dist_t;
    const int n = t.n;
    int       count = 0;
    // the stack holds node indices only: a leaf is stacked only when it lies in the shell
    // (its distance is known when its parent is expanded), an internal node when it is within
    // r_max, so a popped leaf is always counted
    int       sn[kStack];
    int       sp = 0;
    const D   d0 = node_dist_soa<T, PER>(t, 0, px, py, pz);
    if (d0 <= RM2 && (n > 1 || d0 >= rm2)) {
        sn[0] = 0;
        sp    = 1;
    }
    long long budget = 2ll * n + 64;
    while (sp > 0) {
        if (--budget < 0) {
            atomicOr(status, STATUS_TRAVERSAL_LIMIT);
            break;
        }
        --sp;
        const int node = sn[sp];
        if (node >= n - 1) { // leaf in the shell (the n == 1 root included)
            if (count < max_per) results[off + count] = ret_orig ? t.orig_idx[node] : node - (n - 1);
            ++count;
            continue;
        }
        T        lb[6], rb[6];
        int      l, r;
        uint32_t il, ir;
        load_rec_info(t.recs, node, lb, rb, l, r, il, ir);
        const D    dl = box_dist<T, PER>(px, py, pz, lb), dr = box_dist<T, PER>(px, py, pz, rb);
        const bool full = count >= max_per;
        // right first on the stack, so the left subtree is walked (and written) first
#pragma unroll
        for (int side = 1; side >= 0; --side) {
            const int      c  = side ? r : l;
            const D        dc = side ? dr : dl;
            const uint32_t ic = side ? ir : il;
            if (!(dc <= RM2)) continue;
            if (c >= n - 1 && !(dc >= rm2)) continue; // a leaf inside r_min
            if (full) {
                if (c >= n - 1) { // a leaf: counted now
                    ++count;
                    continue;
                }
                if (dc >= rm2 && info_leaves(ic) < kInfoCountMax) {
                    D far;
                    if (far_dist_box<T, PER>(px, py, pz, side ? rb : lb, far) && far <= RM2) {
                        count += (int)info_leaves(ic); // every leaf below lies in the shell
                        continue;
                    }
                }
            }
            if (sp >= kStack) {
                atomicOr(status, STATUS_TRAVERSAL_LIMIT);
                break;
            }
            sn[sp] = c;
            ++sp;
        }
    }
    return count;
}

// One query's range walk over the 4-wide records (trees of height <= 62 whose box distance
// is monotone over nested boxes): each expansion judges up to four grandchildren at once,
// and they are stacked rightmost first, so the walk stays depth-first and left-first and
// writes the row in the reference's order.  Skipping the binary level between is exact here:
// a grandchild beyond r_max has a parent beyond it too, and the reference prunes there.  Once
// the row is full, a leaf is counted at once and an internal grandchild inside the shell is
// counted from its leaf count.
// STOP: return as soon as the row is full (*filled set), leaving the count to range_count_group.
template <class T, int PER, bool STOP = false>
FT_D int range_one_wide(const TreeDev<T> &t, T px, T py, T pz, typename Coord<T>::dist_t rm2,
                        typename Coord<T>::dist_t RM2, int32_t *__restrict__ results, size_t off, int max_per,
                        int ret_orig, uint32_t *status, bool *filled = nullptr) {
    using D     = typename Coord<T>::dist_t;
    const int n = t.n;
    int       count = 0;
    int       sn[kStack * 2];
    int       sp = 0;
    const D   d0 = node_dist_soa<T, PER>(t, 0, px, py, pz);
    if (d0 <= RM2 && (n > 1 || d0 >= rm2)) {
        sn[0] = 0;
        sp    = 1;
    }
    if constexpr (STOP) {
        *filled = false;
        if (max_per <= 0) {
            *filled = sp > 0;
            return 0;
        }
    }
    long long budget = 2ll * n + 64;
    while (sp > 0) {
        if (--budget < 0) {
            atomicOr(status, STATUS_TRAVERSAL_LIMIT);
            break;
        }
        const int node = sn[--sp];
        if (node >= n - 1) { // leaf in the shell (the n == 1 root included)
            if (count < max_per) results[off + count] = ret_orig ? t.orig_idx[node] : node - (n - 1);
            ++count;
            if constexpr (STOP) {
                if (count >= max_per) {
                    *filled = true;
                    break;
                }
            }
            continue;
        }
        T   bx[4][6];
        int ch[4];
        load_wide(t.wide, node, bx, ch);
        D d[4];
#pragma unroll
        for (int i = 0; i < 4; ++i) d[i] = ch[i] >= 0 ? box_dist<T, PER>(px, py, pz, bx[i]) : D(0);
        const bool full = count >= max_per;
        bool       over = false;
#pragma unroll
        for (int i = 3; i >= 0; --i) {
            const int c = ch[i];
            if (c < 0 || !(d[i] <= RM2)) continue;
            if (c >= n - 1) {             // a leaf
                if (!(d[i] >= rm2)) continue; // inside r_min
                if (full) {
                    ++count;
                    continue;
                }
            } else if (full && d[i] >= rm2) {
                D far;
                if (far_dist_box<T, PER>(px, py, pz, bx[i], far) && far <= RM2) {
                    count += t.leaves[c]; // every leaf below lies in the shell
                    continue;
                }
            }
            if (sp >= kStack * 2) {
                over = true;
                break;
            }
            sn[sp++] = c;
        }
        if (over) {
            atomicOr(status, STATUS_TRAVERSAL_LIMIT);
            break;
        }
    }
    return count;
}

template <class T, int PER>
__global__ void __launch_bounds__(128)
    range_wide_kernel(TreeDev<T> t, const T *__restrict__ qx, const T *__restrict__ qy, const T *__restrict__ qz,
                      const T *__restrict__ rmin, const T *__restrict__ rmax, int nq, int32_t *__restrict__ results,
                      int32_t *__restrict__ counts, int max_per, int ret_orig, const uint32_t *__restrict__ order,
                      uint32_t *status) {
    using D     = typename Coord<T>::dist_t;
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= nq) return;
    const int q = order ? (int)order[i] : i;
    D         rm2, RM2;
    range_radii<T>(rmin, rmax, q, rm2, RM2);
    counts[q] = range_one_wide<T, PER>(t, qx[q], qy[q], qz[q], rm2, RM2, results, (size_t)q * (size_t)max_per,
                                       max_per, ret_orig, status);
}

// -----------------------------------------------------------------------------------------
// range_query counts, a warp's queries together.  A row's count is the number of leaves in
// the query's shell (rmin^2 <= d <= rmax^2): on trees where the box distance is monotone over
// nested boxes (the 4-wide walk's condition) a leaf's own distance decides it, whatever order
// the walk takes, so the count needs no walk order.  The lanes that still need a count (their
// rows are full) are neighbours on the curve; their query points lie in a small group box.
// For a node box, group_near_far bounds, per axis, the gap node_distance_sq measures between
// any of the group's points and any point of the box (near: no gap is smaller; far: none is
// larger); the squared distances built from them bound every lane's distance to every leaf
// below the node, since the shift, the squares, rounding and the sums are monotone.  A node
// beyond every lane's r_max is skipped; one inside every lane's shell adds its leaf count to
// every lane; the rest are expanded, and their leaves are staged for a test by each lane.
// -----------------------------------------------------------------------------------------
// Group frame: per axis the group's points lie in [g0, g0 + span] (for the 42-bit periodic
// metric an arc of the circle starting at g0; for floating point, [g0, g1]).
template <class T> struct RangeGroup {
    T                  g0[3], g1[3];
    unsigned long long span[3];
};

template <class T, int PER>
FT_D void group_near_far(const RangeGroup<T> &g, const T b[6], typename Coord<T>::dist_t &near,
                         typename Coord<T>::dist_t &far) {
    using C = Coord<T>;
    if constexpr (C::is_float) {
        T n3[3], f3[3];
#pragma unroll
        for (int a = 0; a < 3; ++a) {
            const T lo = b[2 * a], hi = b[2 * a + 1];
            n3[a] = c_fmax(c_fmax(T(0), sub_rn(lo, g.g1[a])), sub_rn(g.g0[a], hi));
            f3[a] = c_fmax(sub_rn(hi, g.g0[a]), sub_rn(g.g1[a], lo));
        }
        near = (double)add_rn(add_rn(mul_rn(n3[0], n3[0]), mul_rn(n3[1], n3[1])), mul_rn(n3[2], n3[2]));
        far  = (double)add_rn(add_rn(mul_rn(f3[0], f3[0]), mul_rn(f3[1], f3[1])), mul_rn(f3[2], f3[2]));
    } else if constexpr (PER == 2) {
        // gaps between the arc G = [g0, g0 + span] and the box [lo, hi] are the circular
        // distances w(u) = min(u, P - u) of the differences u in D = [lo - g0 - span, hi - g0]
        // (mod P), an arc of length len: w is 0 where D holds 0, P/2 where it holds P/2, and
        // otherwise takes its extremes at D's ends
        constexpr unsigned long long P = 1ull << C::bits, M = P - 1ull, H = P >> 1;
        unsigned long long sn = 0, sf = 0;
#pragma unroll
        for (int a = 0; a < 3; ++a) {
            const unsigned long long lo = (unsigned long long)b[2 * a], hi = (unsigned long long)b[2 * a + 1];
            const unsigned long long st  = (lo - (unsigned long long)g.g0[a] - g.span[a]) & M;
            const unsigned long long len = (hi - lo) + g.span[a];
            unsigned long long       gn = 0, gf = H;
            if (len < P) {
                const unsigned long long en = (st + len) & M;
                const unsigned long long wa = st <= H ? st : P - st, we = en <= H ? en : P - en;
                const bool               z  = st == 0 || st + len >= P;
                const bool               h  = ((H - st) & M) <= len;
                gn = z ? 0ull : (wa < we ? wa : we);
                gf = h ? H : (wa > we ? wa : we);
            }
            sn += Metric<T>::sq((unsigned long long)(uint32_t)(gn >> C::dist_shift));
            sf += Metric<T>::sq((unsigned long long)(uint32_t)(gf >> C::dist_shift));
        }
        near = sn;
        far  = sf;
    } else {
        unsigned long long sn = 0, sf = 0;
#pragma unroll
        for (int a = 0; a < 3; ++a) {
            const T lo = b[2 * a], hi = b[2 * a + 1], g0 = g.g0[a], g1 = g.g1[a];
            const unsigned long long gn = lo > g1   ? (unsigned long long)(T)(lo - g1)
                                          : g0 > hi ? (unsigned long long)(T)(g0 - hi)
                                                    : 0ull;
            const unsigned long long fa = g1 > lo ? (unsigned long long)(T)(g1 - lo) : 0ull;
            const unsigned long long fb = hi > g0 ? (unsigned long long)(T)(hi - g0) : 0ull;
            sn += Metric<T>::sq(gn >> C::dist_shift);
            sf += Metric<T>::sq((fa > fb ? fa : fb) >> C::dist_shift);
        }
        near = sn;
        far  = sf;
    }
}

// Offset of coordinate v from the group's corner, as a float for the leaf filter: the signed
// 42-bit wrapped difference (periodic), else the plain difference.
template <class T, int PER> FT_D float group_off(T v, const RangeGroup<T> &g, int a) {
    if constexpr (Coord<T>::is_float) {
        return (float)sub_rn(v, g.g0[a]);
    } else if constexpr (PER == 2) {
        constexpr int sh = 64 - Coord<T>::bits;
        return (float)((long long)(((unsigned long long)v - (unsigned long long)g.g0[a]) << sh) >> sh);
    } else {
        return (float)((long long)(unsigned long long)v - (long long)(unsigned long long)g.g0[a]);
    }
}

// range_split_kernel's shape: two-warp blocks (a block keeps its SM slots until its slowest
// warp ends, and the warps' work is very uneven) compiled for 8 resident blocks (124
// registers a thread, no spills).  Measured on 10M clustered points, all N queries, back to
// back on one GPU: 4-warp blocks 2.83 s, 2-warp 2.85 s, 1-warp 2.80 s (123 registers each),
// 2-warp with 10 / 12 resident blocks 2.42 / 2.44 s; with the threshold leaf filter, 8 / 10 /
// 12 resident blocks 1.93 / 2.05 / 2.11 s (the tighter budgets spill).
#ifndef FT_RANGE_WARPS
#define FT_RANGE_WARPS 2
#endif
#ifndef FT_RANGE_MINB
#define FT_RANGE_MINB 8
#endif
static constexpr int kRangeWarps = FT_RANGE_WARPS, kRangeGStack = 512, kRangeStage = 256;
// The group counts a warp's full rows together when its points' largest axis extent is at
// most 1/FT_RANGE_SPREAD of the smallest radius (measured on 10M clustered points, r = 2e-3 of
// the box, all N queries: factors 1 / 4 / 16 2.38 / 2.39 / 3.48 s, every group together
// 2.37 s, the per-query 4-wide walk 5.87 s; then 2.04 s with the threshold leaf filter, of
// which the rows take 0.12 s).
#ifndef FT_RANGE_SPREAD
#define FT_RANGE_SPREAD 1
#endif

// The group count of the lanes with `need` (every lane of the warp calls it).  Returns false
// (counts unset) when the group is too spread out for its bounds to help (FORCE: only when
// the float filter's accuracy needs it), or a stack would overflow; the caller then counts
// per lane.  count: this lane's shell count.
template <class T, int PER, bool FORCE = false>
FT_D bool range_count_group(const TreeDev<T> &t, bool need, T px, T py, T pz, typename Coord<T>::dist_t rm2,
                            typename Coord<T>::dist_t RM2, int32_t *stk, float4 *stage, int &count) {
    using C                = Coord<T>;
    using D                = typename C::dist_t;
    const unsigned FULL    = 0xffffffffu;
    const int      lane    = threadIdx.x & 31;
    const int      n       = t.n;
    if (n < 2) return false;
    if constexpr (PER == 1) return false; // the general periodic form: no group bounds
    RangeGroup<T> g;
    T             v[3] = {px, py, pz};
    if constexpr (PER == 2) {
#pragma unroll
        for (int a = 0; a < 3; ++a) v[a] = (T)((unsigned long long)v[a] & ((1ull << C::bits) - 1ull));
    }
    if constexpr (C::is_float) {
        bool fin = true;
#pragma unroll
        for (int a = 0; a < 3; ++a) fin = fin && isfinite((double)v[a]);
        if (!__all_sync(FULL, !need || fin)) return false;
    }
    const unsigned nm  = __ballot_sync(FULL, need);
    const int      ref = __ffs(nm) - 1;
    double         spread = 0.0; // largest axis extent, in coordinate units
#pragma unroll
    for (int a = 0; a < 3; ++a) {
        if constexpr (PER == 2) {
            constexpr int sh = 64 - C::bits;
            const T       r  = __shfl_sync(FULL, v[a], ref);
            long long     o  = (long long)(((unsigned long long)v[a] - (unsigned long long)r) << sh) >> sh;
            long long     lo = need ? o : LLONG_MAX, hi = need ? o : LLONG_MIN;
#pragma unroll
            for (int m = 16; m > 0; m >>= 1) {
                lo = min(lo, __shfl_xor_sync(FULL, lo, m));
                hi = max(hi, __shfl_xor_sync(FULL, hi, m));
            }
            g.g0[a]   = (T)(((unsigned long long)r + (unsigned long long)lo) & ((1ull << C::bits) - 1ull));
            g.span[a] = (unsigned long long)(hi - lo);
            g.g1[a]   = g.g0[a];
            spread    = fmax(spread, (double)g.span[a]);
        } else {
            const T r  = __shfl_sync(FULL, v[a], ref);
            T       lo = need ? v[a] : r, hi = lo;
#pragma unroll
            for (int m = 16; m > 0; m >>= 1) {
                const T u = __shfl_xor_sync(FULL, lo, m), w = __shfl_xor_sync(FULL, hi, m);
                lo        = u < lo ? u : lo;
                hi        = w > hi ? w : hi;
            }
            g.g0[a]   = lo;
            g.g1[a]   = hi;
            g.span[a] = C::is_float ? 0ull : (unsigned long long)(T)(hi - lo);
            spread    = fmax(spread, (double)hi - (double)lo);
        }
    }
    // the lanes' radii
    D R_lo = need ? RM2 : dist_heap_max<D>(), R_hi = need ? RM2 : D(0);
    D r_lo = need ? rm2 : dist_heap_max<D>(), r_hi = need ? rm2 : D(0);
#pragma unroll
    for (int m = 16; m > 0; m >>= 1) {
        const D a = __shfl_xor_sync(FULL, R_lo, m), b = __shfl_xor_sync(FULL, R_hi, m);
        const D c = __shfl_xor_sync(FULL, r_lo, m), d = __shfl_xor_sync(FULL, r_hi, m);
        R_lo = a < R_lo ? a : R_lo;
        R_hi = b > R_hi ? b : R_hi;
        r_lo = c < r_lo ? c : r_lo;
        r_hi = d > r_hi ? d : r_hi;
    }
    // worth it only when the group is small against the radius (its fuzzy shell thin), and the
    // leaf filter's float offsets stay accurate: every staged leaf lies within
    // lam = spread + (sqrt(R_hi) + 2) 2^shift of the group's corner on each axis
    const double unit = C::is_float ? 1.0 : (double)(1ull << C::dist_shift);
    const double rad  = sqrt((double)R_lo) * unit, Rad = (sqrt((double)R_hi) + 2.0) * unit;
    const double lam  = spread + Rad * (1.0 + 0x1p-20);
    bool         ok   = (FORCE || spread * (double)FT_RANGE_SPREAD <= rad) && lam > 0.0;
    // (floating point: squared offsets stay normal floats)
    if constexpr (C::is_float) ok = ok && lam < 0x1p60 && lam > 0x1p-60;
    else ok = ok && lam < 0x1p40;
    if (!ok) return false; // warp-uniform
    // Leaf filter.  In shifted units u (offsets / 2^shift for integers, plain offsets for
    // floating point) a lane's float estimate of a gap is y = |e - q|, within eps of the exact
    // gap (conversions and the subtraction: at most 2^-22 lam, taken as 2^-20 lam).  Integer
    // terms floor the shifted gap, t in (y - eps - 1, y + eps], so with Y = sum y^2 and
    // sum y <= sqrt(3 Y) the exact distance lies in [Y - c_lo sqrt(Y), Y + c_hi sqrt(Y) + 3 eps^2],
    // c_lo = 2 sqrt(3) (1 + eps), c_hi = 2 sqrt(3) eps; floating-point terms have no floor
    // (c_lo = c_hi) and the reference's rounded sum lies within 1 +- 2^-20 of the real one.
    // Each bound is monotone in Y, so four thresholds on Y decide a leaf: beyond r_max, inside
    // r_max, at least r_min, below r_min.  The leaf's Y is computed in float (relative error
    // under 2^-22, covered by a factor 1 +- 2^-21 on the thresholds) from offsets in units of
    // 2^shift: 3 subtractions and 3 multiply-adds a leaf, the exact distance only in the thin
    // band around the lane's spheres.
    const double eps  = lam * 0x1p-20 / unit;
    const double c_lo = 3.4641016151377546 * ((C::is_float ? 0.0 : 1.0) + eps) * (1.0 + 0x1p-40);
    const double c_hi = 3.4641016151377546 * eps * (1.0 + 0x1p-40);
    const double rho  = C::is_float ? 0x1p-20 : 0.0;
    const double u2   = unit * unit; // shifted units^2 -> offset units^2
    // smallest Y whose lower bound exceeds (or reaches) X, and largest Y whose upper bound
    // stays at or below X (-1: none)
    auto y_lower = [&](double X) {
        const double r = (c_lo + sqrt(c_lo * c_lo + 4.0 * X)) * 0.5;
        return r * r;
    };
    auto y_upper = [&](double X) {
        const double a = X - 3.0 * eps * eps;
        if (a < 0.0) return -1.0;
        const double r = (-c_hi + sqrt(c_hi * c_hi + 4.0 * a)) * 0.5;
        return r * r;
    };
    const double Rd = (double)RM2, rd = (double)rm2;
    // out if Y > t_out; in r_max if Y <= t_in; at least r_min if Y >= t_ge; below r_min if Y < t_lt
    const float t_out = __double2float_ru(y_lower(Rd / (1.0 - rho)) * u2 * (1.0 + 0x1p-21));
    const float t_in  = __double2float_rd(fmax(y_upper(Rd / (1.0 + rho)), -1.0) * u2 * (1.0 - 0x1p-21));
    const float t_ge  = rd <= 0.0 ? 0.0f : __double2float_ru(y_lower(rd / (1.0 - rho)) * u2 * (1.0 + 0x1p-21));
    const float t_lt  = rd <= 0.0 ? -1.0f : __double2float_rd(fmax(y_upper(rd / (1.0 + rho)), -1.0) * u2 * (1.0 - 0x1p-21));
    const float qf[3] = {group_off<T, PER>(v[0], g, 0), group_off<T, PER>(v[1], g, 1), group_off<T, PER>(v[2], g, 2)};

    int       mine = 0;    // this lane's count from staged leaves
    long long part = 0;    // leaves in nodes inside every lane's shell, found by this lane
    int       top = 0, cc = 0;
    bool      overflow = false;
    {
        const T rb[6] = {t.min_x[0], t.max_x[0], t.min_y[0], t.max_y[0], t.min_z[0], t.max_z[0]};
        D       rn, rf;
        group_near_far<T, PER>(g, rb, rn, rf);
        if (rn <= R_hi) {
            if (rn >= r_hi && rf <= R_lo) part = lane == 0 ? n : 0;
            else if (!(rf < r_lo)) top = 1;
        }
    }
    if (lane == 0) stk[0] = 0;
    __syncwarp();
    // each lane tests every staged leaf: the float filter, then the exact distance where the
    // filter cannot decide
    auto flush = [&]() {
        for (int j = 0; j < cc; ++j) {
            const float4 e = stage[j];
            if (!need) continue;
            const float dx = e.x - qf[0], dy = e.y - qf[1], dz = e.z - qf[2];
            const float Y  = fmaf(dz, dz, fmaf(dy, dy, dx * dx));
            if (Y > t_out || Y < t_lt) continue; // surely outside the shell
            if (Y <= t_in && Y >= t_ge) {        // surely inside
                ++mine;
                continue;
            }
            const int s = __float_as_int(e.w);
            const T   x = t.min_x[s], y = t.min_y[s], z = t.min_z[s];
            const D   d = Metric<T>::template dist<(PER != 0), (PER == 2)>(px, py, pz, x, x, y, y, z, z);
            mine += (d >= rm2 && d <= RM2) ? 1 : 0;
        }
        cc = 0;
        __syncwarp();
    };
    long long budget = 2ll * n + 64;
    while (top > 0) {
        const int m = min(min(top, 32), (kRangeGStack - top) / 3);
        if (m <= 0 || (budget -= m) < 0) {
            overflow = true;
            break;
        }
        const int base = top - m;
        const int node = lane < m ? stk[base + lane] : -1;
        top            = base;
        __syncwarp();
        T        bx[4][6];
        int      ch[4] = {-1, -1, -1, -1};
        unsigned kl = 0, ki = 0;
        if (node >= 0) {
            load_wide(t.wide, node, bx, ch);
#pragma unroll
            for (int i = 0; i < 4; ++i) {
                if (ch[i] < 0) continue;
                D dn, dfar;
                group_near_far<T, PER>(g, bx[i], dn, dfar);
                if (!(dn <= R_hi) || dfar < r_lo) continue; // outside every ball, or inside every r_min
                const bool leaf = ch[i] >= n - 1;
                if (dn >= r_hi && dfar <= R_lo) part += leaf ? 1 : t.leaves[ch[i]]; // inside every shell
                else if (leaf) kl |= 1u << i;
                else ki |= 1u << i;
            }
        }
        const int nl = __popc(kl), ni = __popc(ki);
        int       incl = nl | (ni << 16);
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const int u = __shfl_up_sync(FULL, incl, o);
            if (lane >= o) incl += u;
        }
        const int tot = __shfl_sync(FULL, incl, 31);
        if (cc + (tot & 0xffff) > kRangeStage) flush();
        int pl = cc + (incl & 0xffff) - nl, pi = top + (incl >> 16) - ni;
#pragma unroll
        for (int i = 0; i < 4; ++i) {
            if ((kl >> i) & 1u)
                stage[pl++] = make_float4(group_off<T, PER>(bx[i][0], g, 0), group_off<T, PER>(bx[i][2], g, 1),
                                          group_off<T, PER>(bx[i][4], g, 2), __int_as_float(ch[i]));
            if ((ki >> i) & 1u) stk[pi++] = ch[i];
        }
        cc += tot & 0xffff;
        top += tot >> 16;
        __syncwarp();
    }
    if (overflow) return false; // warp-uniform (every lane ran the same steps)
    flush();
#pragma unroll
    for (int m = 16; m > 0; m >>= 1) part += __shfl_xor_sync(FULL, part, m);
    count = (int)min(part + (long long)mine, (long long)INT_MAX);
    return true;
}

// range_query on trees of height <= 62 with a monotone box distance (default): phase 1 writes
// each row in the reference's order with the 4-wide walk and stops once the row is full;
// phase 2 counts the full rows' shells with range_count_group (per lane when the group's
// bounds cannot help).  Counts, rows and their order equal range_wide_kernel's.
template <class T, int PER, bool FORCE = false>
__global__ void __launch_bounds__(32 * kRangeWarps, FT_RANGE_MINB)
    range_split_kernel(TreeDev<T> t, const T *__restrict__ qx, const T *__restrict__ qy, const T *__restrict__ qz,
                       const T *__restrict__ rmin, const T *__restrict__ rmax, int nq, int32_t *__restrict__ results,
                       int32_t *__restrict__ counts, int max_per, int ret_orig, const uint32_t *__restrict__ order,
                       uint32_t *status) {
    using D = typename Coord<T>::dist_t;
    __shared__ int32_t s_stk[kRangeWarps][kRangeGStack];
    __shared__ float4  s_stage[kRangeWarps][kRangeStage];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int base = (blockIdx.x * kRangeWarps + warp) * 32;
    if (base >= nq) return; // warp-uniform
    const int  i      = base + lane;
    const bool active = i < nq;
    const int  q      = active ? (order ? (int)order[i] : i) : (order ? (int)order[base] : base);
    D          rm2 = D(0), RM2 = D(0);
    range_radii<T>(rmin, rmax, q, rm2, RM2);
    const T      px = qx[q], py = qy[q], pz = qz[q];
    const size_t off = (size_t)q * (size_t)max_per;
    bool         filled = false;
    int          cnt    = 0;
    if (active)
        cnt = range_one_wide<T, PER, true>(t, px, py, pz, rm2, RM2, results, off, max_per, ret_orig, status, &filled);
    const bool need = active && filled;
    if (__any_sync(0xffffffffu, need)) {
        int total = 0;
        if (range_count_group<T, PER, FORCE>(t, need, px, py, pz, rm2, RM2, s_stk[warp], s_stage[warp], total)) {
            if (need) cnt = total;
        } else if (need) {
            cnt = range_one_wide<T, PER>(t, px, py, pz, rm2, RM2, results, off, 0, ret_orig, status);
        }
    }
    if (active) counts[q] = cnt;
}

template <class T, int PER>
__global__ void __launch_bounds__(128)
    range_short_kernel(TreeDev<T> t, const T *__restrict__ qx, const T *__restrict__ qy, const T *__restrict__ qz,
                       const T *__restrict__ rmin, const T *__restrict__ rmax, int nq, int32_t *__restrict__ results,
                       int32_t *__restrict__ counts, int max_per, int ret_orig, const uint32_t *__restrict__ order,
                       uint32_t *status) {
    using D     = typename Coord<T>::dist_t;
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= nq) return;
    const int q = order ? (int)order[i] : i;
    D         rm2, RM2;
    range_radii<T>(rmin, rmax, q, rm2, RM2);
    counts[q] = range_one<T, PER>(t, qx[q], qy[q], qz[q], rm2, RM2, results, (size_t)q * (size_t)max_per, max_per,
                                  ret_orig, status);
}

// range_query on trees of height <= 62, a warp's 32 queries (neighbours in SFC order, so their
// balls overlap) walking the tree together: one depth-first, left-first walk over the union
// of the nodes the lanes need, each stack entry carrying the mask of the lanes that need it.
// Every lane takes exactly the decisions range_short_kernel takes for its query (push a child
// within r_max; once its row is full, count a leaf child or a child inside the shell from the
// record instead of walking it), and meets its nodes in the same left-first order, so its
// row and count are the same; the node type and the record are the warp's, so the lanes
// diverge far less than in one walk per lane.
template <class T, int PER>
__global__ void __launch_bounds__(128)
    range_group_kernel(TreeDev<T> t, const T *__restrict__ qx, const T *__restrict__ qy, const T *__restrict__ qz,
                       const T *__restrict__ rmin, const T *__restrict__ rmax, int nq, int32_t *__restrict__ results,
                       int32_t *__restrict__ counts, int max_per, int ret_orig, const uint32_t *__restrict__ order,
                       uint32_t *status) {
    using C                = Coord<T>;
    using D                = typename C::dist_t;
    constexpr int  kWarps  = 4;
    const unsigned FULL    = 0xffffffffu;
    __shared__ int32_t  s_node[kWarps][kStack];
    __shared__ uint32_t s_mask[kWarps][kStack];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int base = (blockIdx.x * kWarps + warp) * 32;
    if (base >= nq) return; // warp-uniform
    const int  i      = base + lane;
    const bool active = i < nq;
    const int  q      = active ? (order ? (int)order[i] : i) : 0;
    const int  n      = t.n;
    D          rm2 = D(0), RM2 = D(0);
    if (active) range_radii<T>(rmin, rmax, q, rm2, RM2);
    const T      px = qx[q], py = qy[q], pz = qz[q];
    // Walk together only when the lanes' balls overlap: the warp's query points lie within a
    // box whose diagonal is no longer than the smallest r_max; otherwise (sparse regions, or
    // points on both sides of a periodic edge) each lane takes its own walk.
    {
        const T  p[3] = {px, py, pz};
        D        span = D(0);
#pragma unroll
        for (int a = 0; a < 3; ++a) {
            T lo = p[a], hi = p[a];
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) {
                const T u = __shfl_xor_sync(FULL, lo, o), w = __shfl_xor_sync(FULL, hi, o);
                lo        = u < lo ? u : lo;
                hi        = w > hi ? w : hi;
            }
            if constexpr (C::is_float) {
                const double e = (double)hi - (double)lo;
                span += e * e;
            } else {
                const unsigned long long e = (unsigned long long)(hi - lo) >> C::dist_shift;
                span += e < (1ull << 31) ? e * e : (1ull << 62);
            }
        }
        D rmin2 = active ? RM2 : dist_heap_max<D>();
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            const D u = __shfl_xor_sync(FULL, rmin2, o);
            rmin2     = u < rmin2 ? u : rmin2;
        }
        if (!(span <= rmin2)) { // warp-uniform
            if (active)
                counts[q] = range_one<T, PER>(t, px, py, pz, rm2, RM2, results, (size_t)q * (size_t)max_per, max_per,
                                              ret_orig, status);
            return;
        }
    }
    const size_t off   = (size_t)q * (size_t)max_per;
    int          count = 0;
    D            sd[kStack]; // this lane's distance of each stacked node
    int          sp = 0;
    const D      d0 = node_dist_soa<T, PER>(t, 0, px, py, pz);
    const unsigned m0 = __ballot_sync(FULL, active && d0 <= RM2);
    if (m0) {
        if (lane == 0) {
            s_node[warp][0] = 0;
            s_mask[warp][0] = m0;
        }
        sd[0] = d0;
        sp    = 1;
    }
    __syncwarp();
    long long budget = 2ll * n + 64;
    while (sp > 0) {
        if (--budget < 0) {
            if (lane == 0) atomicOr(status, STATUS_TRAVERSAL_LIMIT);
            break;
        }
        --sp;
        const int      node = s_node[warp][sp];
        const uint32_t mask = s_mask[warp][sp];
        const bool     in   = (mask >> lane) & 1u;
        const D        d2   = sd[sp];
        __syncwarp(); // every lane has read the entry before pushes reuse the slot
        if (node >= n - 1) { // leaf (the n == 1 root included)
            if (in && d2 >= rm2) {
                if (count < max_per) results[off + count] = ret_orig ? t.orig_idx[node] : node - (n - 1);
                ++count;
            }
            continue;
        }
        T        lb[6], rb[6];
        int      l, r;
        uint32_t il, ir;
        load_rec_info(t.recs, node, lb, rb, l, r, il, ir);
        bool need_l = false, need_r = false;
        D    dl = D(0), dr = D(0);
        if (in) {
            dl              = box_dist<T, PER>(px, py, pz, lb);
            dr              = box_dist<T, PER>(px, py, pz, rb);
            const bool full = count >= max_per;
#pragma unroll
            for (int side = 1; side >= 0; --side) {
                const int      c  = side ? r : l;
                const D        dc = side ? dr : dl;
                const uint32_t ic = side ? ir : il;
                if (!(dc <= RM2)) continue;
                if (full) {
                    if (c >= n - 1) { // a leaf: counted now
                        if (dc >= rm2) ++count;
                        continue;
                    }
                    if (dc >= rm2 && info_leaves(ic) < kInfoCountMax) {
                        D far;
                        if (far_dist_box<T, PER>(px, py, pz, side ? rb : lb, far) && far <= RM2) {
                            count += (int)info_leaves(ic); // every leaf below lies in the shell
                            continue;
                        }
                    }
                }
                if (side) need_r = true;
                else need_l = true;
            }
        }
        const unsigned mr = __ballot_sync(FULL, need_r), ml = __ballot_sync(FULL, need_l);
        const int      add = (mr != 0u) + (ml != 0u);
        if (sp + add > kStack) {
            if (lane == 0) atomicOr(status, STATUS_TRAVERSAL_LIMIT);
            break;
        }
        // right first on the stack, so the left subtree is walked (and written) first
        if (mr) {
            if (lane == 0) {
                s_node[warp][sp] = r;
                s_mask[warp][sp] = mr;
            }
            sd[sp] = dr;
            ++sp;
        }
        if (ml) {
            if (lane == 0) {
                s_node[warp][sp] = l;
                s_mask[warp][sp] = ml;
            }
            sd[sp] = dl;
            ++sp;
        }
        __syncwarp();
    }
    if (active) counts[q] = count;
}

template <class T, int PER>
__global__ void __launch_bounds__(128) range_kernel(TreeDev<T> t, const T *__restrict__ qx, const T *__restrict__ qy,
                                                    const T *__restrict__ qz, const T *__restrict__ rmin,
                                                    const T *__restrict__ rmax, int nq, int32_t *__restrict__ results,
                                                    int32_t *__restrict__ counts, int max_per, int ret_orig,
                                                    const uint32_t *__restrict__ order, uint32_t *status) {
    using C = Coord<T>;
    using D = typename C::dist_t;
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= nq) return;
    const int q = order ? (int)order[i] : i; // queries taken in SFC order when given
    const int n = t.n;
    D         rm2, RM2;
    if constexpr (C::is_float) {
        double a = (double)rmin[q], b = (double)rmax[q];
        rm2      = __dmul_rn(a, a);
        RM2      = __dmul_rn(b, b);
    } else {
        unsigned long long a = (unsigned long long)rmin[q] >> C::dist_shift;
        unsigned long long b = (unsigned long long)rmax[q] >> C::dist_shift;
        rm2                  = a * a;
        RM2                  = b * b;
    }
    const T px = qx[q], py = qy[q], pz = qz[q];
    int     sn[kStack];
    D       sd[kStack];
    int     sp = 1;
    sn[0]      = 0;
    sd[0]      = node_dist_soa<T, PER>(t, 0, px, py, pz);
    int          count = 0;
    const size_t off   = (size_t)q * (size_t)max_per;
    long long    budget = 2ll * n + 64;
    while (sp > 0) {
        if (--budget < 0) {
            atomicOr(status, STATUS_TRAVERSAL_LIMIT);
            break;
        }
        --sp;
        const int node = sn[sp];
        const D   d2   = sd[sp];
        if (!(d2 <= RM2)) continue;
        if (node >= n - 1) {
            if (d2 >= rm2) {
                if (count < max_per) results[off + count] = ret_orig ? t.orig_idx[node] : node - (n - 1);
                ++count;
            }
        } else {
            // Once the row is full only the count changes.  A subtree that lies entirely in
            // the shell is then counted at once: every leaf under it passes both tests, and
            // the traversal would visit all of them -- popped at stack size sp, a subtree of
            // height h reaches stack size sp + h - 1 < 62 on its deepest path, so the stack
            // guard below drops none of it.
            if (count >= max_per && d2 >= rm2 && sp + (int)t.height[node] <= kStack - 2) {
                D far;
                if (far_dist<T, PER>(px, py, pz, t, node, far) && far <= RM2) {
                    count += t.leaves[node];
                    continue;
                }
            }
            if (sp < kStack - 2) {
                T   lb[6], rb[6];
                int l, r;
                load_rec(t.recs, node, lb, rb, l, r);
                sn[sp]     = r;
                sd[sp]     = box_dist<T, PER>(px, py, pz, rb);
                sn[sp + 1] = l;
                sd[sp + 1] = box_dist<T, PER>(px, py, pz, lb);
                sp += 2;
            }
        }
    }
    counts[q] = count;
}

// =========================================================================================
// Host side
// =========================================================================================
// Heap capacity tiers and the threads per block that keep the heap at <= 96 KB.
template <class T, int CAP, int QT, bool SELF, int PER>
static void launch_exact_t(const TreeDev<T> &tv, const BatchDev &bt, const void *qx, const void *qy, const void *qz,
                           const int32_t *leaf_ids, int num, int k, bool excl, bool ro, uint64_t *idx, void *dist,
                           uint32_t *status, cudaStream_t st) {
    using D     = typename Coord<T>::dist_t;
    size_t smem = (size_t)CAP * QT * (sizeof(D) + 4);
    auto   fn   = exact_knn_kernel<T, CAP, QT, SELF, PER>;
    FT_CUDA(cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    int blocks = (num + QT - 1) / QT;
    fn<<<blocks, QT, smem, st>>>(tv, bt, (const T *)qx, (const T *)qy, (const T *)qz, leaf_ids, num, k,
                                 excl ? 1 : 0, ro ? 1 : 0, (unsigned long long *)idx, (D *)dist, status);
    FT_CUDA(cudaGetLastError());
}

template <class T, bool SELF, int PER>
static void launch_exact_cap(const TreeDev<T> &tv, const BatchDev &bt, const void *qx, const void *qy,
                             const void *qz, const int32_t *leaf_ids, int num, int k, bool excl, bool ro,
                             uint64_t *idx, void *dist, uint32_t *status, cudaStream_t st) {
#define FT_LAUNCH(CAP, QT) \
    launch_exact_t<T, CAP, QT, SELF, PER>(tv, bt, qx, qy, qz, leaf_ids, num, k, excl, ro, idx, dist, status, st)
    if (k <= 32) FT_LAUNCH(32, 128);
    else if (k <= 64) FT_LAUNCH(64, 128);
    else if (k <= 128) FT_LAUNCH(128, 64);
    else if (k <= 256) FT_LAUNCH(256, 32);
    else FT_LAUNCH(512, 32);
#undef FT_LAUNCH
}

template <class T, bool SELF>
static void launch_exact(const ft_options &o, const ft_tree &tr, const void *qx, const void *qy, const void *qz,
                         const int32_t *leaf_ids, int num, int k, bool excl, uint64_t *idx, void *dist,
                         uint32_t *status, cudaStream_t st, const BatchDev &bt = {}) {
    TreeDev<T> tv = tree_view<T>(tr);
    bool       ro = o.return_orig_indices != 0;
    met_dispatch<T>(metric_mode<T>(o, tr), [&](auto M) {
        launch_exact_cap<T, SELF, decltype(M)::value>(tv, bt, qx, qy, qz, leaf_ids, num, k, excl, ro, idx, dist,
                                                      status, st);
    });
}

static constexpr int kMaxExactK = 512;

void self_knn(Context &ctx, const ft_tree &tr, const int32_t *leaf_ids, size_t num, int k, bool excl, uint64_t *idx,
              void *dist, const ft_query_options &qo, cudaStream_t st, const void *bound) {
    int max_k = qo.max_k > 0 ? qo.max_k : (leaf_ids ? 256 : 32);
    if (k > max_k)
        fail(FT_ERR_INVALID_ARGUMENT,
             "k exceeds _MAX_K_ template parameter. Instantiate self_knn_query with larger _MAX_K_.");
    if (tr.num_leaves == 0 || num == 0 || k <= 0) return;
    if (k > kMaxExactK) fail(FT_ERR_RUNTIME, "self_knn_query: k too large for shared memory.");
    if (num > (size_t)INT32_MAX) fail(FT_ERR_INVALID_ARGUMENT, "too many queries");
    ctx.stats.queries  = (int64_t)num;
    ctx.stats.replayed = 0;
    ctx.last_fast      = false;
    ctx.last_rows      = false;
    if ((qo.method != FT_METHOD_PLAIN || bound) &&
        fast_self_knn(ctx, tr, leaf_ids, num, k, excl, idx, dist, bound, qo.reserved[0], qo.reserved[1], st)) {
        ctx.last_fast = true;
        ctx.last_rows = true;
        return;
    }
    switch (ctx.opts.coord_type) {
    case F32: launch_exact<float, true>(ctx.opts, tr, nullptr, nullptr, nullptr, leaf_ids, (int)num, k, excl, idx, dist, ctx.status, st); break;
    case F64: launch_exact<double, true>(ctx.opts, tr, nullptr, nullptr, nullptr, leaf_ids, (int)num, k, excl, idx, dist, ctx.status, st); break;
    case U32: launch_exact<uint32_t, true>(ctx.opts, tr, nullptr, nullptr, nullptr, leaf_ids, (int)num, k, excl, idx, dist, ctx.status, st); break;
    case U64: launch_exact<unsigned long long, true>(ctx.opts, tr, nullptr, nullptr, nullptr, leaf_ids, (int)num, k, excl, idx, dist, ctx.status, st); break;
    }
}

__global__ void iota_i32_kernel(int32_t *a, int n) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) a[i] = i;
}

// Self-kNN whose outputs are host memory.  The leaves are walked in chunks into two device
// buffers in turn; each chunk's rows go to the host on a second stream while the next chunk
// is walked, so the copy-out (16 k bytes per query) overlaps the walk.  Pinned host memory
// gives full overlap; with pageable memory the host waits for each chunk's copy while the
// next chunk runs.  The caller's stream is complete when the last rows are in host memory.
// Query statistics describe the last chunk.
void self_knn_to_host(Context &ctx, const ft_tree &tr, const int32_t *leaf_ids, size_t num, int k, bool excl,
                      uint64_t *h_idx, void *h_dist, const ft_query_options &qo, cudaStream_t st) {
    const int max_k = qo.max_k > 0 ? qo.max_k : (leaf_ids ? 256 : 32);
    if (k > max_k)
        fail(FT_ERR_INVALID_ARGUMENT,
             "k exceeds _MAX_K_ template parameter. Instantiate self_knn_query with larger _MAX_K_.");
    if (tr.num_leaves == 0 || num == 0 || k <= 0) return;
    if (k > kMaxExactK) fail(FT_ERR_RUNTIME, "self_knn_query: k too large for shared memory.");
    if (num > (size_t)INT32_MAX) fail(FT_ERR_INVALID_ARGUMENT, "too many queries");
    ft_query_options q = qo;
    q.max_k            = max_k;
    const size_t chunk = std::max<size_t>(size_t(1) << 18, (num + 15) / 16);
    const size_t rows  = std::min(chunk, num);
    auto ensure = [&](void *&p, size_t bytes) {
        if (p) return;
        cudaError_t e = cudaMalloc(&p, bytes);
        if (e != cudaSuccess) {
            cudaGetLastError();
            p = nullptr;
            fail(FT_ERR_OUT_OF_MEMORY, "cudaMalloc of the host-output staging buffers failed");
        }
    };
    if (rows * (size_t)k > ctx.stage_cap) {
        for (int b = 0; b < 2; ++b) {
            if (ctx.stage_idx[b]) cudaFree(ctx.stage_idx[b]);
            if (ctx.stage_dist[b]) cudaFree(ctx.stage_dist[b]);
            ctx.stage_idx[b] = ctx.stage_dist[b] = nullptr;
        }
        ctx.stage_cap = 0;
        for (int b = 0; b < 2; ++b) {
            ensure(ctx.stage_idx[b], rows * (size_t)k * 8);
            ensure(ctx.stage_dist[b], rows * (size_t)k * 8);
        }
        ctx.stage_cap = rows * (size_t)k;
    }
    if (!ctx.copy_stream) {
        FT_CUDA(cudaStreamCreateWithFlags(&ctx.copy_stream, cudaStreamNonBlocking));
        for (int b = 0; b < 2; ++b) {
            FT_CUDA(cudaEventCreateWithFlags(&ctx.ev_walked[b], cudaEventDisableTiming));
            FT_CUDA(cudaEventCreateWithFlags(&ctx.ev_copied[b], cudaEventDisableTiming));
        }
    }
    const int32_t *ids = leaf_ids;
    if (!ids) { // the full query: leaf ranks 0 .. num-1
        if (num > ctx.iota_cap) {
            if (ctx.iota) cudaFree(ctx.iota);
            ctx.iota     = nullptr;
            ctx.iota_cap = 0;
            void *p      = nullptr;
            ensure(p, num * sizeof(int32_t));
            ctx.iota     = (int32_t *)p;
            ctx.iota_cap = num;
            iota_i32_kernel<<<(int)std::min<size_t>((num + 255) / 256, 148 * 16), 256, 0, st>>>(ctx.iota, (int)num);
            FT_CUDA(cudaGetLastError());
        }
        ids = ctx.iota;
    }
    auto copy_out = [&](size_t c0, size_t cnt, int b) {
        FT_CUDA(cudaStreamWaitEvent(ctx.copy_stream, ctx.ev_walked[b], 0));
        FT_CUDA(cudaMemcpyAsync(h_idx + c0 * k, ctx.stage_idx[b], cnt * k * 8, cudaMemcpyDeviceToHost,
                                ctx.copy_stream));
        FT_CUDA(cudaMemcpyAsync((char *)h_dist + c0 * k * 8, ctx.stage_dist[b], cnt * k * 8, cudaMemcpyDeviceToHost,
                                ctx.copy_stream));
        FT_CUDA(cudaEventRecord(ctx.ev_copied[b], ctx.copy_stream));
    };
    // the first chunk is small: its walk is the only one no copy overlaps
    const size_t first = std::min(rows, size_t(1) << 18);
    size_t       prev0 = 0, prevn = 0;
    int          c     = 0;
    for (size_t c0 = 0, cnt = 0; c0 < num; c0 += cnt) {
        cnt          = std::min(c == 0 ? first : rows, num - c0);
        const int    b   = c & 1;
        if (c >= 2) FT_CUDA(cudaStreamWaitEvent(st, ctx.ev_copied[b], 0)); // buffer b's last rows are out
        self_knn(ctx, tr, ids + c0, cnt, k, excl, (uint64_t *)ctx.stage_idx[b], ctx.stage_dist[b], q, st);
        FT_CUDA(cudaEventRecord(ctx.ev_walked[b], st));
        if (c >= 1) copy_out(prev0, prevn, b ^ 1); // the previous chunk, while this one is walked
        prev0 = c0;
        prevn = cnt;
        ++c;
    }
    copy_out(prev0, prevn, (c - 1) & 1);
    FT_CUDA(cudaStreamWaitEvent(st, ctx.ev_copied[(c - 1) & 1], 0));
    ctx.last_rows = false; // the replay list holds the last chunk's rows, numbered within it
}

template <class T, int CAP, int QT, int PER>
static void replay_t(const TreeDev<T> &tv, const BatchDev &bt, const int32_t *ranks, const int32_t *rows,
                     uint32_t *cnt, int k, bool excl, bool ro, uint64_t *idx, void *dist, uint32_t *status,
                     int num_sms, cudaStream_t st) {
    using D     = typename Coord<T>::dist_t;
    size_t smem = (size_t)CAP * QT * (sizeof(D) + 4);
    auto   fn   = exact_replay_kernel<T, CAP, QT, PER>;
    FT_CUDA(cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    fn<<<num_sms * 4, QT, smem, st>>>(tv, bt, ranks, rows, cnt, k, excl ? 1 : 0, ro ? 1 : 0,
                                       (unsigned long long *)idx, (D *)dist, status);
    FT_CUDA(cudaGetLastError());
}

template <class T>
static void replay_typed(Context &ctx, const ft_tree &tr, const BatchDev &bt, const int32_t *ranks,
                         const int32_t *rows, uint32_t *cnt, int k, bool excl, uint64_t *idx, void *dist,
                         cudaStream_t st) {
    TreeDev<T> tv  = tree_view<T>(tr);
    bool       ro  = ctx.opts.return_orig_indices != 0;
    int        met = metric_mode<T>(ctx.opts, tr);
    int        sms = ctx.num_sms;
#define FT_RP(CAP, QT)                                                                                             \
    met_dispatch<T>(met, [&](auto M) {                                                                             \
        replay_t<T, CAP, QT, decltype(M)::value>(tv, bt, ranks, rows, cnt, k, excl, ro, idx, dist, ctx.status, sms, \
                                                 st);                                                              \
    })
    if (k <= 32) FT_RP(32, 128);
    else if (k <= 64) FT_RP(64, 128);
    else if (k <= 128) FT_RP(128, 64);
    else if (k <= 256) FT_RP(256, 32);
    else FT_RP(512, 32);
#undef FT_RP
}

void replay_exact(Context &ctx, const ft_tree &tr, const int32_t *ranks, const int32_t *rows, uint32_t *cnt, int k,
                  bool excl, uint64_t *idx, void *dist, cudaStream_t st, const BatchDev &bt) {
    switch (ctx.opts.coord_type) {
    case F32: replay_typed<float>(ctx, tr, bt, ranks, rows, cnt, k, excl, idx, dist, st); break;
    case F64: replay_typed<double>(ctx, tr, bt, ranks, rows, cnt, k, excl, idx, dist, st); break;
    case U32: replay_typed<uint32_t>(ctx, tr, bt, ranks, rows, cnt, k, excl, idx, dist, st); break;
    case U64: replay_typed<unsigned long long>(ctx, tr, bt, ranks, rows, cnt, k, excl, idx, dist, st); break;
    }
}

void batch_self_knn_exact(Context &ctx, const ft_tree &all, const BatchDev &bt, size_t num, int k, bool excl,
                          uint64_t *idx, void *dist, cudaStream_t st) {
    if (num == 0 || k <= 0) return;
    if (k > kMaxExactK) fail(FT_ERR_RUNTIME, "self_knn_query: k too large for shared memory.");
    const int n = (int)num;
    switch (ctx.opts.coord_type) {
    case F32: launch_exact<float, true>(ctx.opts, all, nullptr, nullptr, nullptr, nullptr, n, k, excl, idx, dist, ctx.status, st, bt); break;
    case F64: launch_exact<double, true>(ctx.opts, all, nullptr, nullptr, nullptr, nullptr, n, k, excl, idx, dist, ctx.status, st, bt); break;
    case U32: launch_exact<uint32_t, true>(ctx.opts, all, nullptr, nullptr, nullptr, nullptr, n, k, excl, idx, dist, ctx.status, st, bt); break;
    case U64: launch_exact<unsigned long long, true>(ctx.opts, all, nullptr, nullptr, nullptr, nullptr, n, k, excl, idx, dist, ctx.status, st, bt); break;
    }
}

template <class T, int PER>
static void launch_merge(const TreeDev<T> &tv, const void *qx, const void *qy, const void *qz, int nq, int k, int cap,
                         bool ro, uint64_t *idx, void *dist, uint32_t *status, cudaStream_t st) {
    using D     = typename Coord<T>::dist_t;
    size_t smem = (size_t)kMergeWarps * (cap + 32) * (sizeof(D) + 4);
    auto   fn   = merge_knn_kernel<T, PER>;
    FT_CUDA(cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    int blocks = (nq + kMergeWarps - 1) / kMergeWarps;
    fn<<<blocks, 32 * kMergeWarps, smem, st>>>(tv, (const T *)qx, (const T *)qy, (const T *)qz, nq, k, cap,
                                               ro ? 1 : 0, (unsigned long long *)idx, (D *)dist, status);
    FT_CUDA(cudaGetLastError());
}

template <class T>
static void knn_typed(const ft_options &o, const ft_tree &tr, const void *qx, const void *qy, const void *qz, int nq,
                      int k, int max_k, uint64_t *idx, void *dist, uint32_t *status, cudaStream_t st) {
    if (k <= 32 || max_k <= 32) {
        launch_exact<T, false>(o, tr, qx, qy, qz, nullptr, nq, k, false, idx, dist, status, st);
        return;
    }
    int cap = 1;
    while (cap < max_k) cap <<= 1;
    TreeDev<T> tv = tree_view<T>(tr);
    bool       ro = o.return_orig_indices != 0;
    met_dispatch<T>(metric_mode<T>(o, tr), [&](auto M) {
        launch_merge<T, decltype(M)::value>(tv, qx, qy, qz, nq, k, cap, ro, idx, dist, status, st);
    });
}

template <class T>
static void replay_external_typed(Context &ctx, const ft_tree &tr, const void *qx, const void *qy, const void *qz,
                                  const int32_t *rows, uint32_t *cnt, int k, int max_k, uint64_t *idx, void *dist,
                                  cudaStream_t st) {
    using D       = typename Coord<T>::dist_t;
    TreeDev<T> tv = tree_view<T>(tr);
    const bool ro = ctx.opts.return_orig_indices != 0;
    const int  sms = ctx.num_sms;
    met_dispatch<T>(metric_mode<T>(ctx.opts, tr), [&](auto M) {
        constexpr int PER = decltype(M)::value;
        if (k <= 32 || max_k <= 32) {
            auto   fn   = exact_replay_ext_kernel<T, 32, 128, PER>;
            size_t smem = (size_t)32 * 128 * (sizeof(D) + 4);
            FT_CUDA(cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
            fn<<<sms * 4, 128, smem, st>>>(tv, (const T *)qx, (const T *)qy, (const T *)qz, rows, cnt, k, ro ? 1 : 0,
                                          (unsigned long long *)idx, (D *)dist, ctx.status);
        } else {
            int cap = 1;
            while (cap < max_k) cap <<= 1;
            auto   fn   = merge_replay_kernel<T, PER>;
            size_t smem = (size_t)kMergeWarps * (cap + 32) * (sizeof(D) + 4);
            FT_CUDA(cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
            fn<<<sms * 8, 32 * kMergeWarps, smem, st>>>(tv, (const T *)qx, (const T *)qy, (const T *)qz, rows, cnt, k,
                                                       cap, ro ? 1 : 0, (unsigned long long *)idx, (D *)dist,
                                                       ctx.status);
        }
        FT_CUDA(cudaGetLastError());
    });
}

void replay_external(Context &ctx, const ft_tree &tr, const void *qx, const void *qy, const void *qz,
                     const int32_t *rows, uint32_t *cnt, int k, int max_k, uint64_t *idx, void *dist,
                     cudaStream_t st) {
    switch (ctx.opts.coord_type) {
    case F32: replay_external_typed<float>(ctx, tr, qx, qy, qz, rows, cnt, k, max_k, idx, dist, st); break;
    case F64: replay_external_typed<double>(ctx, tr, qx, qy, qz, rows, cnt, k, max_k, idx, dist, st); break;
    case U32: replay_external_typed<uint32_t>(ctx, tr, qx, qy, qz, rows, cnt, k, max_k, idx, dist, st); break;
    case U64: replay_external_typed<unsigned long long>(ctx, tr, qx, qy, qz, rows, cnt, k, max_k, idx, dist, st); break;
    }
}

void knn(Context &ctx, const ft_tree &tr, const void *qx, const void *qy, const void *qz, size_t nq, int k, int max_k,
         uint64_t *idx, void *dist, const ft_query_options &qo, cudaStream_t st, const void *bound) {
    if (max_k <= 0) max_k = 256;
    if (tr.num_leaves == 0 || nq == 0 || k <= 0) return;
    if (max_k > 32 && k > 32 && k > max_k)
        fail(FT_ERR_INVALID_ARGUMENT, "k exceeds _MAX_K_ template parameter. Instantiate knn_query with larger _MAX_K_.");
    if (max_k <= 32 && k > 32)
        fail(FT_ERR_INVALID_ARGUMENT, "k exceeds _MAX_K_ template parameter. Instantiate knn_query with larger _MAX_K_.");
    if (max_k > 4096) fail(FT_ERR_RUNTIME, "knn_query_large_k: k too large, local memory requirement exceeds device limit.");
    if (nq > (size_t)INT32_MAX) fail(FT_ERR_INVALID_ARGUMENT, "too many queries");
    ctx.stats.queries  = (int64_t)nq;
    ctx.stats.replayed = 0;
    ctx.last_fast      = false;
    ctx.last_rows      = false;
    if ((qo.method != FT_METHOD_PLAIN || bound) &&
        fast_knn(ctx, tr, qx, qy, qz, nq, k, max_k, idx, dist, qo.reserved[0], st, bound, qo.reserved[1])) {
        ctx.last_fast = true;
        ctx.last_rows = true;
        return;
    }
    switch (ctx.opts.coord_type) {
    case F32: knn_typed<float>(ctx.opts, tr, qx, qy, qz, (int)nq, k, max_k, idx, dist, ctx.status, st); break;
    case F64: knn_typed<double>(ctx.opts, tr, qx, qy, qz, (int)nq, k, max_k, idx, dist, ctx.status, st); break;
    case U32: knn_typed<uint32_t>(ctx.opts, tr, qx, qy, qz, (int)nq, k, max_k, idx, dist, ctx.status, st); break;
    case U64: knn_typed<unsigned long long>(ctx.opts, tr, qx, qy, qz, (int)nq, k, max_k, idx, dist, ctx.status, st); break;
    }
}

template <class T>
static void range_typed(const ft_options &o, const ft_tree &tr, const void *qx, const void *qy, const void *qz,
                        const void *rmin, const void *rmax, int nq, int32_t *results, int32_t *counts, int max_per,
                        const uint32_t *order, uint32_t *status, cudaStream_t st, int walk) {
    TreeDev<T> tv     = tree_view<T>(tr);
    bool       ro     = o.return_orig_indices != 0;
    // trees of height <= 62 never reach the reference's stack guard (range_short_kernel)
    const TreeImpl *impl  = (const TreeImpl *)tr.impl;
    const bool      short_walk = impl && impl->height_root >= 0 && impl->height_root <= 62;
    // the 4-wide walk skips the binary level between a node and its grandchildren, exact when
    // the box distance is monotone over nested boxes (the fast walks' condition)
    const bool      wide = impl && fast_walk_applies(o, *impl);
    met_dispatch<T>(metric_mode<T>(o, tr), [&](auto M) {
        auto fn = !short_walk ? range_kernel<T, decltype(M)::value>
                  : walk == 2 ? range_group_kernel<T, decltype(M)::value>
                  : (walk == 1 || !wide) ? range_short_kernel<T, decltype(M)::value>
                  : walk == 3 ? range_wide_kernel<T, decltype(M)::value>
                  : walk == 4 ? range_split_kernel<T, decltype(M)::value, true>
                              : range_split_kernel<T, decltype(M)::value>;
        // the split kernel's blocks have 32 * kRangeWarps threads, the others 128
        const bool split = short_walk && wide && walk != 1 && walk != 2 && walk != 3;
        const int  thr   = split ? 32 * kRangeWarps : 128;
        fn<<<(nq + thr - 1) / thr, thr, 0, st>>>(tv, (const T *)qx, (const T *)qy, (const T *)qz, (const T *)rmin,
                                                 (const T *)rmax, nq, results, counts, max_per, ro ? 1 : 0, order,
                                                 status);
    });
    FT_CUDA(cudaGetLastError());
}

void range(Context &ctx, const ft_tree &tr, const void *qx, const void *qy, const void *qz, const void *rmin,
           const void *rmax, size_t nq, int32_t *results, int32_t *counts, int max_per, cudaStream_t st) {
    if (tr.num_leaves == 0 || nq == 0) return;
    if (nq > (size_t)INT32_MAX) fail(FT_ERR_INVALID_ARGUMENT, "too many queries");
    // each query's output is independent of the others: take them in SFC order
    const uint32_t *order = sfc_query_order(ctx, tr, qx, qy, qz, nq, st);
    switch (ctx.opts.coord_type) {
    case F32: range_typed<float>(ctx.opts, tr, qx, qy, qz, rmin, rmax, (int)nq, results, counts, max_per, order, ctx.status, st, ctx.range_walk); break;
    case F64: range_typed<double>(ctx.opts, tr, qx, qy, qz, rmin, rmax, (int)nq, results, counts, max_per, order, ctx.status, st, ctx.range_walk); break;
    case U32: range_typed<uint32_t>(ctx.opts, tr, qx, qy, qz, rmin, rmax, (int)nq, results, counts, max_per, order, ctx.status, st, ctx.range_walk); break;
    case U64: range_typed<unsigned long long>(ctx.opts, tr, qx, qy, qz, rmin, rmax, (int)nq, results, counts, max_per, order, ctx.status, st, ctx.range_walk); break;
    }
}

} // namespace ft
