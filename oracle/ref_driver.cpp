// ref_driver.cpp -- C entry points around the reference's own headers (src/hlbvh.hpp and the
// headers it includes), compiled unmodified against the host SYCL shim in sycl_shim/.
//
// TEST INFRASTRUCTURE ONLY: the checker that pins the oracle restatement (ft_oracle.cpp)
// and, through it, the CUDA library.  One shared object per compile-time configuration of
// the reference (SFC type, coordinate type, PERIODIC_BC, RETURN_ORIG_INDICES); see ref.mk.
//
// Entry points mirror ft_oracle.cpp's (same Tree layout, keys as (hi, lo) uint64 pairs) so
// tests can compare the two on the same inputs.
#include "hlbvh.hpp"

#include <cstdint>
#include <cstring>
#include <vector>

// x86-64 fiber switch used by the shim's work-group runtime: saves the callee-saved
// registers on the current stack, swaps stack pointers, restores the other fiber's.
asm(R"(
    .text
    .globl ftshim_switch
    .type ftshim_switch, @function
ftshim_switch:
    pushq %rbp
    pushq %rbx
    pushq %r12
    pushq %r13
    pushq %r14
    pushq %r15
    movq %rsp, (%rdi)
    movq %rsi, %rsp
    popq %r15
    popq %r14
    popq %r13
    popq %r12
    popq %rbx
    popq %rbp
    ret
    .size ftshim_switch, .-ftshim_switch
)");

using namespace fasttree;

namespace {

struct RTree {
    void     *min_x, *max_x, *min_y, *max_y, *min_z, *max_z;
    int32_t  *left_child, *right_child, *parent;
    uint32_t *id;
    int8_t   *is_ghost;
    int32_t  *orig_idx;
    int64_t   num_leaves;
};

sycl::queue &Q() {
    static sycl::queue q;
    return q;
}

// Key -> (hi, lo) in the oracle's convention.
void split_key(const sfc_key &k, uint64_t &hi, uint64_t &lo) {
#if defined(SFC_TYPE_MORTON)
    hi = 0;
    lo = k;
#elif defined(POSITIONS_IN_64BIT)
    hi = k.is;
    lo = k.ls;
#else
    hi = 0;
    lo = (static_cast<uint64_t>(k.is) << 32) | static_cast<uint64_t>(k.ls);
#endif
}

sfc_key join_key(uint64_t hi, uint64_t lo) {
#if defined(SFC_TYPE_MORTON)
    (void)hi;
    return lo;
#elif defined(POSITIONS_IN_64BIT)
    sfc_key k;
    k.hs = 0;
    k.is = hi;
    k.ls = lo;
    return k;
#else
    (void)hi;
    sfc_key k;
    k.hs = 0;
    k.is = static_cast<uint32_t>(lo >> 32);
    k.ls = static_cast<uint32_t>(lo);
    return k;
#endif
}

// A TreeSoA whose arrays are the caller's (no ownership).
TreeSoA view(const RTree &t) {
    TreeSoA v(Q(), 0);
    v.min_x        = static_cast<coord_t *>(t.min_x);
    v.max_x        = static_cast<coord_t *>(t.max_x);
    v.min_y        = static_cast<coord_t *>(t.min_y);
    v.max_y        = static_cast<coord_t *>(t.max_y);
    v.min_z        = static_cast<coord_t *>(t.min_z);
    v.max_z        = static_cast<coord_t *>(t.max_z);
    v.left_child   = t.left_child;
    v.right_child  = t.right_child;
    v.parent       = t.parent;
    v.id           = t.id;
    v.is_ghost     = t.is_ghost;
    v.orig_idx     = t.orig_idx;
    v.num_leaves   = static_cast<size_t>(t.num_leaves);
    v.num_internal = t.num_leaves > 0 ? static_cast<size_t>(t.num_leaves - 1) : 0;
    return v;
}

void copy_out(const TreeSoA &s, RTree &t) {
    size_t n   = s.num_leaves;
    size_t tot = n > 0 ? 2 * n - 1 : 0;
    std::memcpy(t.min_x, s.min_x, tot * sizeof(coord_t));
    std::memcpy(t.max_x, s.max_x, tot * sizeof(coord_t));
    std::memcpy(t.min_y, s.min_y, tot * sizeof(coord_t));
    std::memcpy(t.max_y, s.max_y, tot * sizeof(coord_t));
    std::memcpy(t.min_z, s.min_z, tot * sizeof(coord_t));
    std::memcpy(t.max_z, s.max_z, tot * sizeof(coord_t));
    if (n > 1) {
        std::memcpy(t.left_child, s.left_child, (n - 1) * sizeof(int));
        std::memcpy(t.right_child, s.right_child, (n - 1) * sizeof(int));
        std::memcpy(t.parent, s.parent, tot * sizeof(int));
    }
    // leaf slots of the attribute arrays (internal slots are never written by the reference)
    for (size_t i = 0; i < n; ++i) {
        size_t leaf         = n - 1 + i;
        t.id[leaf]          = s.id[leaf];
        t.is_ghost[leaf]    = s.is_ghost[leaf];
        t.orig_idx[leaf]    = s.orig_idx[leaf];
    }
}

template <int MAXK>
void self_knn_t(const TreeSoA &tv, const int32_t *ids, int64_t num, int k, bool excl, size_t *oi, dist_t *od) {
    if (ids) self_knn_query_subset<MAXK>(Q(), tv, ids, static_cast<int>(num), k, oi, od, excl);
    else self_knn_query<MAXK>(Q(), tv, k, oi, od, excl);
    Q().wait();
}

template <int MAXK>
void knn_t(const TreeSoA &tv, const coord_t *qx, const coord_t *qy, const coord_t *qz, int64_t nq, int k, size_t *oi,
           dist_t *od) {
    knn_query<MAXK>(Q(), tv, qx, qy, qz, k, static_cast<int>(nq), oi, od);
}

} // namespace

extern "C" {

// Compile-time configuration of this build: coord (0 f32, 1 f64, 2 u32, 3 u64), sfc
// (0 Morton, 1 Peano-Hilbert), periodic, return_orig_indices.
void ref_config(int *coord, int *sfc, int *periodic, int *ret_orig) {
#if defined(FASTTREE_INTEGER_COORDS)
#if defined(POSITIONS_IN_64BIT)
    *coord = 3;
#else
    *coord = 2;
#endif
#elif defined(COORDS_TYPE_DOUBLE)
    *coord = 1;
#else
    *coord = 0;
#endif
#if defined(SFC_TYPE_MORTON)
    *sfc = 0;
#else
    *sfc = 1;
#endif
#if defined(PERIODIC_BC)
    *periodic = 1;
#else
    *periodic = 0;
#endif
#if defined(RETURN_ORIG_INDICES)
    *ret_orig = 1;
#else
    *ret_orig = 0;
#endif
}

int ref_compute_bbox(const void *x, const void *y, const void *z, int64_t n, void *out6) {
    BoundingBox<coord_t> b = compute_bbox(Q(), (const coord_t *)x, (const coord_t *)y, (const coord_t *)z, n);
    coord_t              *o = (coord_t *)out6;
    o[0] = b.min_x;
    o[1] = b.max_x;
    o[2] = b.min_y;
    o[3] = b.max_y;
    o[4] = b.min_z;
    o[5] = b.max_z;
    return 0;
}

int ref_sfc_encode(const void *x, const void *y, const void *z, int64_t n, const void *bbox6, uint64_t *hi,
                   uint64_t *lo) {
    const coord_t       *b = (const coord_t *)bbox6;
    BoundingBox<coord_t> bb(0, 0, 0, 0, 0, 0);
    if (b) bb = BoundingBox<coord_t>(b[0], b[1], b[2], b[3], b[4], b[5]);
    std::vector<sfc_key> k(n > 0 ? n : 1);
    sfc_encode(Q(), (const coord_t *)x, (const coord_t *)y, (const coord_t *)z, (size_t)n, k.data(), bb);
    for (int64_t i = 0; i < n; ++i) split_key(k[i], hi[i], lo[i]);
    return 0;
}

int ref_build_bvh(const void *x, const void *y, const void *z, int64_t n, const uint32_t *id, const int8_t *ghost,
                  const void *bbox6, RTree *out, uint64_t *sorted_hi, uint64_t *sorted_lo) {
    try {
        particles<coord_t> p;
        p.pos_x.assign((const coord_t *)x, (const coord_t *)x + n);
        p.pos_y.assign((const coord_t *)y, (const coord_t *)y + n);
        p.pos_z.assign((const coord_t *)z, (const coord_t *)z + n);
        if (id) p.id.assign(id, id + n);
        if (ghost) p.is_ghost.assign(ghost, ghost + n);
        TreeSoA              tree(Q(), (size_t)n);
        BvhScratch           scratch;
        BoundingBox<coord_t> bb(0, 0, 0, 0, 0, 0);
        BoundingBox<coord_t> *bbp = nullptr;
        if (bbox6) {
            const coord_t *b = (const coord_t *)bbox6;
            bb               = BoundingBox<coord_t>(b[0], b[1], b[2], b[3], b[4], b[5]);
            bbp              = &bb;
        }
        build_bvh(Q(), p, tree, scratch, bbp, nullptr);
        if (n == 1) tree.parent[0] = -1; // unset by the reference for a single leaf
        copy_out(tree, *out);
        if (n == 1) out->parent[0] = -1;
        for (int64_t i = 0; i < n; ++i) split_key(scratch.d_smk[i], sorted_hi[i], sorted_lo[i]);
        scratch.free_all(Q());
        tree.free(Q());
    } catch (const std::runtime_error &) {
        return 2;
    }
    return 0;
}

int ref_build_tree(const uint64_t *keys_hi, const uint64_t *keys_lo, const void *sx, const void *sy, const void *sz,
                   int64_t n, RTree *out) {
    std::vector<sfc_key> k(n > 0 ? n : 1);
    for (int64_t i = 0; i < n; ++i) k[i] = join_key(keys_hi ? keys_hi[i] : 0, keys_lo[i]);
    TreeSoA tree(Q(), (size_t)n);
    build_tree(Q(), tree, k.data(), (const coord_t *)sx, (const coord_t *)sy, (const coord_t *)sz);
    if (n == 1) tree.parent[0] = -1;
    copy_out(tree, *out);
    tree.free(Q());
    return 0;
}

int ref_self_knn(const RTree *t, const int32_t *leaf_ids, int64_t num, int k, int exclude_self, uint64_t *out_idx,
                 void *out_dist) {
    TreeSoA tv = view(*t);
    size_t *oi = reinterpret_cast<size_t *>(out_idx);
    dist_t *od = static_cast<dist_t *>(out_dist);
    try {
        if (k <= 32) self_knn_t<32>(tv, leaf_ids, num, k, exclude_self != 0, oi, od);
        else self_knn_t<512>(tv, leaf_ids, num, k, exclude_self != 0, oi, od);
    } catch (const std::invalid_argument &) {
        return 1;
    } catch (const std::runtime_error &) {
        return 2;
    }
    return 0;
}

int ref_knn(const RTree *t, const void *qx, const void *qy, const void *qz, int64_t nq, int k, int max_k,
            uint64_t *out_idx, void *out_dist) {
    TreeSoA        tv = view(*t);
    size_t        *oi = reinterpret_cast<size_t *>(out_idx);
    dist_t        *od = static_cast<dist_t *>(out_dist);
    const coord_t *x = (const coord_t *)qx, *y = (const coord_t *)qy, *z = (const coord_t *)qz;
    try {
        switch (max_k) {
        case 32: knn_t<32>(tv, x, y, z, nq, k, oi, od); break;
        case 48: knn_t<48>(tv, x, y, z, nq, k, oi, od); break;
        case 64: knn_t<64>(tv, x, y, z, nq, k, oi, od); break;
        case 128: knn_t<128>(tv, x, y, z, nq, k, oi, od); break;
        case 256: knn_t<256>(tv, x, y, z, nq, k, oi, od); break;
        case 512: knn_t<512>(tv, x, y, z, nq, k, oi, od); break;
        default: return 3;
        }
    } catch (const std::invalid_argument &) {
        return 1;
    } catch (const std::runtime_error &) {
        return 2;
    }
    return 0;
}

int ref_range(const RTree *t, const void *qx, const void *qy, const void *qz, const void *rmin, const void *rmax,
              int64_t nq, int32_t *results, int32_t *counts, int max_per_q) {
    TreeSoA tv = view(*t);
    range_query(Q(), tv, (const coord_t *)qx, (const coord_t *)qy, (const coord_t *)qz, (const coord_t *)rmin,
                (const coord_t *)rmax, (int)nq, results, counts, max_per_q);
    return 0;
}

// The reference's own heaps on a given sequence (mirrors test/test_self_knn.cpp:374-562):
// RegisterMaxHeap<double, int, 32> / LocalMaxHeap pushes with the prune check, then the
// in-place sort; SortedMergeHeap merge_batch rounds in one 32-wide work-group.
int ref_maxheap_run(int k, const double *d, const int32_t *ix, int m, int use_prune, double *out_d, int32_t *out_i,
                    int *out_count) {
    if (k > 32) return 1;
    RegisterMaxHeap<double, int, 32> h;
    for (int a = 0; a < m; ++a) {
        if (use_prune && h.should_prune(d[a], k)) continue;
        h.push(d[a], ix[a], k);
    }
    *out_count = h.count;
    h.extract_sorted(out_d, out_i, k);
    return 0;
}

int ref_mergeheap_run(int k, int cap, const double *d, const int32_t *ix, int rounds, double *out_d, int32_t *out_i) {
    std::vector<double>  od(cap);
    std::vector<int32_t> oi(cap);
    Q().submit([&](sycl::handler &h) {
        sycl::local_accessor<double, 1>  sh_dist(cap, h);
        sycl::local_accessor<int, 1>     sh_idx(cap, h);
        sycl::local_accessor<double, 1>  st_d(32, h);
        sycl::local_accessor<int, 1>     st_i(32, h);
        sycl::local_accessor<int, 1>     cnt(1, h);
        double                          *pod = od.data();
        int32_t                         *poi = oi.data();
        h.parallel_for(sycl::nd_range<1>(32, 32), [=](sycl::nd_item<1> item) {
            int lid = static_cast<int>(item.get_local_id(0));
            SortedMergeHeap<double, int>::init(item, sh_dist, sh_idx, cnt, cap);
            for (int r = 0; r < rounds; ++r)
                SortedMergeHeap<double, int>::merge_batch(item, sh_dist, sh_idx, cnt, st_d, st_i, d[r * 32 + lid],
                                                          ix[r * 32 + lid], k, cap);
            for (int i = lid; i < cap; i += 32) {
                pod[i] = sh_dist[i];
                poi[i] = sh_idx[i];
            }
        });
    });
    std::memcpy(out_d, od.data(), cap * sizeof(double));
    std::memcpy(out_i, oi.data(), cap * sizeof(int32_t));
    return 0;
}

} // extern "C"
