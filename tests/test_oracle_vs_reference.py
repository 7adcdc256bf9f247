"""The oracle restatement against the reference's own code run on the CPU (CPU only).

oracle/_ref holds the reference's headers compiled unmodified against a host SYCL
stand-in (oracle/ref.mk); these tests compare every output of the restatement with it,
bit for bit, on the reference test suite's input shapes.  Skipped where oracle/_ref was not
built (the reference sources are needed to build it).
"""
import numpy as np
import pytest

from oracle import oracle as O
from oracle import reference as R
from tests.gpu_util import CONFIG_IDS, CONFIGS, gen, radius, to_coord

TREE_ARRAYS = ("min_x", "max_x", "min_y", "max_y", "min_z", "max_z", "left_child", "right_child", "parent", "id",
               "is_ghost", "orig_idx")


def need(opts):
    if not R.available(opts):
        pytest.skip("reference checker not built (oracle/_ref)")


def same(a, b):
    a, b = np.asarray(a), np.asarray(b)
    return a.shape == b.shape and np.array_equal(a.view(np.uint8), b.view(np.uint8))


def trees_equal(a, b):
    return all(same(getattr(a, k), getattr(b, k)) for k in TREE_ARRAYS)


@pytest.mark.parametrize("cfg", CONFIGS, ids=CONFIG_IDS)
@pytest.mark.parametrize("kind", ["uniform", "clustered", "degenerate"])
def test_build_and_self_knn(cfg, kind):
    opts = O.Options(*cfg)
    need(opts)
    x, y, z = gen(kind, 1500, cfg[0], seed=21)
    ids = np.arange(1500, dtype=np.uint32)[::-1].copy()
    gh = (np.arange(1500) % 5 == 0).astype(np.int8)
    rt, ot = R.build_bvh(opts, x, y, z, ids, gh), O.build_bvh(opts, x, y, z, ids, gh)
    assert trees_equal(rt, ot)
    assert same(rt.sorted_hi, ot.sorted_hi) and same(rt.sorted_lo, ot.sorted_lo)
    for k in (1, 8, 32, 33, 64, 100):
        for excl in (True, False):
            ri, rd = R.self_knn(opts, rt, k, excl)
            oi, od = O.self_knn(opts, ot, k, excl)
            assert same(ri, oi) and same(rd, od), (k, excl)
    sub = np.array(sorted(set(range(0, 1500, 88)) | {0, 1499, 750}), np.int32)
    for k in (16, 33):
        ri, rd = R.self_knn(opts, rt, k, True, leaf_ids=sub)
        oi, od = O.self_knn(opts, ot, k, True, leaf_ids=sub)
        assert same(ri, oi) and same(rd, od)


@pytest.mark.parametrize("cfg", CONFIGS, ids=CONFIG_IDS)
@pytest.mark.parametrize("k,max_k", [(5, 256), (32, 32), (33, 64), (48, 128), (64, 64), (64, 256), (128, 128),
                                     (200, 256)])
def test_knn_query_heap_tiers(cfg, k, max_k):
    """knn_query small-k (RegisterMaxHeap) and large-k (SortedMergeHeap, including the
    k == HEAP_CAP case where the merge heap stops accepting candidates)."""
    opts = O.Options(*cfg)
    need(opts)
    x, y, z = gen("clustered", 1200, cfg[0], seed=5)
    rt = R.build_bvh(opts, x, y, z)
    rng = np.random.default_rng(6)
    q = rng.uniform(0, 100.0, (3, 64))
    qx, qy, qz = (to_coord(a, cfg[0]) for a in q)
    qx[:20], qy[:20], qz[:20] = x[:20], y[:20], z[:20]
    ri, rd = R.knn(opts, rt, qx, qy, qz, k, max_k)
    oi, od = O.knn(opts, rt, qx, qy, qz, k, max_k)
    assert same(ri, oi) and same(rd, od)


@pytest.mark.parametrize("cfg", CONFIGS, ids=CONFIG_IDS)
def test_range_query(cfg):
    opts = O.Options(*cfg)
    need(opts)
    x, y, z = gen("uniform", 2000, cfg[0], seed=8)
    rt = R.build_bvh(opts, x, y, z)
    rng = np.random.default_rng(12)
    q = rng.uniform(0, 100.0, (3, 100))
    qx, qy, qz = (to_coord(a, cfg[0]) for a in q)
    dt = qx.dtype
    rmin = np.array([radius(r, cfg[0]) for r in rng.uniform(0, 3, 100)], dt)
    rmax = np.array([radius(r, cfg[0]) for r in rng.uniform(3, 12, 100)], dt)
    rr, rc = R.range_query(opts, rt, qx, qy, qz, rmin, rmax, 16)
    orr, oc = O.range_query(opts, rt, qx, qy, qz, rmin, rmax, 16)
    assert same(rc, oc)
    for i in range(100):
        m = min(int(rc[i]), 16)
        assert same(rr[i, :m], orr[i, :m])


@pytest.mark.parametrize("cfg", CONFIGS, ids=CONFIG_IDS)
def test_encode_bbox_and_build_tree(cfg):
    opts = O.Options(*cfg)
    need(opts)
    x, y, z = gen("clustered", 3000, cfg[0], seed=9)
    assert same(R.compute_bbox(opts, x, y, z), O.compute_bbox(opts, x, y, z))
    bb = O.compute_bbox(opts, x, y, z)
    rh, rl = R.sfc_encode(opts, x, y, z, bb)
    oh, ol = O.sfc_encode(opts, x, y, z, bb)
    assert same(rh, oh) and same(rl, ol)
    order = np.lexsort((ol, oh))
    rt = R.build_tree(opts, oh[order], ol[order], x[order], y[order], z[order])
    ot = O.build_tree(opts, oh[order], ol[order], x[order], y[order], z[order])
    for k in ("min_x", "max_x", "min_y", "max_y", "min_z", "max_z", "left_child", "right_child", "parent"):
        assert same(getattr(rt, k), getattr(ot, k)), k


@pytest.mark.parametrize("ret_cfg", [(O.F64, O.MORTON, False, True), (O.U64, O.PEANO_HILBERT, True, True)],
                         ids=["f64-morton-orig", "u64-ph-per-orig"])
def test_return_orig_indices(ret_cfg):
    opts = O.Options(*ret_cfg)
    need(opts)
    x, y, z = gen("clustered", 1000, ret_cfg[0], seed=4)
    rt = R.build_bvh(opts, x, y, z)
    for k in (16, 40):
        ri, rd = R.self_knn(opts, rt, k, True)
        oi, od = O.self_knn(opts, rt, k, True)
        assert same(ri, oi) and same(rd, od)
    ri, rd = R.knn(opts, rt, x[:10], y[:10], z[:10], 64, 256)
    oi, od = O.knn(opts, rt, x[:10], y[:10], z[:10], 64, 256)
    assert same(ri, oi) and same(rd, od)


def test_edge_sizes():
    opts = O.Options(O.F64, O.MORTON)
    need(opts)
    for n in (1, 2, 7, 31, 33, 65):
        x, y, z = gen("uniform", n, O.F64, seed=777)
        rt, ot = R.build_bvh(opts, x, y, z), O.build_bvh(opts, x, y, z)
        assert trees_equal(rt, ot), n
        for k in (1, 2, 33):
            for excl in (True, False):
                ri, rd = R.self_knn(opts, rt, k, excl)
                oi, od = O.self_knn(opts, ot, k, excl)
                assert same(ri, oi) and same(rd, od), (n, k, excl)


def test_heaps_match_reference():
    opts = O.Options(O.F64, O.MORTON)
    need(opts)
    rng = np.random.default_rng(3)
    for trial in range(20):
        m = int(rng.integers(1, 200))
        d = rng.integers(0, 30, m).astype(np.float64)  # many ties
        ix = np.arange(m, dtype=np.int32)
        for k in (1, 7, 32):
            a = R.maxheap_run(opts, k, d, ix)
            b = O.maxheap_run(k, d, ix)
            assert same(a[0], b[0]) and same(a[1], b[1]) and a[2] == b[2]
    DMAX = np.finfo(np.float64).max
    for trial in range(10):
        rounds = int(rng.integers(1, 6))
        d = rng.integers(0, 20, (rounds, 32)).astype(np.float64)
        i = rng.integers(0, 1000, (rounds, 32)).astype(np.int32)
        d[rng.random((rounds, 32)) < 0.3] = DMAX
        for k, cap in ((48, 64), (64, 64), (20, 32), (100, 128)):
            a = R.mergeheap_run(opts, k, cap, d, i)
            b = O.mergeheap_run(k, cap, d, i)
            assert same(a[0], b[0]) and same(a[1], b[1]), (k, cap)
