"""GPU library vs CPU oracle: trees, self-kNN, kNN and range queries, bit-exact.

Every case runs the same seeded input through the CUDA library (through the C ABI) and the
oracle restatement, and compares every output array bit for bit: leaf order, topology,
boxes, neighbour indices (ties included) and distances.
"""
import numpy as np
import pytest

from oracle import oracle as O
from tests.gpu_util import (CONFIG_IDS, CONFIGS, NAMES, assert_tree_equal, dist_bits, gen, radius,
                            to_coord, tree_height)

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")
if not torch.cuda.is_available():
    pytest.skip("no CUDA device", allow_module_level=True)

import fasttree_b200 as ft  # noqa: E402


def make(coord, sfc, periodic, ret_orig=False):
    ctx = ft.Context(NAMES[coord], sfc, periodic=periodic, return_orig_indices=ret_orig)
    opts = O.Options(coord, sfc, periodic, ret_orig)
    return ctx, opts


def build_both(ctx, opts, x, y, z, **kw):
    tree = ft.TreeSoA(ctx, len(x))
    ft.build_bvh(ctx, ft.particles(x, y, z, kw.get("id"), kw.get("ghost")), tree, bbox=kw.get("bbox"))
    ot = O.build_bvh(opts, x, y, z, kw.get("id"), kw.get("ghost"), kw.get("bbox"))
    return tree, ot


@pytest.mark.parametrize("cfg", CONFIGS, ids=CONFIG_IDS)
@pytest.mark.parametrize("kind", ["uniform", "clustered", "degenerate"])
def test_build_matches_oracle(cfg, kind):
    coord, sfc, per = cfg
    ctx, opts = make(coord, sfc, per)
    n = 20000
    x, y, z = gen(kind, n, coord, seed=11)
    ids = np.arange(n, dtype=np.uint32)[::-1].copy()
    ghost = (np.arange(n) % 7 == 0).astype(np.int8)
    tree, ot = build_both(ctx, opts, x, y, z, id=ids, ghost=ghost)
    g = tree.to_numpy()
    assert_tree_equal(g, ot, n)
    assert tree.height() == tree_height(ot.parent, n)


@pytest.mark.parametrize("cfg", CONFIGS, ids=CONFIG_IDS)
@pytest.mark.parametrize("kind", ["uniform", "clustered", "degenerate"])
@pytest.mark.parametrize("k", [1, 16, 32, 33, 64])
@pytest.mark.parametrize("method", ["plain", "fast"])
def test_self_knn_matches_oracle(cfg, kind, k, method):
    coord, sfc, per = cfg
    ctx, opts = make(coord, sfc, per)
    n = 4000
    x, y, z = gen(kind, n, coord, seed=5)
    tree, ot = build_both(ctx, opts, x, y, z)
    for excl in (True, False):
        gi, gd = ft.self_knn_query(ctx, tree, k, exclude_self=excl, max_k=max(k, 32), method=method)
        torch.cuda.synchronize()
        oi, od = O.self_knn(opts, ot, k, excl)
        gi, gd = gi.cpu().numpy(), gd.cpu().numpy()
        assert np.array_equal(gi, oi), f"indices differ (excl={excl}), first row {np.argmax((gi != oi).any(1))}"
        assert np.array_equal(dist_bits(gd), dist_bits(od)), f"distances differ (excl={excl})"


@pytest.mark.parametrize("cfg", [CONFIGS[1], CONFIGS[7]], ids=[CONFIG_IDS[1], CONFIG_IDS[7]])
@pytest.mark.parametrize("k", [16, 33, 128, 256])
@pytest.mark.parametrize("method", ["plain", "fast"])
def test_self_knn_subset_and_orig_indices(cfg, k, method):
    coord, sfc, per = cfg
    for ret_orig in (False, True):
        ctx, opts = make(coord, sfc, per, ret_orig)
        n = 3000
        x, y, z = gen("clustered", n, coord, seed=7)
        tree, ot = build_both(ctx, opts, x, y, z)
        sub = sorted(set(list(range(0, n, n // 17)) + [0, n - 1, n // 2]))
        leaf_ids = torch.tensor(sub, dtype=torch.int32, device="cuda")
        for excl in (True, False):
            gi, gd = ft.self_knn_query_subset(ctx, tree, leaf_ids, k, exclude_self=excl, method=method)
            torch.cuda.synchronize()
            oi, od = O.self_knn(opts, ot, k, excl, leaf_ids=np.array(sub, np.int32))
            assert np.array_equal(gi.cpu().numpy(), oi)
            assert np.array_equal(dist_bits(gd.cpu().numpy()), dist_bits(od))


@pytest.mark.parametrize("cfg", CONFIGS, ids=CONFIG_IDS)
@pytest.mark.parametrize("k,max_k", [(5, 256), (32, 256), (33, 256), (48, 128), (64, 256), (64, 64), (128, 128)])
@pytest.mark.parametrize("method", ["plain", "fast"])
def test_knn_query_matches_oracle(cfg, k, max_k, method):
    coord, sfc, per = cfg
    ctx, opts = make(coord, sfc, per)
    n = 3000
    x, y, z = gen("clustered", n, coord, seed=3)
    tree, ot = build_both(ctx, opts, x, y, z)
    rng = np.random.default_rng(9)
    q = rng.uniform(0, 100.0, (3, 200))
    qx, qy, qz = (to_coord(a, coord) for a in q)
    # half the queries on particles (ties with exact hits)
    qx[:50], qy[:50], qz[:50] = x[:50], y[:50], z[:50]
    gi, gd = ft.knn_query(ctx, tree, qx, qy, qz, k, max_k=max_k, method=method)
    oi, od = O.knn(opts, ot, qx, qy, qz, k, max_k)
    assert np.array_equal(gi.cpu().numpy(), oi)
    assert np.array_equal(dist_bits(gd.cpu().numpy()), dist_bits(od))


@pytest.mark.parametrize("cfg", CONFIGS, ids=CONFIG_IDS)
@pytest.mark.parametrize("max_per", [0, 7, 64])
def test_range_query_matches_oracle(cfg, max_per):
    coord, sfc, per = cfg
    ctx, opts = make(coord, sfc, per)
    n = 5000
    x, y, z = gen("uniform", n, coord, seed=4)
    tree, ot = build_both(ctx, opts, x, y, z)
    rng = np.random.default_rng(10)
    q = rng.uniform(0, 100.0, (3, 300))
    qx, qy, qz = (to_coord(a, coord) for a in q)
    dt = qx.dtype
    rmin = np.array([radius(r, coord) for r in rng.uniform(0, 2, 300)], dt)
    rmax = np.array([radius(r, coord) for r in rng.uniform(2, 8, 300)], dt)
    gr, gc = ft.range_query(ctx, tree, qx, qy, qz, rmin, rmax, max_per)
    orr, oc = O.range_query(opts, ot, qx, qy, qz, rmin, rmax, max_per)
    gc = gc.cpu().numpy()
    assert np.array_equal(gc, oc)
    if max_per == 0:
        return
    gr = gr.cpu().numpy().reshape(300, max_per)
    for i in range(300):
        m = min(oc[i], max_per)
        assert np.array_equal(gr[i, :m], orr[i, :m])


@pytest.mark.parametrize("cfg", [CONFIGS[1], CONFIGS[4], CONFIGS[7]], ids=[CONFIG_IDS[1], CONFIG_IDS[4], CONFIG_IDS[7]])
@pytest.mark.parametrize("n", [1, 2, 7, 31, 33, 63, 65, 99])
@pytest.mark.parametrize("method", ["plain", "fast"])
def test_edge_sizes(cfg, n, method):
    """n = 1, 2 and partial warps (test/test_self_knn.cpp:876-1003)."""
    coord, sfc, per = cfg
    ctx, opts = make(coord, sfc, per)
    x, y, z = gen("uniform", n, coord, seed=777)
    tree, ot = build_both(ctx, opts, x, y, z)
    assert_tree_equal(tree.to_numpy(), ot, n)
    for k in (1, 2, 4, 32, 33, 64):
        for excl in (True, False):
            gi, gd = ft.self_knn_query(ctx, tree, k, exclude_self=excl, max_k=max(k, 32), method=method)
            torch.cuda.synchronize()
            oi, od = O.self_knn(opts, ot, k, excl)
            assert np.array_equal(gi.cpu().numpy(), oi), (n, k, excl)
            assert np.array_equal(dist_bits(gd.cpu().numpy()), dist_bits(od)), (n, k, excl)
        gi, gd = ft.knn_query(ctx, tree, x[:3], y[:3], z[:3], k, max_k=64, method=method)
        oi, od = O.knn(opts, ot, x[:3], y[:3], z[:3], k, 64)
        assert np.array_equal(gi.cpu().numpy(), oi)


def test_caller_keys_sorted_in_place():
    """build_bvh with caller keys sorts them in place (src/hlbvh.hpp:2198-2232)."""
    ctx, opts = make(O.U64, O.PEANO_HILBERT, True)
    x, y, z = gen("clustered", 5000, O.U64, seed=8)
    keys = ft.sfc_encode(ctx, x, y, z)  # (n, 3) uint64 {hs, is, ls}
    hi, lo = O.sfc_encode(opts, x, y, z)
    assert np.array_equal(keys[:, 1], hi) and np.array_equal(keys[:, 2], lo) and not keys[:, 0].any()
    tree = ft.TreeSoA(ctx, 5000)
    k2 = keys.copy()
    ft.build_bvh(ctx, ft.particles(x, y, z), tree, key=k2)
    ot = O.build_bvh(opts, x, y, z, keys=(hi.copy(), lo.copy()))
    assert np.array_equal(k2[:, 1], ot.sorted_hi) and np.array_equal(k2[:, 2], ot.sorted_lo)
    assert_tree_equal(tree.to_numpy(), ot, 5000)


@pytest.mark.parametrize("coord", [O.F32, O.F64])
def test_build_tree_line_fixture(coord):
    """test/test_mpi.cpp:183-217: 1000 points on a line, keys 0..999, 20 within 10 of 500.5."""
    ctx, opts = make(coord, O.MORTON, False)
    n = 1000
    xs = np.arange(n).astype(O.NP_COORD[coord])
    zs = np.zeros(n, O.NP_COORD[coord])
    tree = ft.TreeSoA(ctx, n)
    ft.build_tree(ctx, tree, np.arange(n, dtype=np.uint64), xs, zs, zs)
    res, cnt = ft.range_query(ctx, tree, [500.5], [0.0], [0.0], [0.0], [10.0], 100)
    assert int(cnt[0]) == 20
    ot = O.build_tree(opts, None, np.arange(n, dtype=np.uint64), xs, zs, zs)
    g = tree.to_numpy()
    for k in ("left_child", "right_child", "parent", "min_x", "max_x"):
        o = getattr(ot, k)
        assert np.array_equal(g[k], o[:len(g[k])]), k


def test_ghost_fixture():
    """test/test_domain_decomposition.cpp:360-470: ghosts survive the sort and are found."""
    ctx, opts = make(O.F64, O.MORTON, False)
    x = np.array([1.0, 2.0, 3.0, -1.0, 10.0])
    y = np.zeros(5)
    z = np.zeros(5)
    ids = np.array([100, 101, 102, 200, 201], np.uint32)
    gh = np.array([0, 0, 0, 1, 1], np.int8)
    tree = ft.TreeSoA(ctx, 5)
    ft.build_bvh(ctx, ft.particles(x, y, z, ids, gh), tree)
    g = tree.to_numpy()
    assert int((g["is_ghost"][4:] == 1).sum()) == 2
    res, cnt = ft.range_query(ctx, tree, [-0.5], [0.0], [0.0], [0.0], [2.0], 10)
    hit = sorted(int(g["id"][4 + int(r)]) for r in res.cpu().numpy()[0, :int(cnt[0])])
    assert hit == [100, 200]
    idx, d = ft.knn_query(ctx, tree, [9.5], [0.0], [0.0], 2)
    first = int(idx.cpu().numpy()[0, 0])
    assert g["id"][4 + first] == 201 and g["is_ghost"][4 + first] == 1
    assert abs(float(d.cpu().numpy()[0, 0]) - 0.25) < 1e-12


def test_invalid_arguments():
    ctx, opts = make(O.F64, O.MORTON, False)
    x, y, z = gen("uniform", 100, O.F64, seed=1)
    tree = ft.TreeSoA(ctx, 100)
    ft.build_bvh(ctx, ft.particles(x, y, z), tree)
    with pytest.raises(ValueError):
        ft.self_knn_query(ctx, tree, 33, max_k=32)  # k > MAXK (src/hlbvh.hpp:1940-1944)
    with pytest.raises(ValueError):
        ft.knn_query(ctx, tree, x[:2], y[:2], z[:2], 300, max_k=256)
    small = ft.TreeSoA(ctx, 10)
    with pytest.raises(ValueError):
        ft.build_bvh(ctx, ft.particles(x, y, z), small)
    with pytest.raises(ValueError):
        ft.Context("u64", "morton")


@pytest.mark.parametrize("cfg", CONFIGS, ids=CONFIG_IDS)
@pytest.mark.parametrize("kind", ["uniform", "clustered", "degenerate"])
@pytest.mark.parametrize("k", [1, 8, 32, 33, 64])
def test_fast_self_knn_matches_oracle(cfg, kind, k):
    """method "fast" (warp-shared walk + SFC-window seeding + exact replay of tied queries) gives
    the reference's output bit for bit."""
    coord, sfc, per = cfg
    ctx, opts = make(coord, sfc, per)
    n = 6000
    x, y, z = gen(kind, n, coord, seed=15)
    tree, ot = build_both(ctx, opts, x, y, z)
    for excl in (True, False):
        gi, gd = ft.self_knn_query(ctx, tree, k, exclude_self=excl, max_k=max(k, 32), method="fast")
        torch.cuda.synchronize()
        stats = ctx.query_stats()
        oi, od = O.self_knn(opts, ot, k, excl)
        assert np.array_equal(gi.cpu().numpy(), oi), (excl, stats)
        assert np.array_equal(dist_bits(gd.cpu().numpy()), dist_bits(od)), (excl, stats)
        if kind == "degenerate" and k > 1:
            assert stats["replayed"] > 0  # duplicate points force the exact replay


@pytest.mark.parametrize("cfg", CONFIGS, ids=CONFIG_IDS)
@pytest.mark.parametrize("variant", [1, 2, 3, 4, 5])
def test_fast_walk_variants_match_oracle(cfg, variant):
    """Every walk of the fast path (1 per-lane, 2 compact per-lane, 3 warp-shared, 4 over the
    4-wide records, 5 the group walk) gives the reference's output, ties included."""
    coord, sfc, per = cfg
    ctx, opts = make(coord, sfc, per)
    for kind, k in (("clustered", 32), ("degenerate", 16), ("uniform", 64)):
        x, y, z = gen(kind, 5000, coord, seed=23)
        tree, ot = build_both(ctx, opts, x, y, z)
        gi, gd = ft.self_knn_query(ctx, tree, k, max_k=max(k, 32), method="fast", variant=variant)
        torch.cuda.synchronize()
        oi, od = O.self_knn(opts, ot, k, True)
        assert np.array_equal(gi.cpu().numpy(), oi), (kind, k)
        assert np.array_equal(dist_bits(gd.cpu().numpy()), dist_bits(od)), (kind, k)


@pytest.mark.parametrize("cfg", [CONFIGS[1], CONFIGS[7]], ids=[CONFIG_IDS[1], CONFIG_IDS[7]])
def test_fast_self_knn_subset_and_orig(cfg):
    coord, sfc, per = cfg
    for ret_orig in (False, True):
        ctx, opts = make(coord, sfc, per, ret_orig)
        n = 5000
        x, y, z = gen("clustered", n, coord, seed=19)
        tree, ot = build_both(ctx, opts, x, y, z)
        rng = np.random.default_rng(1)
        sub = np.sort(rng.choice(n, 700, replace=False)).astype(np.int32)
        ids = torch.from_numpy(sub).cuda()
        for k in (16, 40):
            gi, gd = ft.self_knn_query_subset(ctx, tree, ids, k, exclude_self=True, method="fast")
            torch.cuda.synchronize()
            oi, od = O.self_knn(opts, ot, k, True, leaf_ids=sub)
            assert np.array_equal(gi.cpu().numpy(), oi)
            assert np.array_equal(dist_bits(gd.cpu().numpy()), dist_bits(od))


@pytest.mark.parametrize("method,variant", [("plain", 0), ("fast", 0), ("fast", 5)])
def test_periodic_wrap_edges_u64(method, variant):
    """42-bit periodic distances at the wrap: points at 0, 2^41 (half the period) and
    2^42 - 1, where the wrapped gap reaches its extreme values."""
    ctx, opts = make(O.U64, O.PEANO_HILBERT, True)
    rng = np.random.default_rng(5)
    n = 3000
    B = 1 << 42
    base = np.array([0, 1, B // 2 - 1, B // 2, B // 2 + 1, B - 2, B - 1, 3 * (B // 4)], np.uint64)
    x = rng.choice(base, n).astype(np.uint64)
    y = rng.choice(base, n).astype(np.uint64)
    z = (rng.integers(0, B, n)).astype(np.uint64)
    tree, ot = build_both(ctx, opts, x, y, z)
    for k in (4, 32):
        gi, gd = ft.self_knn_query(ctx, tree, k, method=method, variant=variant)
        torch.cuda.synchronize()
        oi, od = O.self_knn(opts, ot, k, True)
        assert np.array_equal(gi.cpu().numpy(), oi) and np.array_equal(gd.cpu().numpy(), od)
    q = np.array([0, B // 2, B - 1, B // 4], np.uint64)
    gi, gd = ft.knn_query(ctx, tree, q, q, q, 16, method=method, variant=variant)
    oi, od = O.knn(opts, ot, q, q, q, 16)
    assert np.array_equal(gi.cpu().numpy(), oi) and np.array_equal(gd.cpu().numpy(), od)


@pytest.mark.parametrize("coord", [O.U64, O.U32])
def test_periodic_coordinates_beyond_the_period(coord):
    """Periodic integer trees holding coordinates at or above the period (2^42 / 2^21): the
    reference masks only the query's coordinate, so its box distance is not monotone there;
    the fast walk must not be taken and every method returns the reference's rows."""
    ctx, opts = make(coord, O.PEANO_HILBERT, True)
    x, y, z = gen("clustered", 4000, coord, seed=51)
    bits = 42 if coord == O.U64 else 21
    dt = x.dtype.type
    x = x.copy()
    x[::53] += dt(1 << bits)
    tree, ot = build_both(ctx, opts, x, y, z)
    for k in (8, 32):
        oi, od = O.self_knn(opts, ot, k, True)
        for method in ("plain", "fast"):
            gi, gd = ft.self_knn_query(ctx, tree, k, max_k=32, method=method)
            torch.cuda.synchronize()
            assert np.array_equal(gi.cpu().numpy(), oi), (k, method)
            assert np.array_equal(dist_bits(gd.cpu().numpy()), dist_bits(od)), (k, method)
    qx, qy, qz = gen("uniform", 300, coord, seed=52)
    oi, od = O.knn(opts, ot, qx, qy, qz, 16)
    gi, gd = ft.knn_query(ctx, tree, qx, qy, qz, 16, method="fast")
    assert np.array_equal(gi.cpu().numpy(), oi) and np.array_equal(dist_bits(gd.cpu().numpy()), dist_bits(od))


@pytest.mark.parametrize("long_runs", [False, True])
def test_u64_keys_equal_in_the_high_word(long_runs):
    """126-bit keys that share their high word (points a few units apart) come out in the full
    key order with equal keys by input index, through the short-run fix-up and, with runs
    longer than it takes, through the full two-word sort."""
    ctx, opts = make(O.U64, O.PEANO_HILBERT, True)
    rng = np.random.default_rng(17)
    n_cl = 1500
    centres = rng.integers(0, 1 << 42, (3, n_cl), dtype=np.uint64)
    sizes = rng.integers(1, 12, n_cl)
    if long_runs:
        sizes[::300] = 60  # runs longer than the fix-up's cap
    cols = []
    for d in range(3):
        c = np.repeat(centres[d], sizes)
        off = rng.integers(0, 1 << 12, len(c), dtype=np.uint64)  # below the high word's last bit
        cols.append(np.minimum(c + off, np.uint64((1 << 42) - 1)))
    perm = rng.permutation(len(cols[0]))
    x, y, z = (a[perm] for a in cols)
    x[:50] = x[50:100]  # exact duplicates as well
    y[:50] = y[50:100]
    z[:50] = z[50:100]
    tree, ot = build_both(ctx, opts, x, y, z)
    assert_tree_equal(tree.to_numpy(), ot, len(x))
    gi, gd = ft.self_knn_query(ctx, tree, 16, method="fast")
    oi, od = O.self_knn(opts, ot, 16, True)
    torch.cuda.synchronize()
    assert np.array_equal(gi.cpu().numpy(), oi) and np.array_equal(gd.cpu().numpy(), od)
