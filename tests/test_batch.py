"""Batched point sets (ft_batch_*): every set of a batch must equal its own independent
build_bvh + self_knn_query, bit for bit -- tree arrays, heights, neighbour indices and
distances -- for uneven sizes including empty sets and sets of 1, 2 and 3 points.  The
single-tree path is itself pinned to the oracle; a few sets are also checked against the
oracle directly."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")
if not torch.cuda.is_available():
    pytest.skip("no CUDA device", allow_module_level=True)

import fasttree_b200 as ft  # noqa: E402
from fasttree_b200 import datasets  # noqa: E402
from oracle import oracle as O  # noqa: E402
from tests.gpu_util import assert_tree_equal, dist_bits, gen  # noqa: E402

CASES = [
    ("f32", "morton", False),
    ("f64", "morton", False),
    ("f32", "ph", False),
    ("f64", "ph", False),
    ("u32", "ph", False),
    ("u32", "ph", True),
]
CODES = {"f32": O.F32, "f64": O.F64, "u32": O.U32, "morton": O.MORTON, "ph": O.PEANO_HILBERT}
SIZES = [0, 300, 1, 2, 0, 3, 17, 1000, 257, 64, 4096, 5, 2000, 0]
KINDS = ["uniform", "clustered", "degenerate"]


def make_sets(coord, sizes, seed=7):
    parts = [gen(KINDS[i % 3], int(n), CODES[coord], seed + i) for i, n in enumerate(sizes)]
    x, y, z = (np.concatenate([p[d] for p in parts]) for d in range(3))
    off = np.zeros(len(sizes) + 1, np.int64)
    off[1:] = np.cumsum(sizes)
    return x, y, z, off


def single(ctx, xs, ys, zs, k, method="plain", ids=None):
    tree = ft.TreeSoA(ctx, len(xs))
    ft.build_bvh(ctx, ft.particles(xs, ys, zs, ids), tree)
    i, d = ft.self_knn_query(ctx, tree, k, max_k=max(32, k), method=method)
    torch.cuda.synchronize()
    return tree, i.cpu().numpy(), d.cpu().numpy()


def rows(a, off, s):
    return a[off[s]:off[s + 1]]


@pytest.mark.parametrize("coord,sfc,periodic", CASES, ids=[f"{c}-{s}{'-per' if p else ''}" for c, s, p in CASES])
def test_each_set_equals_its_own_calls(coord, sfc, periodic):
    ctx = ft.Context(coord, sfc, periodic=periodic)
    x, y, z, off = make_sets(coord, SIZES)
    b = ft.BatchedSets(ctx, len(x), len(SIZES))
    b.build(off, x, y, z)
    b.check()
    box, heights = b.set_info()
    for k in (1, 16, 32):
        for method in ("plain", "fast"):
            bi, bd = b.self_knn(k, method=method)
            torch.cuda.synchronize()
            b.check()
            bi, bd = bi.cpu().numpy(), bd.cpu().numpy()
            for s, n in enumerate(SIZES):
                if n == 0:
                    continue
                sl = slice(off[s], off[s + 1])
                tree, si, sd = single(ctx, x[sl], y[sl], z[sl], k)
                assert np.array_equal(rows(bi, off, s), si), (s, k, method)
                assert np.array_equal(dist_bits(rows(bd, off, s)), dist_bits(sd)), (s, k, method)
                if k == 16 and method == "plain":
                    view = b.tree(s)
                    got, want = view.to_numpy(), tree.to_numpy()
                    for name, a in want.items():
                        g = got[name]
                        assert np.array_equal(g.view(np.uint8), a.view(np.uint8)), (s, name)
                    assert heights[s] == tree.height() == view.height()
                    if ctx.is_float:
                        want_box = ft.compute_bbox(ctx, x[sl], y[sl], z[sl])
                        assert np.array_equal(box[s].view(np.uint8), want_box.view(np.uint8)), s


@pytest.mark.parametrize("coord,sfc,periodic", [("f32", "morton", False), ("u32", "ph", True)])
def test_sets_against_the_oracle(coord, sfc, periodic):
    ctx = ft.Context(coord, sfc, periodic=periodic)
    x, y, z, off = make_sets(coord, SIZES, seed=11)
    b = ft.BatchedSets(ctx, len(x), len(SIZES))
    b.build(off, x, y, z)
    bi, bd = b.self_knn(32, method="fast")
    torch.cuda.synchronize()
    b.check()
    bi, bd = bi.cpu().numpy(), bd.cpu().numpy()
    opts = O.Options(CODES[coord], CODES[sfc], periodic)
    for s in (1, 2, 5, 7, 10, 12):
        n = SIZES[s]
        sl = slice(off[s], off[s + 1])
        ot = O.build_bvh(opts, x[sl], y[sl], z[sl])
        assert_tree_equal(b.tree(s).to_numpy(), ot, n)
        oi, od = O.self_knn(opts, ot, 32)
        assert np.array_equal(rows(bi, off, s), oi), s
        assert np.array_equal(dist_bits(rows(bd, off, s)), dist_bits(od)), s


def test_ids_ghosts_and_original_indices():
    ctx = ft.Context("f64", "morton", return_orig_indices=True)
    sizes = [500, 1, 0, 77, 1200]
    x, y, z, off = make_sets("f64", sizes, seed=3)
    rng = np.random.default_rng(5)
    ids = rng.integers(0, 2**32, len(x), dtype=np.uint64).astype(np.uint32)
    ghost = (rng.random(len(x)) < 0.2).astype(np.int8)
    b = ft.BatchedSets(ctx, len(x), len(sizes))
    b.build(off, x, y, z, id=ids, is_ghost=ghost)
    bi, bd = b.self_knn(8, method="fast", max_k=32)
    torch.cuda.synchronize()
    b.check()
    bi, bd = bi.cpu().numpy(), bd.cpu().numpy()
    for s, n in enumerate(sizes):
        if n == 0:
            continue
        sl = slice(off[s], off[s + 1])
        tree = ft.TreeSoA(ctx, n)
        ft.build_bvh(ctx, ft.particles(x[sl], y[sl], z[sl], ids[sl], ghost[sl]), tree)
        si, sd = ft.self_knn_query(ctx, tree, 8)
        torch.cuda.synchronize()
        got, want = b.tree(s).to_numpy(), tree.to_numpy()
        for name in ("id", "is_ghost", "orig_idx"):
            assert np.array_equal(got[name], want[name]), (s, name)
        assert np.array_equal(rows(bi, off, s), si.cpu().numpy())
        assert np.array_equal(dist_bits(rows(bd, off, s)), dist_bits(sd.cpu().numpy()))


def test_large_k_takes_the_reference_traversal():
    ctx = ft.Context("f32", "ph")
    sizes = [3000, 2, 150, 0, 900]
    x, y, z, off = make_sets("f32", sizes, seed=9)
    b = ft.BatchedSets(ctx, len(x), len(sizes))
    b.build(off, x, y, z)
    for k, method in ((100, "fast"), (100, "plain"), (64, "fast")):
        bi, bd = b.self_knn(k, method=method, max_k=128)
        torch.cuda.synchronize()
        b.check()
        bi, bd = bi.cpu().numpy(), bd.cpu().numpy()
        for s, n in enumerate(sizes):
            if n == 0:
                continue
            sl = slice(off[s], off[s + 1])
            _, si, sd = single(ctx, x[sl], y[sl], z[sl], k)
            assert np.array_equal(rows(bi, off, s), si), (s, k)
            assert np.array_equal(dist_bits(rows(bd, off, s)), dist_bits(sd)), (s, k)


def test_plummer_sets_fast_equals_plain_and_sampled_sets_equal_single_builds():
    # the batched-sets workload's shape at 512 sets (log-normal sizes, Plummer spheres, f32 Morton)
    sizes = datasets.batched_set_sizes(512, seed=4, median=2000.0, hi=60_000)
    x, y, z, off = datasets.batched_sets(sizes=sizes, seed=4)
    ctx = ft.Context("f32", "morton")
    b = ft.BatchedSets(ctx, len(x), len(sizes))
    b.build(off, x, y, z)
    fi, fd = b.self_knn(32, method="fast")
    torch.cuda.synchronize()
    st = b.query_stats()
    pi, pd = b.self_knn(32, method="plain")
    torch.cuda.synchronize()
    b.check()
    assert torch.equal(fi, pi) and torch.equal(fd, pd)
    assert st["replayed"] < len(x)
    fi, fd = fi.cpu().numpy(), fd.cpu().numpy()
    for s in np.random.default_rng(1).choice(len(sizes), 12, replace=False):
        sl = slice(off[s], off[s + 1])
        _, si, sd = single(ctx, x[sl], y[sl], z[sl], 32)
        assert np.array_equal(rows(fi, off, s), si), s
        assert np.array_equal(dist_bits(rows(fd, off, s)), dist_bits(sd)), s


def test_graph_replay_follows_new_coordinates():
    sizes = [700, 1, 3, 0, 2500, 40]
    ctx = ft.Context("f32", "morton")
    x, y, z, off = make_sets("f32", sizes, seed=21)
    N, k = len(x), 32
    dx, dy, dz = (torch.as_tensor(a, device="cuda") for a in (x, y, z))
    doff = torch.as_tensor(off, device="cuda")
    gi = torch.empty(N * k, dtype=torch.uint64, device="cuda")
    gd = torch.empty(N * k, dtype=torch.float64, device="cuda")
    b = ft.BatchedSets(ctx, N, len(sizes))
    ref = ft.BatchedSets(ctx, N, len(sizes))
    for rnd in range(3):
        if rnd:
            # new coordinates in the same buffers: the replayed graph must read them
            x2, y2, z2, _ = make_sets("f32", sizes, seed=100 + rnd)
            for d, a in zip((dx, dy, dz), (x2, y2, z2)):
                d.copy_(torch.as_tensor(a, device="cuda"))
        b.build_knn(doff, dx, dy, dz, k, gi, gd, method="fast")
        ref.build(doff, dx, dy, dz)
        ri, rd = ref.self_knn(k, method="plain")
        torch.cuda.synchronize()
        b.check()
        assert torch.equal(gi.view(N, k), ri) and torch.equal(gd.view(N, k), rd), rnd


def test_bad_offsets_are_reported_and_contained():
    ctx = ft.Context("f32", "morton")
    x, y, z, off = make_sets("f32", [100, 50, 80], seed=2)
    b = ft.BatchedSets(ctx, len(x), 3)
    for bad in (np.array([0, 100, 40, 230]), np.array([0, 100, 150, 200]), np.array([5, 100, 150, 230])):
        b.build(bad, x, y, z)
        b.self_knn(4)
        with pytest.raises(ValueError):
            b.check()
    b.build(off, x, y, z)  # the batch stays usable
    b.self_knn(4)
    b.check()


def test_rejections():
    with pytest.raises(ValueError):
        ft.BatchedSets(ft.Context("u64", "ph", periodic=True), 100, 0)  # no sets
    ctx = ft.Context("f32", "morton")
    x, y, z, off = make_sets("f32", [10, 20], seed=1)
    b = ft.BatchedSets(ctx, 30, 2)
    with pytest.raises(ValueError):
        b.self_knn(4)  # not built yet
    with pytest.raises(ValueError):
        ft.BatchedSets(ctx, 10, 2).build(off, x, y, z)  # more points than max_points
    b.build(off, x, y, z)
    with pytest.raises(ValueError):
        b.self_knn(40)  # k > max_k
    view = b.tree(1)
    with pytest.raises(ValueError):
        ft.build_bvh(ctx, ft.particles(x[:20], y[:20], z[:20]), view)
    with pytest.raises(ValueError):
        b.tree(5)


def test_periodic_sets_beyond_the_period():
    """u32 periodic sets where some sets hold coordinates at or above 2^21: those sets keep the
    reference traversal (non-monotone box distance there); every set equals the oracle."""
    ctx = ft.Context("u32", "ph", periodic=True)
    sizes = [900, 1500, 700, 2000]
    x, y, z, off = make_sets("u32", sizes, seed=21)
    x = x.copy()
    for s in (1, 3):  # push a few points of sets 1 and 3 past the period
        x[off[s]:off[s + 1]:37] += np.uint32(1 << 21)
    b = ft.BatchedSets(ctx, len(x), len(sizes))
    b.build(off, x, y, z)
    bi, bd = b.self_knn(16, method="fast")
    torch.cuda.synchronize()
    b.check()
    bi, bd = bi.cpu().numpy(), bd.cpu().numpy()
    opts = O.Options(CODES["u32"], CODES["ph"], True)
    for s in range(len(sizes)):
        sl = slice(off[s], off[s + 1])
        ot = O.build_bvh(opts, x[sl], y[sl], z[sl])
        oi, od = O.self_knn(opts, ot, 16)
        assert np.array_equal(rows(bi, off, s), oi), s
        assert np.array_equal(dist_bits(rows(bd, off, s)), dist_bits(od)), s
        vi, vd = ft.self_knn_query(ctx, b.tree(s), 16, method="fast")  # the set as a single tree
        torch.cuda.synchronize()
        assert np.array_equal(vi.cpu().numpy(), oi), s


@pytest.mark.parametrize("coord,sfc,periodic", [("f32", "morton", False), ("u32", "ph", True), ("f64", "ph", False)])
def test_batch_features_equal_single_tree_features(coord, sfc, periodic):
    """The learned bound's features of every leaf of a batch equal those of each set built as a
    tree of its own."""
    from fasttree_b200 import learned as L
    ctx = ft.Context(coord, sfc, periodic=periodic)
    x, y, z, off = make_sets(coord, [0, 300, 1, 2, 3, 17, 1000, 257, 2000])
    b = ft.BatchedSets(ctx, len(x), len(off) - 1)
    b.build(off, x, y, z)
    for k in (1, 8, 32, 64):
        f = b.bound_features(k).cpu().numpy()
        for s in range(len(off) - 1):
            a, e = int(off[s]), int(off[s + 1])
            if e - a < 1:
                continue
            tree = ft.TreeSoA(ctx, e - a)
            ft.build_bvh(ctx, ft.particles(x[a:e], y[a:e], z[a:e]), tree)
            want = L.features(ctx, tree, k).cpu().numpy()
            assert np.array_equal(f[a:e].view(np.uint32), want.view(np.uint32)), (k, s)


@pytest.mark.parametrize("coord,sfc,periodic", [("f32", "morton", False), ("u32", "ph", True)])
def test_learned_batched_query_is_exact_for_any_network(coord, sfc, periodic):
    """ft_batch_self_knn_learned and ft_batch_build_knn_learned return ft_batch_self_knn's rows
    for a trained, an untrained, a far-too-small and a far-too-large network; queries whose
    bound proves too small rerun the walk without it, and only ties reach the replay."""
    from fasttree_b200 import learned as L
    from oracle import bound_oracle as BOR
    ctx = ft.Context(coord, sfc, periodic=periodic)
    sizes = [int(s) for s in datasets.batched_set_sizes(200, seed=14, median=2000.0)]
    x, y, z, off = make_sets(coord, sizes, seed=31)
    tx, ty, tz, toff = make_sets(coord, sizes[:120], seed=77)
    N, k = len(x), 32
    trained, _ = L.train_bound_batched(ctx, toff, tx, ty, tz, k, steps=300, batch=4096)
    untrained = L.BoundModel(ctx, seed=3)
    tiny, huge = L.BoundModel(ctx, seed=3), L.BoundModel(ctx, seed=3)
    p = tiny.params
    p[BOR.OFF_B3] = -60.0
    tiny.params = p
    p[BOR.OFF_B3] = 60.0
    huge.params = p
    b = ft.BatchedSets(ctx, N, len(sizes))
    b.build(off, x, y, z)
    b.self_knn(k, method="fast")
    fast_replayed = b.query_stats()["replayed"]  # genuine ties (a third of the sets are duplicates)
    pi, pd = b.self_knn(k, method="plain")
    pi, pd = pi.clone(), pd.clone()
    for name, model in (("trained", trained), ("untrained", untrained), ("tiny", tiny), ("huge", huge)):
        li, ld = b.self_knn_learned(model, k, inflation=1.15)
        b.check()
        assert torch.equal(li, pi) and torch.equal(ld, pd), name
        st = b.query_stats()
        if name == "tiny":
            # every bound is about zero: every row whose k-th distance is not zero misses it
            # (the sets hold duplicate points, whose rows stay within a zero bound)
            positive = int((pd[:, -1].view(torch.int64) > 0).sum())
            assert st["bound_misses"] >= positive - 10, (st["bound_misses"], positive)
            # the misses rerun the walk without the bound, so the replay list holds the rows
            # the unbounded fast walk flags for ties (plus the few tied rows the first launch
            # finished within the zero bound), not the misses
            assert st["replayed"] <= fast_replayed + 0.01 * N, (st["replayed"], fast_replayed)
    # the same through one CUDA graph (build + learned query), replayed twice
    dx, dy, dz = (torch.from_numpy(a).cuda() for a in (x, y, z))
    doff = torch.from_numpy(off).cuda()
    gi = torch.empty(N * k, dtype=torch.uint64, device="cuda")
    gd = torch.empty(N * k, dtype=pd.dtype, device="cuda")
    for _ in range(2):
        gi.zero_()
        b.build_knn_learned(trained, doff, dx, dy, dz, k, gi, gd, inflation=1.3)
        b.check()
        assert torch.equal(gi.view(N, k), pi) and torch.equal(gd.view(N, k), pd)
