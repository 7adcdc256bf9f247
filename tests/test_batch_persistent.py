"""The persistent batched launch (ft_batch_build_knn with FT_METHOD_PERSISTENT) and batches of
64-bit integer positions (126-bit keys), whose builds always take the persistent launch's
per-set path: every set must equal its own build_bvh + self_knn_query, bit for bit -- tree
arrays, heights, boxes, neighbour rows -- and the persistent launch must return the same
rows and trees as the launch sequence."""
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
    ("u64", "ph", False),
    ("u64", "ph", True),
]
IDS = [f"{c}-{s}{'-per' if p else ''}" for c, s, p in CASES]
CODES = {"f32": O.F32, "f64": O.F64, "u32": O.U32, "u64": O.U64, "morton": O.MORTON, "ph": O.PEANO_HILBERT}
SIZES = [0, 300, 1, 2, 0, 3, 17, 1000, 257, 64, 4096, 5, 2000, 0, 9000]
KINDS = ["uniform", "clustered", "degenerate"]
TREE_ARRAYS = ("min_x", "max_x", "min_y", "max_y", "min_z", "max_z", "left_child", "right_child", "parent", "id",
               "is_ghost", "orig_idx")


def make_sets(coord, sizes, seed=7):
    parts = [gen(KINDS[i % 3], int(n), CODES[coord], seed + i) for i, n in enumerate(sizes)]
    x, y, z = (np.concatenate([p[d] for p in parts]) for d in range(3))
    off = np.zeros(len(sizes) + 1, np.int64)
    off[1:] = np.cumsum(sizes)
    return x, y, z, off


def rows(a, off, s):
    return a[off[s]:off[s + 1]]


def persistent(ctx, x, y, z, off, k, **kw):
    N = len(x)
    b = ft.BatchedSets(ctx, N, len(off) - 1)
    dx, dy, dz = (torch.as_tensor(a, device="cuda") for a in (x, y, z))
    doff = torch.as_tensor(off, device="cuda")
    gi = torch.empty(max(N, 1) * k, dtype=torch.uint64, device="cuda")
    gd = torch.empty(max(N, 1) * k, dtype=ft.dist_torch_dtype(ctx.coord), device="cuda")
    b.build_knn(doff, dx, dy, dz, k, gi, gd, method="persistent", max_k=max(32, k), **kw)
    torch.cuda.synchronize()
    b.check()
    return b, gi[:N * k].view(N, k), gd[:N * k].view(N, k), (doff, dx, dy, dz, gi, gd)


@pytest.mark.parametrize("coord,sfc,periodic", CASES, ids=IDS)
def test_persistent_sets_equal_their_own_calls(coord, sfc, periodic):
    ctx = ft.Context(coord, sfc, periodic=periodic)
    x, y, z, off = make_sets(coord, SIZES)
    k = 16
    b, gi, gd, _ = persistent(ctx, x, y, z, off, k)
    box, heights = b.set_info()
    gi, gd = gi.cpu().numpy(), gd.cpu().numpy()
    for s, n in enumerate(SIZES):
        if n == 0:
            continue
        sl = slice(off[s], off[s + 1])
        tree = ft.TreeSoA(ctx, n)
        ft.build_bvh(ctx, ft.particles(x[sl], y[sl], z[sl]), tree)
        si, sd = ft.self_knn_query(ctx, tree, k, method="plain")
        torch.cuda.synchronize()
        assert np.array_equal(rows(gi, off, s), si.cpu().numpy()), s
        assert np.array_equal(dist_bits(rows(gd, off, s)), dist_bits(sd.cpu().numpy())), s
        view = b.tree(s)
        got, want = view.to_numpy(), tree.to_numpy()
        for name in TREE_ARRAYS:
            assert np.array_equal(got[name].view(np.uint8), want[name].view(np.uint8)), (s, name)
        assert heights[s] == tree.height() == view.height(), s
        want_box = ft.compute_bbox(ctx, x[sl], y[sl], z[sl])
        assert np.array_equal(box[s].view(np.uint8), want_box.view(np.uint8)), s


@pytest.mark.parametrize("coord,sfc,periodic", [("f32", "morton", False), ("f64", "ph", False),
                                                ("u32", "ph", True)])
def test_persistent_equals_the_launch_sequence(coord, sfc, periodic):
    """Same trees (every node array of the batch) and rows as ft_batch_build_knn's launch
    sequence, at k = 1, 32 and 64 (both heap tiers), with and without exclude_self."""
    ctx = ft.Context(coord, sfc, periodic=periodic)
    x, y, z, off = make_sets(coord, SIZES, seed=41)
    N = len(x)
    seq = ft.BatchedSets(ctx, N, len(SIZES))
    seq.build(off, x, y, z)
    want = {s: seq.tree(s).to_numpy() for s, n in enumerate(SIZES) if n > 0}
    for k, excl in ((32, True), (1, True), (64, True), (32, False)):
        b, gi, gd, _ = persistent(ctx, x, y, z, off, k, exclude_self=excl)
        for s, w in want.items():
            got = b.tree(s).to_numpy()
            for name in TREE_ARRAYS:
                assert np.array_equal(got[name].view(np.uint8), w[name].view(np.uint8)), (k, s, name)
        si, sd = seq.self_knn(k, exclude_self=excl, max_k=max(32, k), method="plain")
        torch.cuda.synchronize()
        assert torch.equal(gi, si) and torch.equal(gd, sd), (k, excl)


def test_persistent_u64_sets_against_the_oracle():
    for periodic in (False, True):
        ctx = ft.Context("u64", "ph", periodic=periodic)
        x, y, z, off = make_sets("u64", SIZES, seed=13)
        b, gi, gd, _ = persistent(ctx, x, y, z, off, 32)
        gi, gd = gi.cpu().numpy(), gd.cpu().numpy()
        opts = O.Options(O.U64, O.PEANO_HILBERT, periodic)
        for s in (1, 2, 5, 7, 10, 14):
            n = SIZES[s]
            sl = slice(off[s], off[s + 1])
            ot = O.build_bvh(opts, x[sl], y[sl], z[sl])
            assert_tree_equal(b.tree(s).to_numpy(), ot, n)
            oi, od = O.self_knn(opts, ot, 32)
            assert np.array_equal(rows(gi, off, s), oi), (periodic, s)
            assert np.array_equal(rows(gd, off, s), od), (periodic, s)


def test_u64_batch_build_then_queries():
    """ft_batch_build of 126-bit-key sets, then the fast and plain batched queries and the
    learned bound: each equals the set's own calls."""
    from fasttree_b200 import learned as L
    ctx = ft.Context("u64", "ph", periodic=True)
    x, y, z, off = make_sets("u64", SIZES, seed=17)
    b = ft.BatchedSets(ctx, len(x), len(SIZES))
    b.build(off, x, y, z)
    b.check()
    fi, fd = b.self_knn(32, method="fast")
    fi, fd = fi.clone(), fd.clone()
    pi, pd = b.self_knn(32, method="plain")
    li, ld = b.self_knn_learned(L.BoundModel(ctx, seed=3), 32, inflation=1.3)
    torch.cuda.synchronize()
    b.check()
    assert torch.equal(fi, pi) and torch.equal(fd, pd)
    assert torch.equal(li, pi) and torch.equal(ld, pd)
    pi, pd = pi.cpu().numpy(), pd.cpu().numpy()
    for s, n in enumerate(SIZES):
        if n == 0:
            continue
        sl = slice(off[s], off[s + 1])
        tree = ft.TreeSoA(ctx, n)
        ft.build_bvh(ctx, ft.particles(x[sl], y[sl], z[sl]), tree)
        si, sd = ft.self_knn_query(ctx, tree, 32, method="plain")
        torch.cuda.synchronize()
        assert np.array_equal(rows(pi, off, s), si.cpu().numpy()), s
        assert np.array_equal(rows(pd, off, s), sd.cpu().numpy()), s
        got, want = b.tree(s).to_numpy(), tree.to_numpy()
        for name in TREE_ARRAYS:
            assert np.array_equal(got[name].view(np.uint8), want[name].view(np.uint8)), (s, name)


def test_persistent_plummer_sets_and_graph_replay():
    """The batched-sets workload's shape (log-normal sizes, Plummer spheres, f32 Morton) with a
    few large sets: the persistent graph, replayed with new coordinates in the same buffers,
    keeps returning the launch sequence's rows."""
    sizes = datasets.batched_set_sizes(600, seed=4, median=2000.0, hi=200_000)
    sizes[3] = 250_000  # one set far larger than the rest: its build is the longest
    x, y, z, off = datasets.batched_sets(sizes=sizes, seed=4)
    ctx = ft.Context("f32", "morton")
    b, gi, gd, bufs = persistent(ctx, x, y, z, off, 32)
    seq = ft.BatchedSets(ctx, len(x), len(sizes))
    for rnd in range(3):
        if rnd:
            x2, y2, z2, _ = datasets.batched_sets(sizes=sizes, seed=50 + rnd)
            for d, a in zip(bufs[1:4], (x2, y2, z2)):
                d.copy_(torch.as_tensor(a, device="cuda"))
            b.build_knn(bufs[0], *bufs[1:4], 32, bufs[4], bufs[5], method="persistent")
            torch.cuda.synchronize()
            b.check()
        seq.build(bufs[0], *bufs[1:4])
        si, sd = seq.self_knn(32, method="plain")
        torch.cuda.synchronize()
        assert torch.equal(gi, si) and torch.equal(gd, sd), rnd
    st = b.query_stats()
    assert st["queries"] == len(x) and st["replayed"] < 0.01 * len(x)


def test_persistent_ids_ghosts_and_original_indices():
    ctx = ft.Context("f64", "morton", return_orig_indices=True)
    sizes = [500, 1, 0, 77, 1200]
    x, y, z, off = make_sets("f64", sizes, seed=3)
    rng = np.random.default_rng(5)
    ids = rng.integers(0, 2**32, len(x), dtype=np.uint64).astype(np.uint32)
    ghost = (rng.random(len(x)) < 0.2).astype(np.int8)
    b, gi, gd, _ = persistent(ctx, x, y, z, off, 8, id=ids, is_ghost=ghost)
    gi, gd = gi.cpu().numpy(), gd.cpu().numpy()
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
        assert np.array_equal(rows(gi, off, s), si.cpu().numpy())
        assert np.array_equal(dist_bits(rows(gd, off, s)), dist_bits(sd.cpu().numpy()))


def test_persistent_bad_offsets_are_reported_and_contained():
    ctx = ft.Context("u64", "ph")
    x, y, z, off = make_sets("u64", [100, 50, 80], seed=2)
    for bad in (np.array([0, 100, 40, 230]), np.array([0, 100, 150, 200]), np.array([5, 100, 150, 230])):
        with pytest.raises(ValueError):
            persistent(ctx, x, y, z, bad, 4)
    b, gi, gd, _ = persistent(ctx, x, y, z, off, 4)  # a fresh batch with good offsets works
    assert b.query_stats()["queries"] == len(x)


@pytest.mark.parametrize("coord,sfc,periodic", [("f32", "morton", False), ("u32", "ph", True)])
def test_per_set_build_method(coord, sfc, periodic):
    """ft_batch_set_build_method(FT_METHOD_PERSISTENT): ft_batch_build through the per-set
    builds gives the launch sequence's trees, and the batched queries on them its rows."""
    ctx = ft.Context(coord, sfc, periodic=periodic)
    x, y, z, off = make_sets(coord, SIZES, seed=23)
    seq = ft.BatchedSets(ctx, len(x), len(SIZES))
    seq.build(off, x, y, z)
    per = ft.BatchedSets(ctx, len(x), len(SIZES))
    per.set_build_method("persistent")
    per.build(off, x, y, z)
    per.check()
    for s, n in enumerate(SIZES):
        if n == 0:
            continue
        got, want = per.tree(s).to_numpy(), seq.tree(s).to_numpy()
        for name in TREE_ARRAYS:
            assert np.array_equal(got[name].view(np.uint8), want[name].view(np.uint8)), (s, name)
    a = per.self_knn(32, method="fast")
    b = seq.self_knn(32, method="plain")
    torch.cuda.synchronize()
    assert torch.equal(a[0], b[0]) and torch.equal(a[1], b[1])


def test_default_build_knn_is_the_persistent_launch():
    """ft_batch_build_knn's default method runs the persistent launch for k <= 64 (the launch
    sequence with FT_METHOD_FAST); both give the plain batched traversal's rows."""
    ctx = ft.Context("f32", "morton")
    x, y, z, off = make_sets("f32", SIZES, seed=29)
    N, k = len(x), 16
    dx, dy, dz = (torch.as_tensor(a, device="cuda") for a in (x, y, z))
    doff = torch.as_tensor(off, device="cuda")
    ref = ft.BatchedSets(ctx, N, len(SIZES))
    ref.build(doff, dx, dy, dz)
    pi, pd = ref.self_knn(k, method="plain")
    for method in ("default", "fast"):
        b = ft.BatchedSets(ctx, N, len(SIZES))
        gi = torch.empty(N * k, dtype=torch.uint64, device="cuda")
        gd = torch.empty(N * k, dtype=torch.float64, device="cuda")
        b.build_knn(doff, dx, dy, dz, k, gi, gd, method=method)
        torch.cuda.synchronize()
        b.check()
        assert torch.equal(gi.view(N, k), pi) and torch.equal(gd.view(N, k), pd), method
