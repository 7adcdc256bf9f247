"""range_query with large radii (whole subtrees inside the ball are counted at once when the
row is full) and every query on a tree taller than 62 levels, where the reference's
traversal stack guard drops subtrees: GPU against the oracle, bit for bit."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")
if not torch.cuda.is_available():
    pytest.skip("no CUDA device", allow_module_level=True)

import fasttree_b200 as ft  # noqa: E402
from oracle import oracle as O  # noqa: E402
from tests.gpu_util import dist_bits, gen, radius, to_coord  # noqa: E402

CASES = [("f32", "morton", False, O.F32, O.MORTON), ("f64", "ph", False, O.F64, O.PEANO_HILBERT),
         ("u32", "ph", False, O.U32, O.PEANO_HILBERT), ("u64", "ph", False, O.U64, O.PEANO_HILBERT),
         ("u64", "ph", True, O.U64, O.PEANO_HILBERT), ("u32", "ph", True, O.U32, O.PEANO_HILBERT)]


@pytest.mark.parametrize("coord,sfc,per,oc,os_", CASES, ids=[f"{c[0]}-{c[1]}{'-per' if c[2] else ''}" for c in CASES])
@pytest.mark.parametrize("r_phys,max_per", [(8.0, 16), (30.0, 64), (60.0, 0), (200.0, 7)])
@pytest.mark.parametrize("walk", [0, 1, 2, 3], ids=["default-walk", "binary-walk", "warp-walk", "wide-walk"])
def test_range_large_radii_match_oracle(coord, sfc, per, oc, os_, r_phys, max_per, walk):
    n = 6000
    x, y, z = gen("clustered", n, oc, 12)
    ctx = ft.Context(coord, sfc, periodic=per)
    ctx.set_range_walk(walk)
    tree = ft.TreeSoA(ctx, n)
    ft.build_bvh(ctx, ft.particles(x, y, z), tree)
    opts = O.Options(oc, os_, per)
    ot = O.build_bvh(opts, x, y, z)
    rng = np.random.default_rng(4)
    q = [to_coord(a, oc) for a in rng.uniform(0, 100.0, (3, 700))]
    for d, a in enumerate((x, y, z)):
        q[d][:300] = a[:300]
    r0 = np.zeros(700, q[0].dtype)
    r1 = np.full(700, radius(r_phys, oc), q[0].dtype)
    r0[:100] = radius(r_phys / 4, oc)  # hollow shells too
    gr, gc = ft.range_query(ctx, tree, *q, r0, r1, max_per)
    orr, oc_ = O.range_query(opts, ot, *q, r0, r1, max_per)
    assert np.array_equal(gc.cpu().numpy(), oc_)
    if max_per:
        g, o = gr.cpu().numpy(), orr
        for i in range(700):
            m = min(int(oc_[i]), max_per)
            assert np.array_equal(g[i, :m], o[i, :m]), i


def tall_points():
    """63 points with single-bit Morton keys in the unit box (2^-i on one axis, i = 1..21) and
    16 copies of the origin: a chain of 63 splits over the duplicates' subtree."""
    pts = [(0.0, 0.0, 0.0)] * 16
    for axis in range(3):
        for i in range(1, 22):
            p = [0.0, 0.0, 0.0]
            p[axis] = 2.0 ** -i
            pts.append(tuple(p))
    a = np.array(pts, np.float64)
    return a[:, 0].copy(), a[:, 1].copy(), a[:, 2].copy()


def test_tree_taller_than_62_matches_oracle():
    x, y, z = tall_points()
    n = len(x)
    ctx = ft.Context("f64", "morton")
    opts = O.Options(O.F64, O.MORTON, False)
    box = ft.BoundingBox(0.0, 1.0, 0.0, 1.0, 0.0, 1.0)
    tree = ft.TreeSoA(ctx, n)
    ft.build_bvh(ctx, ft.particles(x, y, z), tree, bbox=box)
    ot = O.build_bvh(opts, x, y, z, bbox=box.array(O.F64))
    assert tree.height() > 62, tree.height()
    for k in (1, 5, 32):
        for method in ("plain", "fast"):
            gi, gd = ft.self_knn_query(ctx, tree, k, max_k=32, method=method)
            oi, od = O.self_knn(opts, ot, k)
            assert np.array_equal(gi.cpu().numpy(), oi), (k, method)
            assert np.array_equal(dist_bits(gd.cpu().numpy()), dist_bits(od)), (k, method)
    rng = np.random.default_rng(3)
    q = [np.concatenate([x, rng.uniform(0, 2.0 ** -10, 40)]) for _ in range(3)]
    for k, mk in ((4, 32), (40, 256)):
        for method in ("plain", "fast"):
            gi, gd = ft.knn_query(ctx, tree, *q, k, max_k=mk, method=method)
            oi, od = O.knn(opts, ot, *q, k, mk)
            assert np.array_equal(gi.cpu().numpy(), oi), (k, method)
            assert np.array_equal(dist_bits(gd.cpu().numpy()), dist_bits(od)), (k, method)
    for r, max_per in ((0.6, 0), (0.6, 5), (1e-4, 3), (2.0, 100)):
        r0 = np.zeros(len(q[0]))
        r1 = np.full(len(q[0]), r)
        gr, gc = ft.range_query(ctx, tree, *q, r0, r1, max_per)
        orr, oc_ = O.range_query(opts, ot, *q, r0, r1, max_per)
        assert np.array_equal(gc.cpu().numpy(), oc_), (r, max_per)
        if max_per:
            assert np.array_equal(gr.cpu().numpy(), orr), (r, max_per)


def tall_chain_unit(duplicates: bool = False):
    """The chain of tall_points() with one point at the origin (or its 16 copies), plus (1, .5,
    .5), (.5, 1, .5) and (.5, .5, 1), so that the computed bounding box is the unit box and the
    chain's keys stay single bits; each added point has one axis at the box maximum (cell 0
    there, the reference's wrap) and its key far from the chain's.  Height 63 (67 with the
    copies)."""
    x, y, z = tall_points()
    if not duplicates:
        x, y, z = x[15:], y[15:], z[15:]
    return np.append(x, [1.0, 0.5, 0.5]), np.append(y, [0.5, 1.0, 0.5]), np.append(z, [0.5, 0.5, 1.0])


def tall_with_background(n_bg: int, seed: int = 5, duplicates: bool = False):
    """Uniform background points in the unit box plus the tall chain of tall_chain_unit() at
    the box's corner: a tree of height > 62 whose deep part is confined to the corner."""
    cx, cy, cz = tall_chain_unit(duplicates)
    rng = np.random.default_rng(seed)
    bg = rng.uniform(0.0, 1.0, (3, n_bg))
    return (np.concatenate([bg[0], cx]), np.concatenate([bg[1], cy]), np.concatenate([bg[2], cz]))


@pytest.mark.parametrize("coord,oc", [("f64", O.F64), ("f32", O.F32)])
def test_tall_tree_fast_walk_replays_only_guarded_queries(coord, oc):
    """On a tree taller than 62 the fast walk answers the queries the reference's stack guard
    cannot reach and hands the others to the reference traversal: rows equal the oracle's
    (the reference's own drops included), and only a small part of the queries is replayed.
    External points near the corner at k = 48 are the case where the guard matters: there the
    reference's rows are not the nearest points (its stack drops part of the chain), and only
    the replay reproduces them."""
    x, y, z = (a.astype(O.NP_COORD[oc]) for a in tall_with_background(50_000))
    n = len(x)
    ctx = ft.Context(coord, "morton")
    opts = O.Options(oc, O.MORTON, False)
    box = ft.BoundingBox(0.0, 1.0, 0.0, 1.0, 0.0, 1.0)
    tree = ft.TreeSoA(ctx, n)
    ft.build_bvh(ctx, ft.particles(x, y, z), tree, bbox=box)
    ot = O.build_bvh(opts, x, y, z, bbox=box.array(oc))
    assert tree.height() > 62, tree.height()
    for k in (1, 8, 32, 64):
        gi, gd = ft.self_knn_query(ctx, tree, k, max_k=max(32, k), method="fast")
        replayed = len(ctx.replayed_queries())
        oi, od = O.self_knn(opts, ot, k)
        assert np.array_equal(gi.cpu().numpy(), oi), k
        assert np.array_equal(dist_bits(gd.cpu().numpy()), dist_bits(od)), k
        assert replayed < n // 20, (k, replayed)
    # external points: background-like queries and points near the corner
    rng = np.random.default_rng(8)
    q = [np.concatenate([rng.uniform(0, 1.0, 3000), rng.uniform(0, 2.0 ** -12, 200)]).astype(O.NP_COORD[oc])
         for _ in range(3)]
    for k, mk in ((16, 32), (48, 256)):
        gi, gd = ft.knn_query(ctx, tree, *q, k, max_k=mk, method="fast")
        replayed = len(ctx.replayed_queries())
        oi, od = O.knn(opts, ot, *q, k, mk)
        assert np.array_equal(gi.cpu().numpy(), oi), k
        assert np.array_equal(dist_bits(gd.cpu().numpy()), dist_bits(od)), k
        if k == 48:
            assert replayed > 0
    # a subset, twice the same leaves
    ids = np.arange(n - 200, n, dtype=np.int32)
    gi, gd = ft.self_knn_query_subset(ctx, tree, torch.from_numpy(ids).cuda(), 16, method="fast")
    oi, od = O.self_knn(opts, ot, 16, True, leaf_ids=ids)
    assert np.array_equal(gi.cpu().numpy(), oi)


def test_tall_set_in_a_batch():
    """A batch holding a set taller than 62 next to ordinary sets: every set's rows equal its
    own single-tree query's."""
    x0, y0, z0 = tall_chain_unit(duplicates=True)
    rng = np.random.default_rng(2)
    sets = [rng.uniform(0.0, 1.0, (3, m)) for m in (500, 3000)]
    tx, ty, tz = tall_with_background(4000, seed=9, duplicates=True)
    parts = [sets[0], np.stack([x0, y0, z0]), sets[1], np.stack([tx, ty, tz])]
    x = np.concatenate([p[0] for p in parts]).astype(np.float32)
    y = np.concatenate([p[1] for p in parts]).astype(np.float32)
    z = np.concatenate([p[2] for p in parts]).astype(np.float32)
    off = np.concatenate([[0], np.cumsum([p.shape[1] for p in parts])]).astype(np.int64)
    ctx = ft.Context("f32", "morton")
    b = ft.BatchedSets(ctx, len(x), len(parts))
    b.build(off, x, y, z)
    _, heights = b.set_info()
    assert heights.max() > 62
    for k in (4, 32):
        fi, fd = b.self_knn(k, method="fast")
        pi, pd = b.self_knn(k, method="plain")
        b.check()
        assert torch.equal(fi, pi) and torch.equal(fd, pd), k
        opts = O.Options(O.F32, O.MORTON, False)
        for s in range(len(parts)):
            a, e = int(off[s]), int(off[s + 1])
            ot = O.build_bvh(opts, x[a:e], y[a:e], z[a:e])
            oi, od = O.self_knn(opts, ot, k)
            assert np.array_equal(fi[a:e].cpu().numpy(), oi), (k, s)
            assert np.array_equal(dist_bits(fd[a:e].cpu().numpy()), dist_bits(od)), (k, s)


@pytest.mark.parametrize("coord,sfc,per,oc,os_", [("f64", "morton", False, O.F64, O.MORTON),
                                                   ("u64", "ph", True, O.U64, O.PEANO_HILBERT)],
                         ids=["f64-morton", "u64-ph-per"])
@pytest.mark.parametrize("walk", [0, 1], ids=["default-walk", "binary-walk"])
def test_range_counts_of_large_balls_match_oracle(coord, sfc, per, oc, os_, walk):
    """Balls of 10% of 400K points: long count-only tails after the rows fill up, counted from
    whole subtrees inside the shell; rows and counts bit for bit."""
    n = 400_000
    x, y, z = gen("uniform", n, oc, 5)
    ctx = ft.Context(coord, sfc, periodic=per)
    ctx.set_range_walk(walk)
    tree = ft.TreeSoA(ctx, n)
    ft.build_bvh(ctx, ft.particles(x, y, z), tree)
    opts = O.Options(oc, os_, per)
    ot = O.build_bvh(opts, x, y, z)
    q = [a[:160].copy() for a in (x, y, z)]
    r0 = np.zeros(160, q[0].dtype)
    r1 = np.full(160, radius(29.0, oc), q[0].dtype)
    r0[:40] = radius(10.0, oc)
    gr, gc = ft.range_query(ctx, tree, *q, r0, r1, 32)
    orr, oc_ = O.range_query(opts, ot, *q, r0, r1, 32)
    assert np.array_equal(gc.cpu().numpy(), oc_)
    g = gr.cpu().numpy()
    for i in range(160):
        m = min(int(oc_[i]), 32)
        assert np.array_equal(g[i, :m], orr[i, :m]), i


GROUP_CASES = CASES


@pytest.mark.parametrize("coord,sfc,per,oc,os_", GROUP_CASES,
                         ids=[f"{c[0]}-{c[1]}{'-per' if c[2] else ''}" for c in GROUP_CASES])
@pytest.mark.parametrize("r_phys,max_per", [(6.0, 16), (15.0, 0)])
@pytest.mark.parametrize("walk", [0, 4], ids=["default-walk", "group-counts"])
def test_range_group_counts_match_oracle(coord, sfc, per, oc, os_, r_phys, max_per, walk):
    """Dense queries with full rows: a warp's neighbouring queries count their shells together
    (nodes inside every query's shell counted whole, nodes beyond every ball skipped, the
    leaves between screened by a float filter and decided exactly where it cannot tell).
    Walk 4 takes every group that way, however spread out; the periodic cases put a cluster
    across the period's edge.  Rows and counts bit for bit against the oracle."""
    n = 40_000
    rng = np.random.default_rng(21)
    p = np.empty((3, n))
    n1, n2 = int(n * 0.45), int(n * 0.85)
    p[:, :n1] = rng.normal(25.0, 4.0, (3, n1))
    p[:, n1:n2] = rng.normal(75.0, 4.0, (3, n2 - n1))
    p[:, n2:] = rng.uniform(0.0, 100.0, (3, n - n2))
    if per:
        p = np.mod(p + 27.0, 100.0)  # the second cluster straddles the period's edge
    p = np.clip(p, 1e-4, 100.0 - 1e-4)
    x, y, z = (to_coord(a, oc) for a in p)
    ctx = ft.Context(coord, sfc, periodic=per)
    ctx.set_range_walk(walk)
    tree = ft.TreeSoA(ctx, n)
    ft.build_bvh(ctx, ft.particles(x, y, z), tree)
    opts = O.Options(oc, os_, per)
    ot = O.build_bvh(opts, x, y, z)
    nq = 3000
    pick = rng.choice(n, nq - 200, replace=False)
    q = [np.concatenate([a[pick], to_coord(rng.uniform(0, 100.0, 200), oc)]) for a in (x, y, z)]
    r0 = np.zeros(nq, q[0].dtype)
    r1 = np.full(nq, radius(r_phys, oc), q[0].dtype)
    r0[::4] = radius(r_phys / 3, oc)  # hollow shells for a quarter of the queries
    gr, gc = ft.range_query(ctx, tree, *q, r0, r1, max_per)
    orr, oc_ = O.range_query(opts, ot, *q, r0, r1, max_per)
    assert (oc_ > max(max_per, 1)).mean() > 0.5  # most rows are full: the counts come from the groups
    assert np.array_equal(gc.cpu().numpy(), oc_)
    if max_per:
        g = gr.cpu().numpy()
        for i in range(nq):
            m = min(int(oc_[i]), max_per)
            assert np.array_equal(g[i, :m], orr[i, :m]), i
