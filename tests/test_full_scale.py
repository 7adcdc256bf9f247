"""Parity at the benchmark workloads' full sizes.

The small parity tests (test_gpu_parity.py) cover every configuration on a few thousand
points.  Tall trees, thousands of radix-sort tiles in one decoupled look-back, genuine
distance ties and the batched sets' largest members only occur at full size, so this module
repeats the comparisons on the bench workloads themselves:

* 10M clustered uint64 points, Peano-Hilbert, periodic (the self-kNN headline workload):
  every tree array and the sorted keys against the oracle's build_bvh; self-kNN at k = 1, 32
  and 64 with both methods, the two methods equal on every row, and the oracle's rows on
  200,000 evenly spaced queries plus every query the fast walk replayed; range_query on a
  sample of queries.
* 1M external queries on 100K uniform float64 points, Morton, knn_query k = 64, MAXK = 256
  (SortedMergeHeap): both methods equal on every row, the oracle on 100,000 rows plus every
  replayed one.
* 4096 Plummer sets, float32, Morton (65.6M points): the batched build and self-kNN k = 32,
  both methods equal on every row, and 64 sets (the largest among them) against the oracle's
  own build_bvh + self_knn_query of that set alone.
* 50M clustered uint64 points, Peano-Hilbert, periodic (the large workload, a tree 65 levels
  tall, where the reference's stack guard can drop subtrees): self-kNN k = 64 on 200,000
  evenly spaced leaves, both methods equal and the oracle's rows.
* 2.2M clustered float64 and uint32 points: launches above 2^21 queries, where the walk
  flags equal heap keys for the replay instead of settling them; both methods equal on every
  row, the oracle on a sample plus every replayed query.

The reference tests pin results by brute force on the fly (test/test_self_knn.cpp:153-266);
the oracle here is the restatement pinned to the reference compiled from its own headers.
"""
import os

import numpy as np
import pytest

from oracle import oracle as O
from tests.gpu_util import assert_tree_equal, dist_bits

pytestmark = [pytest.mark.gpu, pytest.mark.slow]

torch = pytest.importorskip("torch")
if not torch.cuda.is_available():
    pytest.skip("no CUDA device", allow_module_level=True)

import fasttree_b200 as ft  # noqa: E402
from fasttree_b200 import datasets  # noqa: E402

SAMPLE = 200_000


def _threads():
    return O.set_threads(os.cpu_count() or 1)


def _rows_equal(a_idx, a_dist, b_idx, b_dist):
    """Two row sets equal bit for bit (indices and distance bits), on the device."""
    return torch.equal(a_idx, b_idx) and torch.equal(a_dist.view(torch.int64), b_dist.view(torch.int64))


def _sample_rows(n, replayed, count=SAMPLE):
    ids = np.unique(np.concatenate([np.linspace(0, n - 1, min(count, n)).astype(np.int64),
                                    np.asarray(replayed, np.int64)]))
    return ids.astype(np.int32)


def _export_keys(tree: "ft.TreeSoA", two_words: bool):
    """Sorted SFC keys of a built tree from its serialised form (ft_tree_export: 128-byte
    header, then min/max x/y/z, left/right children, parent, id, is_ghost, orig_idx, key low
    words, key high words, each on a 16-byte boundary)."""
    n = tree.num_leaves
    raw = tree.export().numpy()
    cs = 8 if tree.ctx.coord in (ft.F64, ft.U64) else 4
    off = 128
    sizes = [(2 * n - 1) * cs] * 6 + [(n - 1) * 4] * 2 + [(2 * n - 1) * 4] * 2 + [2 * n - 1] + [(2 * n - 1) * 4]
    for s in sizes:
        off += (s + 15) // 16 * 16
    lo = raw[off:off + 8 * n].view(np.uint64)
    off += (8 * n + 15) // 16 * 16
    hi = raw[off:off + 8 * n].view(np.uint64) if two_words else None
    return lo, hi


# -----------------------------------------------------------------------------------------
# 10M clustered uint64 points (the headline workload)
# -----------------------------------------------------------------------------------------
@pytest.fixture(scope="module")
def headline():
    n = 10_000_000
    x, y, z = datasets.clustered_fixed(n, n_spheres=20000, seed=2)
    ctx = ft.Context("u64", "ph", periodic=True)
    tree = ft.TreeSoA(ctx, n)
    ft.build_bvh(ctx, ft.particles(x, y, z), tree)
    _threads()
    opts = O.Options(O.U64, O.PEANO_HILBERT, True)
    ot = O.build_bvh(opts, x, y, z)
    yield dict(n=n, x=x, y=y, z=z, ctx=ctx, tree=tree, opts=opts, ot=ot)
    tree.free()
    torch.cuda.empty_cache()


def test_headline_tree_matches_oracle(headline):
    h = headline
    n, tree, ot = h["n"], h["tree"], h["ot"]
    assert_tree_equal(tree.to_numpy(), ot, n)
    # the sorted 126-bit keys (high and low words)
    lo, hi = _export_keys(tree, True)
    assert np.array_equal(lo, ot.sorted_lo[:n]) and np.array_equal(hi, ot.sorted_hi[:n])


@pytest.mark.parametrize("k", [1, 32, 64])
def test_headline_self_knn(headline, k):
    """Both methods give the same rows on all 10M queries; the oracle's on a 200K sample plus
    every query the fast walk replayed."""
    h = headline
    ctx, tree, n = h["ctx"], h["tree"], h["n"]
    mk = max(32, k)
    pi, pd = ft.self_knn_query(ctx, tree, k, max_k=mk, method="plain")
    fi, fd = torch.empty_like(pi), torch.empty_like(pd)
    ft.self_knn_query(ctx, tree, k, fi, fd, max_k=mk, method="fast")
    replayed = ctx.replayed_queries()
    ctx.check_device_status()
    assert _rows_equal(fi, fd, pi, pd), f"fast and plain rows differ at k={k}"
    ids = _sample_rows(n, replayed)
    oi, od = O.self_knn(h["opts"], h["ot"], k, True, leaf_ids=ids)
    t = torch.from_numpy(ids.astype(np.int64)).to(fi.device)
    gi, gd = fi.index_select(0, t).cpu().numpy(), fd.index_select(0, t).cpu().numpy()
    assert np.array_equal(gi, oi), f"k={k}: first differing sampled row {ids[np.argmax((gi != oi).any(1))]}"
    assert np.array_equal(dist_bits(gd), dist_bits(od))
    del pi, pd, fi, fd
    torch.cuda.empty_cache()


def test_headline_range_sample(headline):
    """range_query (r_max = 2e-3 of the box, 512 results per row) on 1,000 of the particles,
    against the oracle: counts and every written result."""
    h = headline
    rng = np.random.default_rng(21)
    q = np.sort(rng.choice(h["n"], 1000, replace=False))
    qx, qy, qz = h["x"][q], h["y"][q], h["z"][q]
    r0 = np.zeros(len(q), np.uint64)
    r1 = np.full(len(q), int(2e-3 * 2 ** 40), np.uint64)
    gr, gc = ft.range_query(h["ctx"], h["tree"], qx, qy, qz, r0, r1, 512)
    orr, oc = O.range_query(h["opts"], h["ot"], qx, qy, qz, r0, r1, 512)
    gc = gc.cpu().numpy()
    assert np.array_equal(gc, oc)
    gr = gr.cpu().numpy().reshape(len(q), 512)
    for i in range(len(q)):
        m = min(oc[i], 512)
        assert np.array_equal(gr[i, :m], orr[i, :m]), i


# -----------------------------------------------------------------------------------------
# 1M external queries, knn_query k = 64 with MAXK = 256
# -----------------------------------------------------------------------------------------
def test_external_knn_1m():
    x, y, z = datasets.uniform(100_000, seed=1)
    qx, qy, qz = datasets.external_queries(x, y, z, 1_000_000, seed=3)
    ctx = ft.Context("f64", "morton")
    tree = ft.TreeSoA(ctx, len(x))
    ft.build_bvh(ctx, ft.particles(x, y, z), tree)
    dq = [torch.from_numpy(a).cuda() for a in (qx, qy, qz)]
    k, mk = 64, 256
    pi, pd = ft.knn_query(ctx, tree, *dq, k, max_k=mk, method="plain")
    fi, fd = torch.empty_like(pi), torch.empty_like(pd)
    ft.knn_query(ctx, tree, *dq, k, fi, fd, max_k=mk, method="fast")
    replayed = ctx.replayed_queries()
    assert _rows_equal(fi, fd, pi, pd)
    _threads()
    opts = O.Options(O.F64, O.MORTON)
    ot = O.build_bvh(opts, x, y, z)
    ids = _sample_rows(len(qx), replayed, 100_000)
    oi, od = O.knn(opts, ot, qx[ids], qy[ids], qz[ids], k, mk)
    t = torch.from_numpy(ids.astype(np.int64)).cuda()
    assert np.array_equal(fi.index_select(0, t).cpu().numpy(), oi)
    assert np.array_equal(dist_bits(fd.index_select(0, t).cpu().numpy()), dist_bits(od))


# -----------------------------------------------------------------------------------------
# 4096 batched Plummer sets
# -----------------------------------------------------------------------------------------
def test_batched_sets_4096():
    sizes = datasets.batched_set_sizes(4096, seed=4)
    x, y, z, off = datasets.batched_sets(sizes=sizes, seed=4)
    N, S, k = len(x), len(sizes), 32
    ctx = ft.Context("f32", "morton")
    b = ft.BatchedSets(ctx, N, S)
    b.build(off, x, y, z)
    pi, pd = b.self_knn(k, method="plain")
    fi, fd = torch.empty_like(pi), torch.empty_like(pd)
    b.self_knn(k, method="fast", results=fi, result_dists=fd)
    b.check()
    assert _rows_equal(fi, fd, pi, pd)
    # the largest set and 63 others spread over the set numbers, each against its own
    # reference build and query
    chosen = sorted(set([int(np.argmax(sizes))] + list(np.linspace(0, S - 1, 63).astype(int))))
    _threads()
    opts = O.Options(O.F32, O.MORTON)
    for s in chosen:
        a, e = int(off[s]), int(off[s + 1])
        ot = O.build_bvh(opts, x[a:e], y[a:e], z[a:e])
        assert_tree_equal(b.tree(s).to_numpy(), ot, e - a)
        oi, od = O.self_knn(opts, ot, k, True)
        assert np.array_equal(fi[a:e].cpu().numpy(), oi), s
        assert np.array_equal(dist_bits(fd[a:e].cpu().numpy()), dist_bits(od)), s
    del b, pi, pd, fi, fd
    torch.cuda.empty_cache()


# -----------------------------------------------------------------------------------------
# 50M clustered uint64 points (a tree taller than 62 levels)
# -----------------------------------------------------------------------------------------
def test_large_tall_tree_sample():
    n, k = 50_000_000, 64
    x, y, z = datasets.clustered_fixed(n, n_spheres=100_000, seed=5)
    ctx = ft.Context("u64", "ph", periodic=True)
    tree = ft.TreeSoA(ctx, n)
    ft.build_bvh(ctx, ft.particles(x, y, z), tree)
    assert tree.height() > 62, tree.height()
    ids = np.linspace(0, n - 1, SAMPLE).astype(np.int32)
    t = torch.from_numpy(ids).cuda()
    fi, fd = ft.self_knn_query_subset(ctx, tree, t, k, max_k=k, method="fast")
    replayed = len(ctx.replayed_queries())
    pi, pd = ft.self_knn_query_subset(ctx, tree, t, k, max_k=k, method="plain")
    ctx.check_device_status()
    assert _rows_equal(fi, fd, pi, pd)
    assert replayed < SAMPLE // 10, replayed  # the guard hands only some queries to the replay
    _threads()
    opts = O.Options(O.U64, O.PEANO_HILBERT, True)
    ot = O.build_bvh(opts, x, y, z)
    oi, od = O.self_knn(opts, ot, k, True, leaf_ids=ids)
    gi, gd = fi.cpu().numpy(), fd.cpu().numpy()
    assert np.array_equal(gi, oi), f"first differing sampled row {ids[np.argmax((gi != oi).any(1))]}"
    assert np.array_equal(dist_bits(gd), dist_bits(od))
    del tree, fi, fd, pi, pd
    torch.cuda.empty_cache()


# -----------------------------------------------------------------------------------------
# launches above 2^21 queries keep the flag-only keyed heap: float64 and uint32 coordinates
# -----------------------------------------------------------------------------------------
@pytest.mark.parametrize("coord,sfc,per,oc,os_,k", [("f64", "morton", False, O.F64, O.MORTON, 16),
                                                    ("u32", "ph", True, O.U32, O.PEANO_HILBERT, 32)],
                         ids=["f64-k16", "u32-per-k32"])
def test_large_launch_keyed_heap(coord, sfc, per, oc, os_, k):
    """Self-kNN of 2.2M points (a launch above the 2^21 queries below which the walk settles
    the k-th key exactly): equal heap keys go to the replay; every row equal to the plain
    traversal's, and the oracle's on a sample plus every replayed query."""
    from tests.gpu_util import gen
    n = 2_200_000
    x, y, z = gen("clustered", n, oc, 31)
    ctx = ft.Context(coord, sfc, periodic=per)
    tree = ft.TreeSoA(ctx, n)
    ft.build_bvh(ctx, ft.particles(x, y, z), tree)
    pi, pd = ft.self_knn_query(ctx, tree, k, max_k=32, method="plain")
    fi, fd = torch.empty_like(pi), torch.empty_like(pd)
    ft.self_knn_query(ctx, tree, k, fi, fd, max_k=32, method="fast")
    replayed = ctx.replayed_queries()
    ctx.check_device_status()
    assert _rows_equal(fi, fd, pi, pd)
    _threads()
    opts = O.Options(oc, os_, per)
    ot = O.build_bvh(opts, x, y, z)
    ids = _sample_rows(n, replayed, 100_000)
    oi, od = O.self_knn(opts, ot, k, True, leaf_ids=ids)
    t = torch.from_numpy(ids.astype(np.int64)).to(fi.device)
    assert np.array_equal(fi.index_select(0, t).cpu().numpy(), oi)
    assert np.array_equal(dist_bits(fd.index_select(0, t).cpu().numpy()), dist_bits(od))
    del tree, pi, pd, fi, fd
    torch.cuda.empty_cache()
