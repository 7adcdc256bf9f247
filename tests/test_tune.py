"""Autotuner (ft_tune_*): per-shape choices of the build's sort tile and of the fast walk's
variant, seeding window and block shape.  Every candidate returns the same rows, so the tests
check that (the tuners verify it themselves on the device and fail otherwise), that the
choice is kept for the shape and taken by later default calls, and that the rows stay the
oracle's."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")
if not torch.cuda.is_available():
    pytest.skip("no CUDA device", allow_module_level=True)

import fasttree_b200 as ft  # noqa: E402
from fasttree_b200 import datasets  # noqa: E402
from oracle import oracle as O  # noqa: E402
from tests.gpu_util import dist_bits, gen  # noqa: E402


@pytest.mark.parametrize("coord,sfc,per,oc,os_", [("u64", "ph", True, O.U64, O.PEANO_HILBERT),
                                                  ("f32", "morton", False, O.F32, O.MORTON),
                                                  ("f64", "ph", False, O.F64, O.PEANO_HILBERT)])
def test_tuned_self_knn_keeps_the_rows(coord, sfc, per, oc, os_):
    n = 120_000
    x, y, z = gen("clustered", n, oc, 23)
    ctx = ft.Context(coord, sfc, periodic=per)
    tree = ft.TreeSoA(ctx, n)
    ft.build_bvh(ctx, ft.particles(x, y, z), tree)
    opts = O.Options(oc, os_, per)
    ot = O.build_bvh(opts, x, y, z)
    for k in (1, 16, 32, 40):
        pi, pd = ft.self_knn_query(ctx, tree, k, max_k=max(32, k), method="plain")
        pi, pd = pi.clone(), pd.clone()
        r = ft.tune_self_knn(ctx, tree, k)
        assert r["candidates"] >= 5 and r["best_ms"] > 0 and r["best_ms"] <= r["default_ms"]
        assert r["walk_variant"] in (2, 4, 5) and r["block_threads"] in (32, 64)
        # the default call now takes the tuned configuration
        fi, fd = ft.self_knn_query(ctx, tree, k, max_k=max(32, k))
        torch.cuda.synchronize()
        assert torch.equal(fi, pi) and torch.equal(fd, pd), k
        ids = np.arange(0, n, 97, dtype=np.int32)
        oi, od = O.self_knn(opts, ot, k, True, leaf_ids=ids)
        t = torch.from_numpy(ids.astype(np.int64)).cuda()
        assert np.array_equal(fi.index_select(0, t).cpu().numpy(), oi)
        assert np.array_equal(dist_bits(fd.index_select(0, t).cpu().numpy()), dist_bits(od))
    ft.tune_reset(ctx)


@pytest.mark.parametrize("coord,sfc,per,oc,os_", [("u64", "ph", True, O.U64, O.PEANO_HILBERT),
                                                  ("f32", "morton", False, O.F32, O.MORTON)])
def test_tuned_build_keeps_the_tree(coord, sfc, per, oc, os_):
    n = 300_000
    x, y, z = gen("clustered", n, oc, 29)
    ctx = ft.Context(coord, sfc, periodic=per)
    tree = ft.TreeSoA(ctx, n)
    r = ft.tune_build(ctx, ft.particles(x, y, z), tree)
    assert r["sort_items"] in (8, 12, 16, 20) and r["candidates"] >= 3
    opts = O.Options(oc, os_, per)
    ot = O.build_bvh(opts, x, y, z)
    from tests.gpu_util import assert_tree_equal
    assert_tree_equal(tree.to_numpy(), ot, n)
    # a later build of the same shape takes the tuned tile and gives the same tree
    t2 = ft.TreeSoA(ctx, n)
    ft.build_bvh(ctx, ft.particles(x, y, z), t2)
    assert_tree_equal(t2.to_numpy(), ot, n)


def test_tuned_batch_keeps_the_rows():
    sizes = datasets.batched_set_sizes(300, seed=21, median=1500.0)
    x, y, z, off = datasets.batched_sets(sizes=sizes, seed=21)
    ctx = ft.Context("f32", "morton")
    b = ft.BatchedSets(ctx, len(x), len(sizes))
    b.build(off, x, y, z)
    pi, pd = b.self_knn(32, method="plain")
    pi, pd = pi.clone(), pd.clone()
    r = b.tune(32)
    assert r["candidates"] >= 3 and r["best_ms"] <= r["default_ms"]
    fi, fd = b.self_knn(32)
    b.check()
    assert torch.equal(fi, pi) and torch.equal(fd, pd)


def test_tuner_rejections():
    ctx = ft.Context("f64", "morton")
    x, y, z = gen("uniform", 1000, O.F64, 3)
    tree = ft.TreeSoA(ctx, 1000)
    ft.build_bvh(ctx, ft.particles(x, y, z), tree)
    with pytest.raises(ValueError):
        ft.tune_self_knn(ctx, tree, 65)  # the fast walk serves k <= 64
    with pytest.raises(ValueError):
        ft.tune_self_knn(ctx, tree, 0)


def test_build_stage_profile():
    """ft_set_build_profiling / ft_get_build_profile: every stage of a build timed on its
    stream; the stages add up to the whole build; a context without a profiled build says so."""
    ctx = ft.Context("u64", "ph", periodic=True)
    x, y, z = datasets.clustered_fixed(500_000, n_spheres=1000, seed=2)
    tree = ft.TreeSoA(ctx, len(x))
    with pytest.raises(ValueError):
        ctx.build_profile()
    ctx.profile_builds(True)
    ft.build_bvh(ctx, ft.particles(x, y, z), tree)
    prof = ctx.build_profile()
    stages = [prof[k] for k in ("bbox_ms", "encode_ms", "sort_ms", "gather_ms", "topology_ms", "refit_ms",
                                "records_ms")]
    assert all(v >= 0.0 for v in stages) and prof["total_ms"] > 0.0
    assert abs(sum(stages) - prof["total_ms"]) < 0.05 * prof["total_ms"] + 0.01
    ctx.profile_builds(False)
