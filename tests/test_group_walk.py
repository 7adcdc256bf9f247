"""The group walk (fast walk variant 5): a warp's 32 queries walk the tree once together,
pruning by the distance from the group's bounding box, and every lane tests every kept leaf.
Its output must equal the reference traversal's bit for bit in every configuration, with
and without ties, for subsets, original indices, per-query bounds, and queries whose heaps
cannot be seeded full (those warps take the 4-wide walk)."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")
if not torch.cuda.is_available():
    pytest.skip("no CUDA device", allow_module_level=True)

import fasttree_b200 as ft  # noqa: E402
from oracle import oracle as O  # noqa: E402
from tests.gpu_util import gen  # noqa: E402

CFGS = [("u64", "ph", True, O.U64), ("u64", "ph", False, O.U64), ("u32", "ph", True, O.U32),
        ("u32", "ph", False, O.U32), ("f32", "morton", False, O.F32), ("f64", "ph", False, O.F64)]


def _tree(coord, sfc, per, oc, kind, n, seed, ret_orig=False):
    x, y, z = gen(kind, n, oc, seed)
    ctx = ft.Context(coord, sfc, periodic=per, return_orig_indices=ret_orig)
    tree = ft.TreeSoA(ctx, n)
    ft.build_bvh(ctx, ft.particles(x, y, z), tree)
    return ctx, tree


def _same(a, b):
    torch.cuda.synchronize()
    return torch.equal(a[0], b[0]) and torch.equal(a[1], b[1])


@pytest.mark.parametrize("coord,sfc,per,oc", CFGS, ids=[f"{c[0]}-{c[1]}{'-per' if c[2] else ''}" for c in CFGS])
@pytest.mark.parametrize("kind", ["clustered", "uniform", "degenerate"])
def test_group_walk_equals_reference_traversal(coord, sfc, per, oc, kind):
    ctx, tree = _tree(coord, sfc, per, oc, kind, 120_000, 7)
    for k in (5, 16, 32, 64):
        mk = max(32, k)
        for excl in (True, False):
            plain = ft.self_knn_query(ctx, tree, k, exclude_self=excl, max_k=mk, method="plain")
            plain = (plain[0].clone(), plain[1].clone())
            group = ft.self_knn_query(ctx, tree, k, exclude_self=excl, max_k=mk, method="fast", variant=5)
            assert _same(plain, group), (k, excl)


@pytest.mark.parametrize("coord,sfc,per,oc", [CFGS[0], CFGS[4]], ids=["u64-ph-per", "f32-morton"])
def test_group_walk_subsets_orig_and_bounds(coord, sfc, per, oc):
    n, k = 80_000, 24
    ctx, tree = _tree(coord, sfc, per, oc, "clustered", n, 3, ret_orig=True)
    rng = np.random.default_rng(4)
    for ids in (np.sort(rng.choice(n, 5000, replace=False)), rng.choice(n, 5000, replace=False),
                np.arange(n - 37, n), np.array([0, 1, 2])):
        t = torch.from_numpy(ids.astype(np.int32)).cuda()
        a = ft.self_knn_query_subset(ctx, tree, t, k, max_k=32, method="plain")
        a = (a[0].clone(), a[1].clone())
        b = ft.self_knn_query_subset(ctx, tree, t, k, max_k=32, method="fast", variant=5)
        assert _same(a, b), len(ids)
    # per-query bounds: exact (bound at or above the k-th distance), too small, zero
    plain = ft.self_knn_query(ctx, tree, k, max_k=32, method="plain")
    plain = (plain[0].clone(), plain[1].clone())
    kth = plain[1][:, k - 1].contiguous()
    half = (kth.to(torch.int64) // 2).to(kth.dtype) if kth.dtype != torch.float64 else kth * 0.5
    for bound in (kth, half, torch.zeros_like(kth)):
        got = ft.self_knn_query_bounded(ctx, tree, k, bound.contiguous(), max_k=32, variant=5)
        assert _same(plain, got)


def test_group_walk_small_trees_fall_back():
    # trees too small to seed a full heap take the 4-wide walk inside the same launch
    for n in (2, 3, 17, 40, 65, 66, 200):
        ctx, tree = _tree("u64", "ph", True, O.U64, "uniform", n, n)
        for k in (8, 32):
            a = ft.self_knn_query(ctx, tree, k, max_k=32, method="plain")
            a = (a[0].clone(), a[1].clone())
            b = ft.self_knn_query(ctx, tree, k, max_k=32, method="fast", variant=5)
            assert _same(a, b), (n, k)
