"""Fast knn_query (method "fast") of external query points: bit-identical to the plain traversal
with each heap tier (register heap for k <= 32 or MAXK <= 32, SortedMergeHeap above), on
the learned-bound workload's shape (uniform float64 tree, half uniform / half jittered
queries), clustered and duplicate-heavy trees, queries outside the box, and trees whose keys
came from the caller (no seeding window)."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")
if not torch.cuda.is_available():
    pytest.skip("no CUDA device", allow_module_level=True)

import fasttree_b200 as ft  # noqa: E402
from fasttree_b200 import datasets  # noqa: E402
from oracle import oracle as O  # noqa: E402
from tests.gpu_util import dist_bits, gen, to_coord  # noqa: E402


def both(ctx, tree, q, k, max_k, variant=0):
    pi, pd = ft.knn_query(ctx, tree, *q, k, max_k=max_k, method="plain")
    fi, fd = ft.knn_query(ctx, tree, *q, k, max_k=max_k, method="fast", variant=variant)
    torch.cuda.synchronize()
    return (pi, pd), (fi, fd), ctx.query_stats()


@pytest.mark.parametrize("variant", [0, 5])
@pytest.mark.parametrize("k,max_k", [(1, 32), (16, 32), (32, 32), (33, 64), (48, 256), (64, 256), (64, 128)])
def test_external_queries_uniform_f64(k, max_k, variant):
    x, y, z = datasets.uniform(100_000, seed=1)
    ctx = ft.Context("f64", "morton")
    tree = ft.TreeSoA(ctx, len(x))
    ft.build_bvh(ctx, ft.particles(x, y, z), tree)
    qx, qy, qz = datasets.external_queries(x, y, z, 50_000, seed=3)
    (pi, pd), (fi, fd), st = both(ctx, tree, (qx, qy, qz), k, max_k, variant)
    assert torch.equal(pi, fi) and torch.equal(pd, fd)
    assert st["replayed"] < 0.05 * len(qx)


@pytest.mark.parametrize("coord,sfc,per", [("u64", "ph", True), ("u32", "ph", False), ("f32", "ph", False),
                                           ("f32", "morton", False)])
@pytest.mark.parametrize("kind", ["clustered", "degenerate"])
@pytest.mark.parametrize("variant", [0, 5])
def test_external_queries_hard_sets(coord, sfc, per, kind, variant):
    oc = {"u64": O.U64, "u32": O.U32, "f32": O.F32}[coord]
    x, y, z = gen(kind, 40_000, oc, 5)
    ctx = ft.Context(coord, sfc, periodic=per)
    tree = ft.TreeSoA(ctx, len(x))
    ft.build_bvh(ctx, ft.particles(x, y, z), tree)
    rng = np.random.default_rng(2)
    q = [to_coord(a, oc) for a in rng.uniform(0, 100.0, (3, 6000))]
    for d, a in enumerate((x, y, z)):  # a third exactly on particles (exact ties, duplicates)
        q[d][:2000] = a[rng.integers(0, len(x), 2000)]
    for k, max_k in ((8, 32), (32, 256), (64, 256)):
        (pi, pd), (fi, fd), _ = both(ctx, tree, q, k, max_k, variant)
        assert torch.equal(pi, fi) and torch.equal(pd, fd), (k, max_k)


def test_queries_outside_the_box_and_caller_keys():
    ctx = ft.Context("f32", "morton")
    x, y, z = gen("clustered", 20_000, O.F32, 4)
    tree = ft.TreeSoA(ctx, len(x))
    ft.build_bvh(ctx, ft.particles(x, y, z), tree)
    rng = np.random.default_rng(8)
    q = [rng.uniform(-50.0, 150.0, 3000).astype(np.float32) for _ in range(3)]
    for k, max_k in ((16, 32), (40, 256)):
        (pi, pd), (fi, fd), _ = both(ctx, tree, q, k, max_k)
        assert torch.equal(pi, fi) and torch.equal(pd, fd)
    # a tree from caller keys has no seeding window: still exact
    keys = ft.sfc_encode(ctx, x, y, z, bbox=ft.compute_bbox(ctx, x, y, z))
    t2 = ft.TreeSoA(ctx, len(x))
    ft.build_bvh(ctx, ft.particles(x, y, z), t2, key=keys)
    (pi, pd), (fi, fd), _ = both(ctx, t2, q, 16, 32)
    assert torch.equal(pi, fi) and torch.equal(pd, fd)


def test_against_oracle_with_original_indices():
    ctx = ft.Context("f64", "ph", return_orig_indices=True)
    opts = O.Options(O.F64, O.PEANO_HILBERT, False, True)
    x, y, z = gen("clustered", 4000, O.F64, 6)
    tree = ft.TreeSoA(ctx, len(x))
    ft.build_bvh(ctx, ft.particles(x, y, z), tree)
    ot = O.build_bvh(opts, x, y, z)
    qx, qy, qz = (to_coord(a, O.F64) for a in np.random.default_rng(1).uniform(0, 100.0, (3, 500)))
    for k, max_k in ((12, 32), (50, 256)):
        gi, gd = ft.knn_query(ctx, tree, qx, qy, qz, k, max_k=max_k, method="fast")
        oi, od = O.knn(opts, ot, qx, qy, qz, k, max_k)
        assert np.array_equal(gi.cpu().numpy(), oi)
        assert np.array_equal(dist_bits(gd.cpu().numpy()), dist_bits(od))
