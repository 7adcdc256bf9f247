"""ft_self_knn with host output buffers: the leaves are walked in chunks and each chunk's
rows are copied out while the next is walked.  The rows must equal those written to device
memory, for pinned and pageable buffers, the full query and subsets, fast and plain."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")
if not torch.cuda.is_available():
    pytest.skip("no CUDA device", allow_module_level=True)

import fasttree_b200 as ft  # noqa: E402
from fasttree_b200 import datasets  # noqa: E402


@pytest.mark.parametrize("pinned", [True, False])
@pytest.mark.parametrize("method", ["plain", "fast"])
def test_host_rows_equal_device_rows(pinned, method):
    n, k = 700_000, 16  # several chunks of 2^18 leaves
    x, y, z = datasets.clustered_fixed(n, n_spheres=1400, seed=6)
    ctx = ft.Context("u64", "ph", periodic=True)
    tree = ft.TreeSoA(ctx, n)
    ft.build_bvh(ctx, ft.particles(x, y, z), tree)
    di, dd = ft.self_knn_query(ctx, tree, k, method=method)
    torch.cuda.synchronize()
    hi = torch.empty(n * k, dtype=torch.uint64)
    hd = torch.empty(n * k, dtype=torch.uint64)
    if pinned:
        hi, hd = hi.pin_memory(), hd.pin_memory()
    ri, rd = ft.self_knn_query(ctx, tree, k, hi, hd, method=method)
    torch.cuda.synchronize()
    assert torch.equal(ri, di.cpu()) and torch.equal(rd, dd.cpu())
    # subset of leaf ids (device array), outputs to host
    ids = torch.randperm(n, device="cuda")[:300_001].to(torch.int32)
    si, sd = ft.self_knn_query_subset(ctx, tree, ids, k, method=method)
    hi2 = torch.empty(len(ids) * k, dtype=torch.uint64)
    hd2 = torch.empty(len(ids) * k, dtype=torch.uint64)
    ri2, rd2 = ft.self_knn_query_subset(ctx, tree, ids, k, hi2, hd2, method=method)
    torch.cuda.synchronize()
    assert torch.equal(ri2, si.cpu()) and torch.equal(rd2, sd.cpu())


def test_mixed_placement_is_rejected():
    ctx = ft.Context("f64", "morton")
    x, y, z = datasets.uniform(1000, seed=1)
    tree = ft.TreeSoA(ctx, 1000)
    ft.build_bvh(ctx, ft.particles(x, y, z), tree)
    with pytest.raises(ValueError):
        ft.self_knn_query(ctx, tree, 4, torch.empty(4000, dtype=torch.uint64),
                          torch.empty(4000, dtype=torch.float64, device="cuda"))


def test_sharded_rows_concatenate_to_the_full_query():
    from fasttree_b200.sharding import sharded_self_knn
    n, k = 300_000, 32
    x, y, z = datasets.clustered_fixed(n, n_spheres=600, seed=7)
    ctx = ft.Context("u64", "ph", periodic=True)
    tree = ft.TreeSoA(ctx, n)
    ft.build_bvh(ctx, ft.particles(x, y, z), tree)
    fi, fd = ft.self_knn_query(ctx, tree, k, method="fast")
    torch.cuda.synchronize()
    costs = np.random.default_rng(1).lognormal(0, 1, n)
    for world, c in ((3, None), (4, costs)):
        parts = [sharded_self_knn(ctx, tree, k, r, world, costs=c) for r in range(world)]
        torch.cuda.synchronize()
        assert parts[0][0] == 0 and parts[-1][1] == n
        assert torch.equal(torch.cat([p[2] for p in parts]), fi)
        assert torch.equal(torch.cat([p[3] for p in parts]), fd)
