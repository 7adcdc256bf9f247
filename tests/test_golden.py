"""Golden fixtures produced by the reference's own code (tests/golden/make_golden.py).

CPU: the oracle reproduces every fixture bit for bit (this pins the oracle even where the
reference sources are absent).  GPU: the CUDA library reproduces every fixture through the
C ABI.
"""
import glob
import os

import numpy as np
import pytest

from oracle import oracle as O

HERE = os.path.dirname(os.path.abspath(__file__))
FIXTURES = sorted(glob.glob(os.path.join(HERE, "golden", "*.npz")))
IDS = [os.path.basename(f)[:-4] for f in FIXTURES]
TREE = ("min_x", "max_x", "min_y", "max_y", "min_z", "max_z", "left_child", "right_child", "parent", "id",
        "is_ghost", "orig_idx")


def same(a, b):
    a, b = np.asarray(a), np.asarray(b)
    return a.shape == b.shape and np.array_equal(a.view(np.uint8), b.view(np.uint8))


def load(path):
    g = dict(np.load(path))
    c = [int(v) for v in g["config"]]
    return g, O.Options(c[0], c[1], bool(c[2]), bool(c[3]))


def test_fixtures_present():
    assert len(FIXTURES) == 10


@pytest.mark.parametrize("path", FIXTURES, ids=IDS)
def test_oracle_reproduces_golden(path):
    g, opts = load(path)
    t = O.build_bvh(opts, g["x"], g["y"], g["z"])
    for k in TREE:
        assert same(getattr(t, k), g["tree_" + k]), k
    assert same(t.sorted_hi, g["sorted_hi"]) and same(t.sorted_lo, g["sorted_lo"])
    i, d = O.self_knn(opts, t, 16, True)
    assert same(i, g["self16_idx"]) and same(d, g["self16_dist"])
    i, d = O.self_knn(opts, t, 40, False, leaf_ids=g["subset_ids"])
    assert same(i, g["sub40_idx"]) and same(d, g["sub40_dist"])
    i, d = O.knn(opts, t, g["qx"], g["qy"], g["qz"], 5, 256)
    assert same(i, g["knn5_idx"]) and same(d, g["knn5_dist"])
    i, d = O.knn(opts, t, g["qx"], g["qy"], g["qz"], 48, 64)
    assert same(i, g["knn48_idx"]) and same(d, g["knn48_dist"])
    r, c = O.range_query(opts, t, g["qx"], g["qy"], g["qz"], g["rmin"], g["rmax"], 12)
    assert same(c, g["range_cnt"])
    for q in range(len(c)):
        m = min(int(c[q]), 12)
        assert same(r[q, :m], g["range_res"][q, :m])


@pytest.mark.gpu
@pytest.mark.parametrize("path", FIXTURES, ids=IDS)
@pytest.mark.parametrize("method", ["plain", "fast"])
def test_gpu_reproduces_golden(path, method):
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    import fasttree_b200 as ft
    g, opts = load(path)
    names = {O.F32: "f32", O.F64: "f64", O.U32: "u32", O.U64: "u64"}
    ctx = ft.Context(names[opts.coord], opts.sfc, periodic=opts.periodic, return_orig_indices=opts.return_orig)
    n = len(g["x"])
    tree = ft.TreeSoA(ctx, n)
    ft.build_bvh(ctx, ft.particles(g["x"], g["y"], g["z"]), tree)
    a = tree.to_numpy()
    for k in TREE:
        assert same(a[k], g["tree_" + k]), k
    i, d = ft.self_knn_query(ctx, tree, 16, exclude_self=True, method=method)
    torch.cuda.synchronize()
    assert same(i.cpu().numpy(), g["self16_idx"]) and same(d.cpu().numpy(), g["self16_dist"])
    ids = torch.from_numpy(g["subset_ids"]).cuda()
    i, d = ft.self_knn_query_subset(ctx, tree, ids, 40, exclude_self=False, method=method)
    torch.cuda.synchronize()
    assert same(i.cpu().numpy(), g["sub40_idx"]) and same(d.cpu().numpy(), g["sub40_dist"])
    i, d = ft.knn_query(ctx, tree, g["qx"], g["qy"], g["qz"], 5, max_k=256, method=method)
    assert same(i.cpu().numpy(), g["knn5_idx"]) and same(d.cpu().numpy(), g["knn5_dist"])
    i, d = ft.knn_query(ctx, tree, g["qx"], g["qy"], g["qz"], 48, max_k=64, method=method)
    assert same(i.cpu().numpy(), g["knn48_idx"]) and same(d.cpu().numpy(), g["knn48_dist"])
    r, c = ft.range_query(ctx, tree, g["qx"], g["qy"], g["qz"], g["rmin"], g["rmax"], 12)
    c = c.cpu().numpy()
    r = r.cpu().numpy()
    assert same(c, g["range_cnt"])
    for q in range(len(c)):
        m = min(int(c[q]), 12)
        assert same(r[q, :m], g["range_res"][q, :m])
