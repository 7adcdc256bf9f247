"""Tree serialisation (ft_tree_export / ft_tree_import): a tree written out and read back --
through host bytes, a device buffer or a file -- has the same arrays as the original, and
every query on it returns the original's rows, bit for bit."""
import numpy as np
import pytest

from oracle import oracle as O
from tests.gpu_util import NAMES, gen

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")
if not torch.cuda.is_available():
    pytest.skip("no CUDA device", allow_module_level=True)

import fasttree_b200 as ft  # noqa: E402

CASES = [(O.U64, "ph", True), (O.U64, "ph", False), (O.U32, "ph", True), (O.F32, "morton", False),
         (O.F64, "ph", False)]
IDS = [f"{NAMES[c]}-{s}{'-per' if p else ''}" for c, s, p in CASES]


def _same_tree(a, b):
    ta, tb = a.to_numpy(), b.to_numpy()
    for name in ta:
        assert np.array_equal(ta[name].view(np.uint8), tb[name].view(np.uint8)), name
    assert a.height() == b.height()


def _same_queries(ctx, a, b, coord):
    for k, mk, method in ((8, 32, "fast"), (32, 32, "plain"), (40, 64, "fast")):
        ia, da = ft.self_knn_query(ctx, a, k, max_k=mk, method=method)
        ia, da = ia.clone(), da.clone()
        ib, db = ft.self_knn_query(ctx, b, k, max_k=mk, method=method)
        torch.cuda.synchronize()
        assert torch.equal(ia, ib) and torch.equal(da, db), (k, method)
    qx, qy, qz = gen("uniform", 700, coord, 5)
    ia, da = ft.knn_query(ctx, a, qx, qy, qz, 16, method="fast")
    ib, db = ft.knn_query(ctx, b, qx, qy, qz, 16, method="fast")
    assert torch.equal(ia, ib) and torch.equal(da, db)


@pytest.mark.parametrize("coord,sfc,per", CASES, ids=IDS)
def test_export_import_round_trip(coord, sfc, per, tmp_path):
    n = 7000
    x, y, z = gen("clustered", n, coord, 3)
    ctx = ft.Context(NAMES[coord], sfc, periodic=per)
    tree = ft.TreeSoA(ctx, n)
    ids = np.arange(n, dtype=np.uint32) * 3 + 1
    ghost = (np.arange(n) % 7 == 0).astype(np.int8)
    ft.build_bvh(ctx, ft.particles(x, y, z, ids, ghost), tree)
    blob = tree.export()
    # host bytes into a fresh context and tree
    ctx2 = ft.Context(NAMES[coord], sfc, periodic=per)
    t2 = ft.import_tree(ctx2, blob.numpy().tobytes())
    _same_tree(tree, t2)
    _same_queries(ctx2, tree, t2, coord)
    # a device buffer, into a larger existing tree
    dev = torch.empty(blob.numel() + 64, dtype=torch.uint8, device="cuda")
    tree.export(out=dev)
    t3 = ft.TreeSoA(ctx, n + 500)
    ft.import_tree(ctx, dev, t3)
    _same_tree(tree, t3)
    # a file
    path = str(tmp_path / "tree.ftb2")
    tree.save(path)
    t4 = ft.load_tree(ctx, path)
    _same_tree(tree, t4)
    _same_queries(ctx, tree, t4, coord)


def test_round_trip_of_refit_and_small_trees():
    ctx = ft.Context("u64", "ph", periodic=True)
    x, y, z = gen("uniform", 3000, O.U64, 8)
    tree = ft.TreeSoA(ctx, 3000)
    ft.build_bvh(ctx, ft.particles(x, y, z), tree)
    ft.refit_bvh(ctx, ft.particles(y, z, x), tree)  # a refit tree keeps its topology
    t2 = ft.import_tree(ctx, tree.export())
    _same_tree(tree, t2)
    _same_queries(ctx, tree, t2, O.U64)
    for n in (1, 2, 3):
        t = ft.TreeSoA(ctx, n)
        ft.build_bvh(ctx, ft.particles(x[:n], y[:n], z[:n]), t)
        _same_tree(t, ft.import_tree(ctx, t.export()))


def test_import_rejects_bad_input():
    ctx = ft.Context("f32", "morton")
    x, y, z = gen("uniform", 1000, O.F32, 9)
    tree = ft.TreeSoA(ctx, 1000)
    ft.build_bvh(ctx, ft.particles(x, y, z), tree)
    blob = tree.export().numpy()
    with pytest.raises(ValueError, match="differs"):
        ft.import_tree(ft.Context("f64", "morton"), blob)
    with pytest.raises(ValueError, match="differs"):
        ft.import_tree(ft.Context("f32", "ph"), blob)
    bad = blob.copy()
    bad[0] ^= 1
    with pytest.raises(ValueError, match="magic"):
        ft.import_tree(ctx, bad, ft.TreeSoA(ctx, 1000))
    with pytest.raises(ValueError, match="shorter"):
        ft.import_tree(ctx, blob[:len(blob) // 2], ft.TreeSoA(ctx, 1000))
    with pytest.raises(ValueError, match="capacity"):
        ft.import_tree(ctx, blob, ft.TreeSoA(ctx, 10))
    with pytest.raises(ValueError, match="too small"):
        tree.export(out=torch.empty(100, dtype=torch.uint8))
