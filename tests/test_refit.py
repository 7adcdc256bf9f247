"""Refit-only update (ft_refit_bvh): the same points at new positions keep the build's keys,
leaf order and topology, and every box is recomputed.  The updated tree must equal the
oracle's build_tree (src/hlbvh.hpp:773-982) from the build's sorted keys with the new
positions as its leaf arrays, array for array, and queries on it must equal the oracle's
on that tree, bit for bit."""
import numpy as np
import pytest

from oracle import oracle as O
from tests.gpu_util import NAMES, assert_tree_equal, dist_bits, gen

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")
if not torch.cuda.is_available():
    pytest.skip("no CUDA device", allow_module_level=True)

import fasttree_b200 as ft  # noqa: E402

CASES = [(O.U64, O.PEANO_HILBERT, True), (O.U64, O.PEANO_HILBERT, False), (O.U32, O.PEANO_HILBERT, True),
         (O.F32, O.MORTON, False), (O.F64, O.PEANO_HILBERT, False)]
IDS = [f"{NAMES[c]}-{'ph' if s == O.PEANO_HILBERT else 'morton'}{'-per' if p else ''}" for c, s, p in CASES]


def _moved(coord, x, y, z, scale, seed):
    """Positions jittered by `scale` of the box (wrapped / clipped into the coordinate range)."""
    rng = np.random.default_rng(seed)
    out = []
    for a in (x, y, z):
        if coord in (O.F32, O.F64):
            b = a + rng.normal(0.0, scale * 100.0, len(a)).astype(a.dtype)
            out.append(np.clip(b, 0, 100.0).astype(a.dtype))
        else:
            bits = 42 if coord == O.U64 else 21
            m = (1 << bits) - 1
            step = rng.normal(0.0, scale * (1 << bits), len(a)).astype(np.int64)
            out.append(((a.astype(np.int64) + step) & m).astype(a.dtype))
    return out


def _oracle_refit(opts, ot, n, nx, ny, nz):
    """The reference computation a refit stands for: build_tree with the build's sorted keys and
    the new positions gathered into the build's leaf order."""
    orig = ot.orig_idx[n - 1:2 * n - 1].astype(np.int64)
    return O.build_tree(opts, ot.sorted_hi[:n], ot.sorted_lo[:n], nx[orig], ny[orig], nz[orig],
                        ot.id[n - 1:2 * n - 1], ot.is_ghost[n - 1:2 * n - 1], ot.orig_idx[n - 1:2 * n - 1])


@pytest.mark.parametrize("coord,sfc,per", CASES, ids=IDS)
@pytest.mark.parametrize("scale", [1e-4, 0.3])
def test_refit_equals_build_tree_with_the_same_keys(coord, sfc, per, scale):
    n, k = 6000, 16
    x, y, z = gen("clustered", n, coord, 11)
    ctx = ft.Context(NAMES[coord], sfc, periodic=per)
    opts = O.Options(coord, sfc, per)
    tree = ft.TreeSoA(ctx, n)
    ft.build_bvh(ctx, ft.particles(x, y, z), tree)
    ot = O.build_bvh(opts, x, y, z)
    nx, ny, nz = _moved(coord, x, y, z, scale, 12)
    ft.refit_bvh(ctx, ft.particles(nx, ny, nz), tree)
    want = _oracle_refit(opts, ot, n, nx, ny, nz)
    assert_tree_equal(tree.to_numpy(), want, n)
    oi, od = O.self_knn(opts, want, k, True)
    for method in ("plain", "fast"):
        gi, gd = ft.self_knn_query(ctx, tree, k, max_k=32, method=method)
        torch.cuda.synchronize()
        assert np.array_equal(gi.cpu().numpy(), oi), method
        assert np.array_equal(dist_bits(gd.cpu().numpy()), dist_bits(od)), method
    # external queries too (the tree's keys no longer match the moved points: still exact)
    qx, qy, qz = gen("uniform", 500, coord, 13)
    oi, od = O.knn(opts, want, qx, qy, qz, k)
    gi, gd = ft.knn_query(ctx, tree, qx, qy, qz, k, method="fast")
    assert np.array_equal(gi.cpu().numpy(), oi)
    assert np.array_equal(dist_bits(gd.cpu().numpy()), dist_bits(od))


def test_refit_leaf_order_and_repeated_updates():
    coord, sfc, per = O.U64, O.PEANO_HILBERT, True
    n = 5000
    x, y, z = gen("uniform", n, coord, 21)
    ctx = ft.Context("u64", sfc, periodic=per)
    opts = O.Options(coord, sfc, per)
    tree = ft.TreeSoA(ctx, n)
    ft.build_bvh(ctx, ft.particles(x, y, z), tree)
    ot = O.build_bvh(opts, x, y, z)
    orig = ot.orig_idx[n - 1:].astype(np.int64)
    cur = (x, y, z)
    for step in range(3):
        cur = _moved(coord, *cur, 1e-3, 30 + step)
        if step == 1:  # positions handed over in leaf order
            ft.refit_bvh(ctx, ft.particles(*(torch.from_numpy(a[orig]).cuda() for a in cur)), tree, leaf_order=True)
        else:
            ft.refit_bvh(ctx, ft.particles(*cur), tree)
        want = _oracle_refit(opts, ot, n, *cur)
        assert_tree_equal(tree.to_numpy(), want, n)
    gi, gd = ft.self_knn_query(ctx, tree, 32, method="fast")
    oi, od = O.self_knn(opts, want, 32, True)
    torch.cuda.synchronize()
    assert np.array_equal(gi.cpu().numpy(), oi) and np.array_equal(gd.cpu().numpy(), od)


def test_refit_beyond_42_bits_takes_the_general_periodic_form():
    # a periodic 64-bit tree built below 2^42 may use the short wrapped-distance form; a refit
    # that moves a point above 2^42 must fall back to the reference's general form
    coord, sfc, per = O.U64, O.PEANO_HILBERT, True
    n = 4000
    x, y, z = gen("clustered", n, coord, 41)
    ctx = ft.Context("u64", sfc, periodic=per)
    opts = O.Options(coord, sfc, per)
    tree = ft.TreeSoA(ctx, n)
    ft.build_bvh(ctx, ft.particles(x, y, z), tree)
    ot = O.build_bvh(opts, x, y, z)
    nx = x.copy()
    nx[::97] += np.uint64(1 << 42)
    ft.refit_bvh(ctx, ft.particles(nx, y, z), tree)
    want = _oracle_refit(opts, ot, n, nx, y, z)
    assert_tree_equal(tree.to_numpy(), want, n)
    for method in ("plain", "fast"):
        gi, gd = ft.self_knn_query(ctx, tree, 8, method=method)
        oi, od = O.self_knn(opts, want, 8, True)
        torch.cuda.synchronize()
        assert np.array_equal(gi.cpu().numpy(), oi) and np.array_equal(gd.cpu().numpy(), od), method


def test_refit_errors_and_small_trees():
    ctx = ft.Context("f64", "morton")
    tree = ft.TreeSoA(ctx, 100)
    x, y, z = (np.random.default_rng(s).uniform(0, 1, 50) for s in (1, 2, 3))
    with pytest.raises(ValueError):  # not built yet
        ft.refit_bvh(ctx, ft.particles(x, y, z), tree)
    ft.build_bvh(ctx, ft.particles(x, y, z), tree)
    with pytest.raises(ValueError):  # another point count
        ft.refit_bvh(ctx, ft.particles(x[:40], y[:40], z[:40]), tree)
    opts = O.Options(O.F64, O.MORTON, False)
    for n in (1, 2, 3, 50):
        t2 = ft.TreeSoA(ctx, n)
        ft.build_bvh(ctx, ft.particles(x[:n], y[:n], z[:n]), t2)
        ot = O.build_bvh(opts, x[:n], y[:n], z[:n])
        nx = x[:n][::-1].copy()
        ft.refit_bvh(ctx, ft.particles(nx, y[:n], z[:n]), t2)
        assert_tree_equal(t2.to_numpy(), _oracle_refit(opts, ot, n, nx, y[:n], z[:n]), n)
