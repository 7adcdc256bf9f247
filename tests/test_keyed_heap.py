"""The fast walk's heap keys a distance by rounding it toward zero to a float.  Neighbours
whose exact distances differ but share a key test what that rounding must not change: runs of
equal keys inside a row ordered by the exact distances, a candidate or an eviction on the k-th
key (flagged for the replay on self queries, settled exactly on external ones).  Points on
axis rays from a centre at shifted gaps 2^25 + i have squared distances 2^50 + 2^26 i + i^2,
two or three to a float key; rows and counts bit for bit against the oracle."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")
if not torch.cuda.is_available():
    pytest.skip("no CUDA device", allow_module_level=True)

import fasttree_b200 as ft  # noqa: E402
from oracle import oracle as O  # noqa: E402
from tests.gpu_util import dist_bits  # noqa: E402


def ray_points(coord, n_centres=24, per_ray=40, seed=5):
    """Centres spread over the box, each with points along the six axis rays whose distances
    from it differ by less than a float key's resolution; plus some uniform points."""
    rng = np.random.default_rng(seed)
    dirs = np.array([[1, 0, 0], [-1, 0, 0], [0, 1, 0], [0, -1, 0], [0, 0, 1], [0, 0, -1]])
    pts, centres = [], []
    if coord == "u64":
        shift, base = 11, 1 << 25  # shifted gaps 2^25 + i: squared distances 2^50 + 2^26 i + i^2
        lo, hi = 1 << 38, (1 << 42) - (1 << 38)
        for c in rng.integers(lo, hi, (n_centres, 3)):
            centres.append(c)
            pts.append(c)
            for i in range(per_ray):
                # keep the low bits random below the shift: the exact gaps stay (base + i) << shift
                off = ((base + i) << shift) + int(rng.integers(0, 1 << shift))
                pts.append(c + dirs[i % 6] * off)
        extra = rng.integers(lo, hi, (400, 3))
        a = np.concatenate([np.array(pts, np.int64), extra]).astype(np.uint64)
        cen = np.array(centres, np.int64)
        q = cen.astype(np.uint64)  # at the centres: the rays' shifted gaps are base + i exactly
    else:
        for c in rng.uniform(10.0, 90.0, (n_centres, 3)):
            centres.append(c)
            pts.append(c)
            for i in range(per_ray):
                pts.append(c + dirs[i % 6] * (1.0 + i * 2.0 ** -26))  # distances within float keys
        extra = rng.uniform(0.0, 100.0, (400, 3))
        a = np.concatenate([np.array(pts), extra])
        q = np.array(centres) * 1.0
    return (a[:, 0].copy(), a[:, 1].copy(), a[:, 2].copy()), (q[:, 0].copy(), q[:, 1].copy(), q[:, 2].copy())


CASES = [("u64", "ph", False, O.U64, O.PEANO_HILBERT), ("u64", "ph", True, O.U64, O.PEANO_HILBERT),
         ("f64", "morton", False, O.F64, O.MORTON)]


@pytest.mark.parametrize("coord,sfc,per,oc,os_", CASES, ids=["u64", "u64-per", "f64"])
@pytest.mark.parametrize("k", [4, 16, 32, 64])
def test_equal_keys_self_and_external(coord, sfc, per, oc, os_, k):
    (x, y, z), (qx, qy, qz) = ray_points(coord)
    ctx = ft.Context(coord, sfc, periodic=per)
    tree = ft.TreeSoA(ctx, len(x))
    ft.build_bvh(ctx, ft.particles(x, y, z), tree)
    opts = O.Options(oc, os_, per)
    ot = O.build_bvh(opts, x, y, z)
    mk = 32 if k <= 32 else 128  # (k == max_k above 32 is the reference's capacity case)
    gi, gd = ft.self_knn_query(ctx, tree, k, max_k=mk, method="fast")
    torch.cuda.synchronize()
    oi, od = O.self_knn(opts, ot, k, True)
    assert np.array_equal(gi.cpu().numpy(), oi)
    assert np.array_equal(dist_bits(gd.cpu().numpy()), dist_bits(od))
    ei, ed = ft.knn_query(ctx, tree, qx, qy, qz, k, max_k=mk, method="fast")
    torch.cuda.synchronize()
    replayed = ctx.query_stats()["replayed"]
    oi2, od2 = O.knn(opts, ot, qx, qy, qz, k, mk)
    assert np.array_equal(ei.cpu().numpy(), oi2)
    assert np.array_equal(dist_bits(ed.cpu().numpy()), dist_bits(od2))
    # the centres' rows hold runs of distinct distances on equal keys: the 4-wide walk (k > 4)
    # settles them without the replay (its ties are exact ones only; here the rays' distances
    # are all distinct); the compact binary walk of k <= 4 flags them, and the replay's rows
    # are the ones compared above
    if k > 4:
        assert replayed == 0, replayed
