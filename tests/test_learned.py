"""Learned radius bound (ft_bound_* / ft_self_knn_learned).

* the 12 features, the network's forward pass, its gradient and the Adam step against the
  CPU oracle (oracle/bound_oracle.py);
* training on the GPU lowers the loss;
* self-kNN with any learned bound -- trained, untrained, far too small, far too large -- is
  bit-identical to the plain traversal;
* the trained bound saves node visits over the fast walk without it.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")
if not torch.cuda.is_available():
    pytest.skip("no CUDA device", allow_module_level=True)

import fasttree_b200 as ft  # noqa: E402
from fasttree_b200 import datasets  # noqa: E402
from fasttree_b200 import learned as L  # noqa: E402
from oracle import bound_oracle as BO  # noqa: E402
from oracle import oracle as O  # noqa: E402
from tests.gpu_util import gen  # noqa: E402

FEAT_CASES = [("f32", "morton", False, O.F32, O.MORTON), ("f64", "ph", False, O.F64, O.PEANO_HILBERT),
              ("u32", "ph", True, O.U32, O.PEANO_HILBERT), ("u64", "ph", True, O.U64, O.PEANO_HILBERT),
              ("u64", "ph", False, O.U64, O.PEANO_HILBERT)]


@pytest.mark.parametrize("coord,sfc,per,oc,os_", FEAT_CASES, ids=[f"{c[0]}-{c[1]}{'-per' if c[2] else ''}"
                                                                  for c in FEAT_CASES])
@pytest.mark.parametrize("k", [1, 8, 32])
def test_features_match_oracle(coord, sfc, per, oc, os_, k):
    n = 2500
    x, y, z = gen("clustered", n, oc, 31)
    ctx = ft.Context(coord, sfc, periodic=per)
    tree = ft.TreeSoA(ctx, n)
    ft.build_bvh(ctx, ft.particles(x, y, z), tree)
    got = L.features(ctx, tree, k).cpu().numpy()
    ot = O.build_bvh(O.Options(oc, os_, per), x, y, z)
    want = BO.features(O.Options(oc, os_, per), ot, k)
    assert got.shape == want.shape
    # counts, depth and log2 k exactly; logarithms of lengths to float rounding
    assert np.array_equal(got[:, 4:10], want[:, 4:10])
    assert np.allclose(got, want, rtol=0, atol=2e-5), np.abs(got - want).max(0)
    # a subset of leaf ids gives the same rows
    ids = torch.tensor([0, 7, n - 1, 1234], dtype=torch.int32, device="cuda")
    sub = L.features(ctx, tree, k, leaf_ids=ids).cpu().numpy()
    assert np.array_equal(sub, got[ids.cpu().numpy()])


def _training_data(n=3000, seed=5):
    x, y, z = datasets.clustered_fixed(n, n_spheres=20, seed=seed)
    ctx = ft.Context("u64", "ph", periodic=True)
    f, t = L.training_set(ctx, x, y, z, 16)
    return ctx, f, t


def _norm(f, t):
    fd = f.double()
    td = t.double() - fd[:, 10]
    return (fd.mean(0).cpu().numpy().astype(np.float32), fd.std(0).cpu().numpy().astype(np.float32),
            float(td.mean()), float(td.std()))


def test_forward_matches_oracle():
    ctx, f, t = _training_data()
    m = L.BoundModel(ctx, seed=3)
    norm = _norm(f, t)
    m.set_norm(*norm)
    pred = m.predict(f).cpu().numpy()
    want = BO.predict_log2(m.params, f.cpu().numpy(), norm)
    err = np.abs(pred - want)
    assert np.quantile(err, 0.99) < 1e-3 and err.max() < 2e-2, (np.quantile(err, 0.99), err.max())


def test_gradient_matches_oracle():
    ctx, f, t = _training_data()
    m = L.BoundModel(ctx, seed=4)
    norm = _norm(f, t)
    m.set_norm(*norm)
    g, loss = m.gradient(f, t)
    wl, wg = BO.loss_and_grad(m.params, f.cpu().numpy(), t.cpu().numpy(), norm)
    assert abs(loss - wl) <= 1e-3 * max(1.0, abs(wl))
    rel = np.linalg.norm(g - wg) / np.linalg.norm(wg)
    assert rel < 5e-3, rel
    # every parameter block agrees on its own
    for a, b in ((0, 768), (768, 832), (832, 4928), (4928, 4992), (4992, 5056), (5056, 5057)):
        assert np.linalg.norm(g[a:b] - wg[a:b]) <= 1e-2 * np.linalg.norm(wg[a:b]) + 1e-7, (a, b)


def _rows(seed, step, batch, n):
    """The minibatch rows of mlp_rows_kernel (splitmix64 of seed, step, i)."""
    M = (1 << 64) - 1
    out = np.empty(batch, np.int64)
    for i in range(batch):
        z = (seed + 0x9E3779B97F4A7C15 * ((step * 0x100000001 + i + 1) & M)) & M
        z = ((z ^ (z >> 30)) * 0xBF58476D1CE4E5B9) & M
        z = ((z ^ (z >> 27)) * 0x94D049BB133111EB) & M
        z ^= z >> 31
        out[i] = z % n
    return out


def test_adam_steps_match_oracle():
    ctx, f, t = _training_data()
    m = L.BoundModel(ctx, seed=6)
    norm = _norm(f, t)
    m.set_norm(*norm)
    p = m.params.astype(np.float64)
    mm, vv = np.zeros_like(p), np.zeros_like(p)
    fn, tn = f.cpu().numpy(), t.cpu().numpy()
    seed, batch, lr = 77, 512, 1e-3
    for step in range(2):
        m.fit(f, t, steps=1, batch=batch, lr=lr, seed=seed)
        rows = _rows(seed, step, batch, len(tn))
        _, g = BO.loss_and_grad(p.astype(np.float32), fn[rows], tn[rows], norm)
        p, mm, vv = BO.adam(p, mm, vv, g, step + 1, lr)
        got = m.params.astype(np.float64)
        # Adam normalises each coordinate: compare the step taken, not the tiny gradients
        assert np.quantile(np.abs(got - p), 0.99) < 0.05 * lr * (step + 1), step


def test_training_lowers_the_loss():
    x, y, z = datasets.clustered_fixed(200_000, n_spheres=400, seed=12)
    ctx = ft.Context("u64", "ph", periodic=True)
    m, losses = L.train_bound(ctx, x, y, z, 32, steps=400, batch=4096, lr=3e-3, seed=1)
    assert np.all(np.isfinite(losses))
    assert losses[-50:].mean() < 0.5 * losses[:10].mean(), (losses[:10].mean(), losses[-50:].mean())


def _plain(ctx, tree, k):
    i, d = ft.self_knn_query(ctx, tree, k, max_k=max(32, k), method="plain")
    torch.cuda.synchronize()
    return i.clone(), d.clone()


@pytest.mark.parametrize("coord,sfc,per", [("u64", "ph", True), ("f32", "morton", False), ("u32", "ph", True)])
def test_learned_output_is_exact_for_any_network(coord, sfc, per):
    n, k = 150_000, 32
    oc = {"u64": O.U64, "f32": O.F32, "u32": O.U32}[coord]
    x, y, z = gen("clustered", n, oc, 8)
    tx, ty, tz = gen("clustered", 60_000, oc, 9)
    ctx = ft.Context(coord, sfc, periodic=per)
    tree = ft.TreeSoA(ctx, n)
    ft.build_bvh(ctx, ft.particles(x, y, z), tree)
    pi, pd = _plain(ctx, tree, k)
    trained, _ = L.train_bound(ctx, tx, ty, tz, k, steps=200, batch=4096)
    untrained = L.BoundModel(ctx, seed=9)
    tiny = L.BoundModel(ctx, seed=9)
    p = tiny.params
    p[BO.OFF_B3] = -60.0  # predicts ~0: every bound too small, every query replayed
    tiny.params = p
    huge = L.BoundModel(ctx, seed=9)
    p[BO.OFF_B3] = 60.0
    huge.params = p
    for name, model in (("trained", trained), ("untrained", untrained), ("tiny", tiny), ("huge", huge)):
        for infl in (1.0, 1.15):
            i, d = L.self_knn_query_learned(ctx, tree, model, k, inflation=infl)
            torch.cuda.synchronize()
            ctx_stats = ctx.query_stats()
            assert torch.equal(i, pi) and torch.equal(d, pd), (name, infl)
            if name == "tiny":
                # every bound too small: every query reruns the walk without the bound, and
                # only its ties reach the reference traversal
                assert ctx_stats["bound_misses"] >= n - 10
                assert ctx_stats["replayed"] < 0.01 * n
    # subsets too
    ids = torch.randperm(n, device="cuda")[:5000].to(torch.int32)
    i, d = L.self_knn_query_learned(ctx, tree, trained, k, leaf_ids=ids, max_k=32)
    si, sd = ft.self_knn_query_subset(ctx, tree, ids, k, max_k=32)
    torch.cuda.synchronize()
    assert torch.equal(i, si) and torch.equal(d, sd)


def test_trained_bound_saves_visits():
    k = 32
    tx, ty, tz = datasets.clustered_fixed(1_000_000, n_spheres=2000, seed=12)
    x, y, z = datasets.clustered_fixed(1_000_000, n_spheres=2000, seed=2)
    ctx = ft.Context("u64", "ph", periodic=True)
    model, _ = L.train_bound(ctx, tx, ty, tz, k, steps=2000, batch=8192)
    tree = ft.TreeSoA(ctx, len(x))
    ft.build_bvh(ctx, ft.particles(x, y, z), tree)
    pi, pd = _plain(ctx, tree, k)
    ft.self_knn_query(ctx, tree, k, method="fast")
    torch.cuda.synchronize()
    fast = ctx.query_stats()
    i, d = L.self_knn_query_learned(ctx, tree, model, k, inflation=1.15)
    torch.cuda.synchronize()
    learned = ctx.query_stats()
    assert torch.equal(i, pi) and torch.equal(d, pd)
    bounded = learned["visits"] - learned["rerun_visits"]
    print(f"visits/query fast {fast['visits'] / len(x):.1f} learned {bounded / len(x):.1f} in the bounded walk "
          f"+ {learned['rerun_visits'] / len(x):.1f} in the rerun of {learned['bound_misses']} misses, "
          f"replayed fast {fast['replayed']} learned {learned['replayed']}")
    # the trained bound prunes more than the seeded walk alone (the gain), and misses on few
    # queries (the cost, paid by rerunning them without the bound)
    assert bounded < fast["visits"]
    assert learned["bound_misses"] < 0.2 * len(x)
    assert learned["replayed"] < 0.01 * len(x)


def _point_queries(n_q, oc, x, y, z, seed):
    """External points: a uniform draw, copies of tree points (exact key matches) and, for
    float coordinates, points outside the tree's box."""
    qx, qy, qz = gen("uniform", n_q, oc, seed)
    qx, qy, qz = (np.array(a) for a in (qx, qy, qz))
    m = n_q // 4
    qx[:m], qy[:m], qz[:m] = x[:m], y[:m], z[:m]
    if oc in (O.F32, O.F64):
        qx[m:m + 8] = -5.0
        qz[m + 8:m + 16] = qz.max() * 3
    return qx, qy, qz


@pytest.mark.parametrize("coord,sfc,per,oc,os_", FEAT_CASES, ids=[f"{c[0]}-{c[1]}{'-per' if c[2] else ''}"
                                                                  for c in FEAT_CASES])
@pytest.mark.parametrize("k", [1, 8, 32, 48])
def test_point_features_match_oracle(coord, sfc, per, oc, os_, k):
    n, n_q = 2500, 500
    x, y, z = gen("clustered", n, oc, 41)
    qx, qy, qz = _point_queries(n_q, oc, x, y, z, 42)
    ctx = ft.Context(coord, sfc, periodic=per)
    tree = ft.TreeSoA(ctx, n)
    ft.build_bvh(ctx, ft.particles(x, y, z), tree)
    got = L.features_points(ctx, tree, qx, qy, qz, k).cpu().numpy()
    opts = O.Options(oc, os_, per)
    ot = O.build_bvh(opts, x, y, z)
    want = BO.features_points(opts, ot, k, qx, qy, qz, O.compute_bbox(opts, x, y, z))
    assert got.shape == want.shape
    assert np.array_equal(got[:, 4:10], want[:, 4:10])
    assert np.allclose(got, want, rtol=0, atol=2e-5), np.abs(got - want).max(0)


def test_point_features_need_library_keys():
    n = 3000
    x, y, z = gen("uniform", n, O.U64, 3)
    ctx = ft.Context("u64", "ph", periodic=True)
    keys = ft.sfc_encode(ctx, x, y, z)
    tree = ft.TreeSoA(ctx, n)
    ft.build_bvh(ctx, ft.particles(x, y, z), tree, key=keys)
    with pytest.raises(ValueError, match="keys"):
        L.features_points(ctx, tree, x[:10], y[:10], z[:10], 8)


@pytest.mark.parametrize("coord,sfc,per", [("u64", "ph", True), ("f32", "morton", False), ("u32", "ph", True)])
def test_learned_knn_query_is_exact_for_any_network(coord, sfc, per):
    n, n_q = 150_000, 40_000
    oc = {"u64": O.U64, "f32": O.F32, "u32": O.U32}[coord]
    x, y, z = gen("clustered", n, oc, 18)
    qx, qy, qz = _point_queries(n_q, oc, x, y, z, 19)
    tx, ty, tz = gen("clustered", 60_000, oc, 20)
    ctx = ft.Context(coord, sfc, periodic=per)
    tree = ft.TreeSoA(ctx, n)
    ft.build_bvh(ctx, ft.particles(x, y, z), tree)
    trained, _ = L.train_bound(ctx, tx, ty, tz, 16, steps=200, batch=4096)
    untrained = L.BoundModel(ctx, seed=9)
    tiny = L.BoundModel(ctx, seed=9)
    p = tiny.params
    p[BO.OFF_B3] = -60.0
    tiny.params = p
    huge = L.BoundModel(ctx, seed=9)
    p[BO.OFF_B3] = 60.0
    huge.params = p
    # both of knn_query's heap tiers: the register heap (MAXK <= 32) and the merge heap
    for k, max_k in ((16, 32), (16, 256), (32, 32), (40, 64)):
        pi, pd = ft.knn_query(ctx, tree, qx, qy, qz, k, max_k=max_k, method="plain")
        pi, pd = pi.clone(), pd.clone()
        for name, model in (("trained", trained), ("untrained", untrained), ("tiny", tiny), ("huge", huge)):
            i, d = L.knn_query_learned(ctx, tree, model, qx, qy, qz, k, max_k=max_k, inflation=1.15)
            torch.cuda.synchronize()
            assert torch.equal(i, pi) and torch.equal(d, pd), (name, k, max_k)
            if name == "tiny":
                st = ctx.query_stats()
                assert st["bound_misses"] >= n_q - 10
                assert st["replayed"] < 0.05 * n_q
