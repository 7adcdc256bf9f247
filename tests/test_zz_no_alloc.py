"""ft_self_knn_noalloc: self-kNN for callers that cannot let the library allocate device
memory (a code that has handed the GPU to its own memory pool, or a step that must not be
stalled by cudaMalloc's device-wide synchronisation).  Its scratch is a fixed array in the
library; these tests call it through the C ABI twice in a row and check each result
against ft_self_knn's, bit for bit, and the headline-shaped case against the oracle as well.
Kept in a file of its own, collected last."""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")
if not torch.cuda.is_available():
    pytest.skip("no CUDA device", allow_module_level=True)

import fasttree_b200 as ft  # noqa: E402
from fasttree_b200 import capi, datasets  # noqa: E402
from oracle import oracle as O  # noqa: E402
from tests.gpu_util import gen  # noqa: E402

MAX_QUERIES = 1 << 20


def noalloc(ctx, tree, k, leaf_ids=None, exclude_self=True):
    num = tree.num_leaves if leaf_ids is None else len(leaf_ids)
    idx = torch.empty(num * k, dtype=torch.uint64, device="cuda")
    dist = torch.empty(num * k, dtype=ft.dist_torch_dtype(ctx.coord), device="cuda")
    st = capi.lib().ft_self_knn_noalloc(ctx.handle, tree.c, None if leaf_ids is None else leaf_ids.data_ptr(), num,
                                        int(k), int(exclude_self), idx.data_ptr(), dist.data_ptr(),
                                        torch.cuda.current_stream().cuda_stream)
    capi.check(st)
    torch.cuda.synchronize()
    capi.check(capi.lib().ft_check_device_status(ctx.handle, torch.cuda.current_stream().cuda_stream))
    return idx.view(num, k).cpu().numpy(), dist.view(num, k).cpu().numpy()


def existing(ctx, tree, k, leaf_ids=None, exclude_self=True):
    if leaf_ids is None:
        i, d = ft.self_knn_query(ctx, tree, k, exclude_self=exclude_self, max_k=max(k, 32), method="fast")
    else:
        i, d = ft.self_knn_query_subset(ctx, tree, leaf_ids, k, exclude_self=exclude_self, max_k=max(k, 32),
                                        method="fast")
    torch.cuda.synchronize()
    return i.cpu().numpy(), d.cpu().numpy()


def same(a, b):
    return np.array_equal(a[0], b[0]) and np.array_equal(a[1].view(np.uint8), b[1].view(np.uint8))


def test_matches_existing_entry_point_twice_in_a_row():
    # clustered 42-bit periodic points (the benchmark's shape), full self-kNN, k = 32
    x, y, z = datasets.clustered_fixed(200_000, n_spheres=400, seed=2)
    ctx = ft.Context("u64", "ph", periodic=True)
    tree = ft.TreeSoA(ctx, len(x))
    ft.build_bvh(ctx, ft.particles(x, y, z), tree)
    want = existing(ctx, tree, 32)
    want_stats = ctx.query_stats()
    first = noalloc(ctx, tree, 32)
    second = noalloc(ctx, tree, 32)
    assert same(first, want)
    assert same(second, want)
    # the context's query statistics describe the no-allocation call, as after ft_self_knn
    st = ctx.query_stats()
    assert st["queries"] == len(x) and st["replayed"] == want_stats["replayed"]
    assert st["visits"] == want_stats["visits"]
    # and the rows are the oracle's (the reference's algorithm restated on the CPU)
    opts = O.Options(O.U64, O.PEANO_HILBERT, True)
    oi, od = O.self_knn(opts, O.build_bvh(opts, x, y, z), 32, True)
    assert same(second, (oi, od))


def test_shared_scratch_is_reset_between_calls():
    # degenerate points (many ties -> many replays) then a different tree: the second call
    # must not see the first call's replay list
    ctx = ft.Context("f64", "morton")
    xa, ya, za = gen("degenerate", 20_000, 1, seed=3)
    ta = ft.TreeSoA(ctx, len(xa))
    ft.build_bvh(ctx, ft.particles(xa, ya, za), ta)
    xb, yb, zb = gen("uniform", 30_000, 1, seed=4)
    tb = ft.TreeSoA(ctx, len(xb))
    ft.build_bvh(ctx, ft.particles(xb, yb, zb), tb)
    want_a, want_b = existing(ctx, ta, 16), existing(ctx, tb, 16)
    assert same(noalloc(ctx, ta, 16), want_a)
    assert same(noalloc(ctx, tb, 16), want_b)
    sub = torch.arange(0, 20_000, 7, dtype=torch.int32, device="cuda")
    want_s = existing(ctx, ta, 24, leaf_ids=sub)
    assert same(noalloc(ctx, ta, 24, leaf_ids=sub), want_s)
    assert same(noalloc(ctx, ta, 24, leaf_ids=sub), want_s)


def test_large_k_uses_the_reference_traversal():
    ctx = ft.Context("u32", "ph", periodic=True)
    x, y, z = gen("clustered", 5000, 2, seed=5)
    tree = ft.TreeSoA(ctx, len(x))
    ft.build_bvh(ctx, ft.particles(x, y, z), tree)
    want = existing(ctx, tree, 100)
    assert same(noalloc(ctx, tree, 100), want)
    assert same(noalloc(ctx, tree, 100), want)


def test_rejects_more_queries_than_the_fixed_scratch_holds():
    ctx = ft.Context("f64", "morton")
    x, y, z = gen("uniform", 1000, 1, seed=6)
    tree = ft.TreeSoA(ctx, len(x))
    ft.build_bvh(ctx, ft.particles(x, y, z), tree)
    ids = torch.zeros(MAX_QUERIES + 1, dtype=torch.int32, device="cuda")
    out_i = torch.empty(1, dtype=torch.uint64, device="cuda")
    out_d = torch.empty(1, dtype=torch.float64, device="cuda")
    st = capi.lib().ft_self_knn_noalloc(ctx.handle, tree.c, ids.data_ptr(), MAX_QUERIES + 1, 8, 1,
                                        out_i.data_ptr(), out_d.data_ptr(), torch.cuda.current_stream().cuda_stream)
    assert st == capi.FT_ERR_INVALID_ARGUMENT
    assert b"1048576" in capi.lib().ft_last_error()


def test_host_output_buffers_are_rejected_before_any_launch():
    # the kernels write straight into the output arrays, so pageable host memory is refused
    # with an error instead of reaching the GPU
    ctx = ft.Context("f64", "morton")
    x, y, z = gen("uniform", 1000, 1, seed=7)
    tree = ft.TreeSoA(ctx, len(x))
    ft.build_bvh(ctx, ft.particles(x, y, z), tree)
    host_i = np.empty(1000 * 8, np.uint64)
    host_d = np.empty(1000 * 8, np.float64)
    dev_i = torch.empty(1000 * 8, dtype=torch.uint64, device="cuda")
    dev_d = torch.empty(1000 * 8, dtype=torch.float64, device="cuda")
    stream = torch.cuda.current_stream().cuda_stream
    for oi, od in ((host_i.ctypes.data, dev_d.data_ptr()), (dev_i.data_ptr(), host_d.ctypes.data),
                   (host_i.ctypes.data, host_d.ctypes.data)):
        st = capi.lib().ft_self_knn_noalloc(ctx.handle, tree.c, None, 1000, 8, 1, oi, od, stream)
        assert st == capi.FT_ERR_INVALID_ARGUMENT
        assert b"device memory" in capi.lib().ft_last_error()
    host_ids = np.arange(10, dtype=np.int32)
    st = capi.lib().ft_self_knn_noalloc(ctx.handle, tree.c, host_ids.ctypes.data, 10, 8, 1, dev_i.data_ptr(),
                                        dev_d.data_ptr(), stream)
    assert st == capi.FT_ERR_INVALID_ARGUMENT
    capi.check(capi.lib().ft_check_device_status(ctx.handle, stream))
