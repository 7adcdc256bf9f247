"""Domain decomposition front end (fasttree_b200/domain.py): the splitter rules on the
reference test's known answers (test/test_domain_decomposition.cpp:10-51), and the whole
pipeline on 2 and 4 gloo ranks shaped like the reference's MPI pipeline test (:53-357): rank 0
starts with every particle, the others with none; after redistribution every particle is
on exactly one rank, on the rank whose SFC range holds its key, and the ranks are balanced;
the halo exchange delivers exactly the other ranks' particles inside each rank's widened
box, marked as ghosts.  Keys come from the oracle's encoding with the global box."""
import os
import socket
from types import SimpleNamespace

import numpy as np
import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

from fasttree_b200 import domain as D
from fasttree_b200.capi import F64, MORTON, PEANO_HILBERT, U32, U64
from fasttree_b200.hlbvh import particles


def test_splitter_uniform():
    hist = np.zeros(1024, np.int64)
    hist[:1000] = 10
    spl = D.generate_splitters(hist, 4, 10)
    assert spl.tolist() == [0, 249, 499, 749, 1024]


def test_splitter_extreme_clustering():
    hist = np.zeros(1024, np.int64)
    hist[500] = 9900
    hist[:100] = 1
    spl = D.generate_splitters(hist, 4, 10)
    assert spl[0] == 0 and spl[4] == 1024 and all(spl[i] <= spl[i + 1] for i in range(4))
    assert spl.tolist() == [0, 500, 500, 500, 1024]


def test_splitter_empty_histogram():
    assert D.generate_splitters(np.zeros(16, np.int64), 3, 4).tolist() == [0, 0, 0, 16]


def test_bucket_ids_follow_the_key_layouts():
    ph64 = SimpleNamespace(coord=U64, sfc=PEANO_HILBERT, device=0)
    keys = np.array([[0, (1 << 61) | 5, 7]], np.uint64)
    assert D.bucket_ids(ph64, keys, 20).tolist() == [((1 << 61) | 5) >> 43]  # 19 bucket bits
    ph32 = SimpleNamespace(coord=U32, sfc=PEANO_HILBERT, device=0)
    keys = np.array([[0, 0x40000000, 3]], np.uint32)
    assert D.bucket_ids(ph32, keys, 10).tolist() == [((0x40000000 << 32) | 3) >> 53]
    mort = SimpleNamespace(coord=F64, sfc=MORTON, device=0)
    assert D.bucket_ids(mort, np.array([[1 << 62]], np.uint64), 4).tolist() == [8]


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


N = 10_000


def _points(coord):
    """The reference test's diagonal: point i at i / N of the extent on all three axes."""
    frac = np.arange(N, dtype=np.float64) / N
    if coord == F64:
        a = frac * 100.0
        return a.copy(), a.copy(), a.copy()
    a = (frac * float((1 << 42) - 1)).astype(np.uint64)
    return a.copy(), a.copy(), a.copy()


def _ref_keys(coord, sfc, x, y, z, bbox):
    """Oracle keys in the reference's sfc_key layout."""
    from oracle import oracle as O
    opts = O.Options(O.F64 if coord == F64 else O.U64, O.MORTON if sfc == MORTON else O.PEANO_HILBERT, False)
    hi, lo = O.sfc_encode(opts, x, y, z, bbox)
    if sfc == MORTON:
        return lo.reshape(-1, 1)
    if coord == U64:  # 126-bit keys: {hs, is, ls} of 64-bit words
        return np.stack([np.zeros_like(lo), hi, lo], axis=1)
    # 63-bit keys: {hs, is, ls} of 32-bit words
    return np.stack([np.zeros_like(lo), lo >> np.uint64(32), lo & np.uint64(0xFFFFFFFF)], axis=1).astype(np.uint32)


def _pipeline_worker(rank, world, port, coord, sfc, sampling, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        ctx = SimpleNamespace(coord=coord, sfc=sfc, device=0)
        dt = np.float64 if coord == F64 else np.uint64
        if rank == 0:
            x, y, z = _points(coord)
        else:
            x = y = z = np.zeros(0, dt)
        ids = np.arange(len(x), dtype=np.uint32)
        p = particles(x, y, z, ids, np.zeros(len(x), np.int8))
        local = None if len(x) == 0 else np.array([x.min(), x.max(), y.min(), y.max(), z.min(), z.max()], dt)
        bbox = D.get_global_bounding_box(ctx, p, local_bbox=local)
        bb = np.array([bbox.min_x, bbox.max_x, bbox.min_y, bbox.max_y, bbox.min_z, bbox.max_z], dt)
        keys = _ref_keys(coord, sfc, x, y, z, bb)
        m = 20
        if sampling:
            spl = D.get_deterministic_splitters(ctx, p, bbox, keys=keys)
            hist_total = N
        else:
            hist = D.get_global_histogram(ctx, p, bbox, m, keys=keys)
            hist_total = int(hist.sum())
            spl = D.generate_splitters(hist, world, m)
        q = D.redistribute_particles(ctx, p, spl, bbox, m, keys=keys, sampling=sampling)
        # every received particle belongs to this rank's SFC range (the reference test's check)
        qk = _ref_keys(coord, sfc, q.pos_x, q.pos_y, q.pos_z, bb)
        dest = D.destinations(ctx, qk, spl, m, sampling)
        in_range = bool(np.all(dest == rank))
        # halo exchange with h_max = 5% of the extent
        h = 5.0 if coord == F64 else float(int(0.05 * ((1 << 42) - 1)))
        g = D.exchange_halos(ctx, q, h)
        nloc = len(q.pos_x)
        ghosts = set(np.asarray(g.id[nloc:]).tolist())
        out[rank] = dict(bbox=bb.tolist(), hist_total=hist_total, spl=np.asarray(spl).tolist(), ids=q.id.tolist(),
                         in_range=in_range, box=[float(q.pos_x.min()), float(q.pos_x.max())] if nloc else None,
                         ghost_ids=sorted(ghosts), ghost_flags=bool(np.all(np.asarray(g.is_ghost[nloc:]) == 1)),
                         local_flags=bool(np.all(np.asarray(g.is_ghost[:nloc]) == 0)), h=h)
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("world", [2, 4])
@pytest.mark.parametrize("coord,sfc,sampling", [(F64, MORTON, False), (U64, PEANO_HILBERT, False),
                                                (F64, PEANO_HILBERT, True), (U64, PEANO_HILBERT, True)],
                         ids=["f64-morton-hist", "u64-ph-hist", "f64-ph-sampling", "u64-ph-sampling"])
def test_pipeline_on_gloo_ranks(world, coord, sfc, sampling):
    ctx = mp.get_context("spawn")
    with ctx.Manager() as mgr:
        out = mgr.dict()
        mp.start_processes(_pipeline_worker, args=(world, _free_port(), coord, sfc, sampling, out), nprocs=world,
                           start_method="spawn")
        res = [out[r] for r in range(world)]
    # every rank saw the same box and splitters; the histogram counts every particle
    assert all(r["bbox"] == res[0]["bbox"] for r in res)
    assert all(r["spl"] == res[0]["spl"] for r in res)
    assert res[0]["hist_total"] == N
    # every particle on exactly one rank, on the rank whose range holds its key
    ids = sorted(i for r in res for i in r["ids"])
    assert ids == list(range(N))
    assert all(r["in_range"] for r in res)
    counts = [len(r["ids"]) for r in res]
    assert all(c > 0 for c in counts)
    if world == 4:
        assert all(2000 < c < 3000 for c in counts), counts
    # ghosts: rank s sends to rank r when s's box widened by h overlaps r's box, and then the
    # particles of s inside r's box widened by h (the points lie on the diagonal, so the x
    # range decides).  Widening is done in the coordinate type: for uint64 a lower bound below
    # zero wraps around, as the reference's does.
    frac = np.arange(N, dtype=np.float64) / N
    xs = frac * 100.0 if coord == F64 else (frac * float((1 << 42) - 1)).astype(np.uint64)

    def widened(box, h):
        if coord == F64:
            return box[0] - h, box[1] + h
        with np.errstate(over="ignore"):
            return np.uint64(box[0]) - np.uint64(h), np.uint64(box[1]) + np.uint64(h)

    for r, rr in enumerate(res):
        want = set()
        h = rr["h"]
        wlo, whi = widened(rr["box"], h)
        for s_, rs in enumerate(res):
            if s_ == r:
                continue
            slo, shi = widened(rs["box"], h)
            rbox = [np.uint64(v) if coord != F64 else v for v in rr["box"]]
            if not (slo <= rbox[1] and shi >= rbox[0]):
                continue  # r is not s's neighbour
            ids_s = np.array(rs["ids"], np.int64)
            xv = xs[ids_s]
            want |= set(ids_s[(xv >= wlo) & (xv <= whi)].tolist())
        assert set(rr["ghost_ids"]) == want, (r, len(want), len(rr["ghost_ids"]))
        assert rr["ghost_flags"] and rr["local_flags"]
    if coord == F64:
        assert sum(len(r["ghost_ids"]) for r in res) > 0


@pytest.mark.gpu
def test_one_nccl_rank_with_the_library_encoding():
    """The front end on one GPU rank over NCCL: the box from compute_bbox, the keys from this
    library's encoding (equal to the oracle's), every particle kept, no ghosts."""
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    import fasttree_b200 as ft
    from oracle import oracle as O
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(_free_port()))
    dist.init_process_group("nccl", rank=0, world_size=1)
    try:
        for coord, sfc, oc, os_ in (("u64", "ph", O.U64, O.PEANO_HILBERT), ("f64", "morton", O.F64, O.MORTON),
                                    ("f32", "ph", O.F32, O.PEANO_HILBERT)):
            ctx = ft.Context(coord, sfc)
            rng = np.random.default_rng(3)
            if coord == "u64":
                x, y, z = (rng.integers(0, 1 << 42, 5000, dtype=np.uint64) for _ in range(3))
            else:
                x, y, z = (rng.uniform(0, 10, 5000).astype(np.float32 if coord == "f32" else np.float64)
                           for _ in range(3))
            p = particles(x, y, z)
            for sampling in (False, True):
                q, bbox, spl = D.decompose(ctx, p, h_max=1, sampling=sampling)
                assert sorted(np.asarray(q.id).tolist()) == list(range(5000))
                assert len(q.pos_x) == 5000  # one rank: no ghosts
            bb = np.array([bbox.min_x, bbox.max_x, bbox.min_y, bbox.max_y, bbox.min_z, bbox.max_z], x.dtype)
            assert np.array_equal(bb, O.compute_bbox(O.Options(oc, os_, False), x, y, z))
            got = D.sfc_keys(ctx, p, bbox)
            hi, lo = O.sfc_encode(O.Options(oc, os_, False), x, y, z, bb)
            ghi, glo = D._key_words(ctx, got)
            assert np.array_equal(glo, lo) and np.array_equal(ghi, hi)
    finally:
        dist.destroy_process_group()
