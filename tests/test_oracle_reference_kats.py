"""The oracle against the reference's own known answers and test rules (CPU only).

* test/test_mpi.cpp:183-217 -- 1000-point line, keys 0..999: 20 points within 10 of 500.5.
* test/test_domain_decomposition.cpp:360-470 -- ghost visibility (range count 2, kNN ghost).
* test/main.cpp:140-323 -- 10^3 grid: SFC monotonicity, range count vs brute force, kNN
  distances vs brute force (k = 5, 48 with knn_query<128>).
* test/test_self_knn.cpp:374-562 -- isolated LocalMaxHeap / SortedMergeHeap runs.
* test/test_self_knn.cpp:75-266, 571-1003 -- self-kNN / subset / knn_query vs host brute force
  with the reference's rules: exact integer distances, 1e-4 relative float tolerance,
  indices compared only at untied ranks, no duplicate indices, sentinels past the count.
* the Morton max-point quirk: a coordinate at the bbox maximum lands in cell 0.
"""
import numpy as np
import pytest

from oracle import oracle as O
from tests.gpu_util import BOX, CONFIG_IDS, CONFIGS, gen, radius, to_coord


def brute_force(opts, tree, query_ranks, k, exclude_self, box=BOX):
    """compute_host_brute_force_knn (test/test_self_knn.cpp:75-147) with tie flags."""
    lx, ly, lz = tree.leaf_coords()
    n = tree.n
    out = []
    for q in query_ranks:
        p = np.array([lx[q], ly[q], lz[q]])
        cand = []
        for j in range(n):
            if exclude_self and j == q:
                continue
            b = np.array([lx[j], lx[j], ly[j], ly[j], lz[j], lz[j]])
            d = O.point_dist(opts, p, b)
            ret = int(tree.orig_idx[j + n - 1]) if opts.return_orig else j
            cand.append((d, ret))
        cand.sort(key=lambda c: (c[0], c[1]))
        tied = []
        for i in range(len(cand)):
            t = False
            for jj in (i - 1, i + 1):
                if 0 <= jj < len(cand):
                    if opts.coord in (O.U32, O.U64):
                        t |= cand[i][0] == cand[jj][0]
                    else:
                        a, b = float(cand[i][0]), float(cand[jj][0])
                        t |= abs(a - b) <= 1e-4 * max(a, 1.0) + 1e-9
            tied.append(t)
        out.append([(c[0], c[1], t) for c, t in zip(cand[:k], tied[:k])])
    return out


def verify(opts, idx, dist, expected, k):
    """verify_results (test/test_self_knn.cpp:153-266)."""
    for q, exp in enumerate(expected):
        row = [int(v) for v in idx[q] if int(v) != 0xFFFFFFFFFFFFFFFF]
        assert len(row) == len(set(row)), "duplicate index"
        for i in range(k):
            if i < len(exp):
                d_exp, i_exp, tied = exp[i]
                if opts.coord in (O.U32, O.U64):
                    assert int(dist[q, i]) == int(d_exp)
                else:
                    assert abs(float(dist[q, i]) - float(d_exp)) <= 1e-4 * max(float(d_exp), 1.0) + 1e-9
                if not tied:
                    assert int(idx[q, i]) == i_exp
            else:
                assert int(idx[q, i]) == 0xFFFFFFFFFFFFFFFF


@pytest.mark.parametrize("coord", [O.F32, O.F64])
def test_line_range_count_is_20(coord):
    opts = O.Options(coord, O.MORTON)
    n = 1000
    xs = np.arange(n).astype(O.NP_COORD[coord])
    zs = np.zeros(n, O.NP_COORD[coord])
    t = O.build_tree(opts, None, np.arange(n, dtype=np.uint64), xs, zs, zs)
    _, cnt = O.range_query(opts, t, [500.5], [0], [0], [0], [10], 100)
    assert cnt[0] == 20


def test_ghost_visibility():
    opts = O.Options(O.F64, O.MORTON)
    x = np.array([1.0, 2.0, 3.0, -1.0, 10.0])
    z = np.zeros(5)
    ids = np.array([100, 101, 102, 200, 201], np.uint32)
    gh = np.array([0, 0, 0, 1, 1], np.int8)
    t = O.build_bvh(opts, x, z, z, ids, gh)
    assert (t.is_ghost[4:] == 1).sum() == 2
    res, cnt = O.range_query(opts, t, [-0.5], [0], [0], [0], [2.0], 10)
    assert cnt[0] == 2
    assert sorted(int(t.id[4 + r]) for r in res[0, :2]) == [100, 200]
    ki, kd = O.knn(opts, t, [9.5], [0], [0], 2)
    assert t.id[4 + ki[0, 0]] == 201 and t.is_ghost[4 + ki[0, 0]] == 1
    assert abs(kd[0, 0] - 0.25) < 1e-4


def test_morton_max_point_maps_to_cell_zero():
    """1 + nextafter(1, 0) rounds to 2.0, whose mantissa is 0 (src/hlbvh.hpp:395, 411-414)."""
    for coord in (O.F32, O.F64):
        opts = O.Options(coord, O.MORTON)
        x = np.array([0.0, 0.5, 1.0], O.NP_COORD[coord])
        hi, lo = O.sfc_encode(opts, x, x, x, np.array([0, 1, 0, 1, 0, 1], O.NP_COORD[coord]))
        assert lo[0] == 0 and lo[2] == 0 and lo[1] != 0
    # Peano-Hilbert clamps below 2 instead (src/sfc.peano_hilbert.hpp:472-476)
    opts = O.Options(O.F64, O.PEANO_HILBERT)
    x = np.array([0.0, 1.0])
    hi, lo = O.sfc_encode(opts, x, x, x, np.array([0, 1, 0, 1, 0, 1.0]))
    assert lo[1] != 0


@pytest.mark.parametrize("coord,periodic", [(O.F64, False), (O.F32, False), (O.U32, False), (O.U32, True),
                                            (O.U64, False), (O.U64, True)])
def test_grid_sfc_range_knn(coord, periodic):
    """test/main.cpp: 10x10x10 grid in [0,100)^3, bbox [0,100]^3 for floats."""
    sfc = O.PEANO_HILBERT if coord in (O.U32, O.U64) else O.MORTON
    opts = O.Options(coord, sfc, periodic)
    g = (np.arange(10) + 0.5) * 10.0
    X, Y, Z = np.meshgrid(g, g, g, indexing="ij")
    x, y, z = (to_coord(a.ravel(), coord) for a in (X, Y, Z))
    bbox = np.array([0, 100, 0, 100, 0, 100], O.NP_COORD[coord]) if coord in (O.F32, O.F64) else None
    t = O.build_bvh(opts, x, y, z, bbox=bbox)
    # TEST 1 -- keys of the sorted leaves are non-decreasing
    lx, ly, lz = t.leaf_coords()
    hi, lo = O.sfc_encode(opts, lx, ly, lz, t.bbox)
    k = [(int(a) << 64) | int(b) for a, b in zip(hi, lo)]
    assert all(k[i] <= k[i + 1] for i in range(len(k) - 1))
    # TEST 2 -- range count vs brute force (query (52,52,52), r in [0, 20])
    qp = to_coord(np.array([52.0]), coord)
    rmax = np.array([radius(20.0, coord)], O.NP_COORD[coord])
    rmin = np.zeros(1, O.NP_COORD[coord])
    _, cnt = O.range_query(opts, t, qp, qp, qp, rmin, rmax, 1000)
    P = np.stack([lx, ly, lz], 1)
    if coord in (O.F32, O.F64):
        d = np.sqrt(((P.astype(np.float64) - 52.0) ** 2).sum(1))
        assert cnt[0] == int(((d >= 0) & (d <= 20)).sum())
    else:
        d2 = np.array([O.point_dist(opts, np.repeat(qp, 3), np.array([p[0], p[0], p[1], p[1], p[2], p[2]]))
                       for p in P])
        rm = int(rmax[0]) >> (11 if coord == O.U64 else 0)
        assert cnt[0] == int((d2 <= rm * rm).sum())
    # TEST 3 -- kNN k = 5 and 48 with knn_query<128>: distances match the brute force
    for kk in (5, 48):
        qi, qd = O.knn(opts, t, qp, qp, qp, kk, 128)
        d2 = np.sort(np.array([O.point_dist(opts, np.repeat(qp, 3),
                                            np.array([p[0], p[0], p[1], p[1], p[2], p[2]])) for p in P]))
        assert np.array_equal(np.asarray(qd[0], dtype=d2.dtype), d2[:kk])


def test_isolated_local_max_heap():
    """LocalMaxHeap test (test/test_self_knn.cpp:380-448): 32 lanes, k = 48, values with duplicates."""
    for lane in range(32):
        vals = [((v * 17 + lane * 13) % 73) for v in range(100, 0, -1)]
        d, i, cnt = O.maxheap_run(48, np.array(vals, np.float64), np.arange(100, 0, -1, dtype=np.int32))
        assert cnt == 48
        assert np.array_equal(d, np.sort(np.array(vals, np.float64))[:48])


def test_isolated_sorted_merge_heap():
    """SortedMergeHeap test (test/test_self_knn.cpp:450-558): three 32-wide rounds, k = 48, cap 64."""
    lid = np.arange(32)
    DMAX = np.finfo(np.float64).max
    r1 = ((31 - lid) * 10).astype(np.float64), lid.astype(np.int32)
    r2 = ((lid % 4) * 5).astype(np.float64), (100 + lid).astype(np.int32)
    r3 = np.where(lid < 16, lid + 1, DMAX).astype(np.float64), np.where(lid < 16, 200 + lid, -1).astype(np.int32)
    d = np.stack([r1[0], r2[0], r3[0]])
    i = np.stack([r1[1], r2[1], r3[1]])
    od, oi = O.mergeheap_run(48, 64, d, i)
    exp = sorted(list(zip(r1[0], r1[1])) + list(zip(r2[0], r2[1])) + [(float(a), int(b)) for a, b in
                                                                       zip(r3[0][:16], r3[1][:16])])
    assert np.array_equal(od[:48], np.array([e[0] for e in exp[:48]]))


@pytest.mark.parametrize("cfg", CONFIGS, ids=CONFIG_IDS)
@pytest.mark.parametrize("kind", ["uniform", "clustered", "degenerate"])
def test_self_knn_vs_brute_force(cfg, kind):
    coord, sfc, per = cfg
    opts = O.Options(coord, sfc, per)
    n = 300
    x, y, z = gen(kind, n, coord, seed=42)
    t = O.build_bvh(opts, x, y, z)
    ranks = list(range(0, n, 7))
    for k in (16, 33):
        for excl in (True, False):
            idx, dist = O.self_knn(opts, t, k, excl, leaf_ids=np.array(ranks, np.int32))
            verify(opts, idx, dist, brute_force(opts, t, ranks, k, excl), k)


@pytest.mark.parametrize("n", [1, 2, 7, 33])
def test_edge_cases_vs_brute_force(n):
    opts = O.Options(O.F64, O.MORTON)
    x, y, z = gen("uniform", n, O.F64, seed=777)
    t = O.build_bvh(opts, x, y, z)
    for k in (1, 2, 5, 33):
        for excl in (True, False):
            idx, dist = O.self_knn(opts, t, k, excl)
            verify(opts, idx, dist, brute_force(opts, t, list(range(n)), k, excl), k)
    if n == 1:
        assert t.parent[0] == -1


def test_orig_indices_mode():
    opts = O.Options(O.F64, O.MORTON, return_orig=True)
    x, y, z = gen("uniform", 200, O.F64, seed=2)
    t = O.build_bvh(opts, x, y, z)
    idx, dist = O.self_knn(opts, t, 8, True)
    # neighbours are input indices: recompute distances from the input arrays
    for q in range(0, 200, 13):
        src = t.orig_idx[q + 199]
        for j in range(8):
            o = int(idx[q, j])
            d = (x[src] - x[o]) ** 2 + (y[src] - y[o]) ** 2 + (z[src] - z[o]) ** 2
            assert abs(d - dist[q, j]) <= 1e-12 * max(d, 1.0)


def test_int_overflow_limit_raises():
    opts = O.Options(O.F64, O.MORTON)
    # only the size check is exercised: the arrays are never read when n is rejected
    with pytest.raises(RuntimeError):
        import ctypes
        x = np.zeros(1)
        t = O.Tree(1, O.F64)
        ct = t.c()
        rc = O.lib().ora_build_bvh(ctypes.byref(opts.c()), x.ctypes.data_as(ctypes.c_void_p),
                                   x.ctypes.data_as(ctypes.c_void_p), x.ctypes.data_as(ctypes.c_void_p),
                                   ctypes.c_int64(2 ** 30 + 5), None, None, None, None, None, ctypes.byref(ct),
                                   None, None, None)
        if rc == 2:
            raise RuntimeError("n > INT_MAX / 2")
