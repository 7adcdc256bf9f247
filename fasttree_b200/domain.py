"""Domain decomposition front end: particles spread over ranks (one process per GPU) are
redistributed so that each rank owns one contiguous stretch of the space-filling curve, then
each rank receives copies (ghosts) of its neighbours' particles near its boundary.

The same five phases as the reference's MPI front end (src/domain_decomposition.hpp), with
torch.distributed collectives in place of MPI -- NCCL over NVLink / NVSwitch when the process
group is on GPUs, gloo on CPUs -- and this library's SFC encoding on the GPU:

1. get_global_bounding_box (src/domain_decomposition.hpp:69-155): the local box, then a
   min / max all-reduce, so every rank quantises with the same box.
2. get_global_histogram (168-220): the top m bits of every local key, counted per bucket,
   summed over ranks.
3. generate_splitters (227-264): P contiguous bucket ranges of about N / P particles each,
   computed identically on every rank; or get_deterministic_splitters (306-400): 128
   stride samples of each rank's sorted keys, pooled, and P - 1 key splitters taken from them.
4. redistribute_particles (410-682): each particle's destination rank by binary search over
   the splitters, a stable order by destination, then an all-to-all of the counts and one of
   each attribute.
5. exchange_halos (687-1030): every rank's box all-gathered; a rank sends to each rank whose
   box, widened by h_max, overlaps its own, the particles inside that widened box, marked as
   ghosts; the received ghosts are appended after the local particles.

Orders the reference leaves to its device sort or to atomics are fixed here: particles bound
for one rank keep their input order (the reference's sort by destination is not stable), and
the particles sent to one neighbour go in input order (the reference appends them with an
atomic counter).  The histogram and key arithmetic, the splitter rules, the empty-rank box of
the halo exchange (all zeros) and its unsigned wrap-around for integer positions follow the
reference as written.
"""
from __future__ import annotations

from typing import Optional

import numpy as np

from .capi import F32, F64, U32, U64, MORTON

S_SAMPLES = 128  # stride samples per rank (src/domain_decomposition.hpp:313)


def _torch():
    import torch
    return torch


def _dist():
    import torch.distributed as dist
    return dist


def _device(ctx, group=None):
    """The device a collective of `group` works on: the context's GPU for NCCL, else the CPU."""
    torch = _torch()
    backend = _dist().get_backend(group)
    return torch.device(f"cuda:{ctx.device}") if backend == "nccl" else torch.device("cpu")


def _np_coord(coord):
    return {F32: np.float32, F64: np.float64, U32: np.uint32, U64: np.uint64}[coord]


def _host(a, dtype=None):
    """numpy copy of an array or tensor."""
    torch = _torch()
    if isinstance(a, torch.Tensor):
        a = a.detach().cpu().numpy()
    a = np.asarray(a)
    return a if dtype is None else a.astype(dtype, copy=False)


def _as_particles(p, coord):
    """Host SoA arrays (x, y, z, id, is_ghost) of particles p; missing ids are 0..n-1 and
    missing ghost flags 0 (normalize_particles, src/domain_decomposition.hpp:273-293)."""
    dt = _np_coord(coord)
    x, y, z = (np.ascontiguousarray(_host(a, dt)) for a in (p.pos_x, p.pos_y, p.pos_z))
    n = len(x)
    ids = np.arange(n, dtype=np.uint32) if p.id is None else np.ascontiguousarray(_host(p.id, np.uint32))
    gh = np.zeros(n, np.int8) if p.is_ghost is None else np.ascontiguousarray(_host(p.is_ghost, np.int8))
    if len(ids) < n:
        ids = np.concatenate([ids, np.arange(len(ids), n, dtype=np.uint32)])
    if len(gh) < n:
        gh = np.concatenate([gh, np.zeros(n - len(gh), np.int8)])
    return x, y, z, ids[:n], gh[:n]


# ---- order-preserving 64-bit images (collectives reduce signed integers or floats) ----
def _to_ord(a: np.ndarray, coord) -> np.ndarray:
    if coord in (F32, F64):
        return a.astype(np.float64)
    return (a.astype(np.uint64) ^ np.uint64(1 << 63)).view(np.int64)


def _from_ord(a: np.ndarray, coord) -> np.ndarray:
    if coord in (F32, F64):
        return a.astype(_np_coord(coord))
    return (a.view(np.uint64) ^ np.uint64(1 << 63)).astype(_np_coord(coord))


def _identity_box(coord) -> np.ndarray:
    """{type_identity_min, type_identity_max} per axis (src/hlbvh.hpp:46-69)."""
    if coord in (F32, F64):
        big = np.finfo(_np_coord(coord)).max
        lo, hi = big, -big
    else:
        lo, hi = np.iinfo(_np_coord(coord)).max, 0
    return np.array([lo, hi, lo, hi, lo, hi], _np_coord(coord))


def get_global_bounding_box(ctx, p, local_bbox=None, group=None):
    """Phase 1: the box of every rank's particles (src/domain_decomposition.hpp:69-155).  The
    local box comes from compute_bbox on this rank's particles (or `local_bbox`, 6 values
    min_x, max_x, ...); a rank without particles contributes the identity box."""
    from .hlbvh import BoundingBox, compute_bbox
    torch, dist = _torch(), _dist()
    coord = ctx.coord
    n = len(p.pos_x)
    if n == 0:
        box = _identity_box(coord)
    elif local_bbox is not None:
        box = np.asarray(_host(local_bbox), _np_coord(coord))
    else:
        box = compute_bbox(ctx, p.pos_x, p.pos_y, p.pos_z)
    dev = _device(ctx, group)
    o = _to_ord(box, coord)
    lo = torch.as_tensor(o[0::2].copy(), device=dev)
    hi = torch.as_tensor(o[1::2].copy(), device=dev)
    dist.all_reduce(lo, op=dist.ReduceOp.MIN, group=group)
    dist.all_reduce(hi, op=dist.ReduceOp.MAX, group=group)
    lo, hi = _from_ord(lo.cpu().numpy(), coord), _from_ord(hi.cpu().numpy(), coord)
    return BoundingBox(lo[0], hi[0], lo[1], hi[1], lo[2], hi[2])


# ---- keys ----
def sfc_keys(ctx, p, global_bbox, keys=None) -> np.ndarray:
    """This rank's SFC keys in the reference's sfc_key layout, shape (n, words): sfc_encode with
    the global box (this library's encoding kernel), or the `keys` given."""
    from .hlbvh import ref_key_dtype, sfc_encode
    dt, words = ref_key_dtype(ctx)
    if keys is not None:
        return np.asarray(_host(keys), dt).reshape(-1, words)
    if len(p.pos_x) == 0:
        return np.zeros((0, words), dt)
    return sfc_encode(ctx, p.pos_x, p.pos_y, p.pos_z, bbox=global_bbox).reshape(-1, words)


def _key_words(ctx, keys: np.ndarray):
    """(high, low) uint64 words of each key in sort order: Morton and 63-bit Peano-Hilbert
    keys have one sort word (to_sort_key, src/sfc.peano_hilbert.hpp:286-294); 126-bit keys
    compare by (is, ls) (hs is zero)."""
    if ctx.sfc == MORTON:
        lo = keys[:, 0].astype(np.uint64)
        return np.zeros_like(lo), lo
    if ctx.coord == U64:
        return keys[:, 1].astype(np.uint64), keys[:, 2].astype(np.uint64)
    lo = (keys[:, 1].astype(np.uint64) << np.uint64(32)) | keys[:, 2].astype(np.uint64)
    return np.zeros_like(lo), lo


def bucket_ids(ctx, keys: np.ndarray, m: int = 20) -> np.ndarray:
    """extract_bucket_id (src/sfc.peano_hilbert.hpp:308-320): the top m bits of a 63-bit key;
    for 126-bit keys the middle word shifted by 63 - m (its 62 bits give m - 1 bucket bits)."""
    hi, lo = _key_words(ctx, keys)
    if ctx.coord == U64 and ctx.sfc != MORTON:
        return (hi >> np.uint64(max(63 - m, 0))).astype(np.uint32)
    return (lo >> np.uint64(max(63 - m, 0))).astype(np.uint32)


def get_global_histogram(ctx, p, global_bbox, m: int = 20, keys=None, group=None) -> np.ndarray:
    """Phase 2 (src/domain_decomposition.hpp:168-220): particles per top-m-bit SFC bucket,
    summed over ranks (the sum runs on the process group's device)."""
    torch, dist = _torch(), _dist()
    b = bucket_ids(ctx, sfc_keys(ctx, p, global_bbox, keys), m)
    hist = np.bincount(b.astype(np.int64), minlength=1 << m)[: 1 << m].astype(np.int64)
    t = torch.as_tensor(hist, device=_device(ctx, group))
    dist.all_reduce(t, op=dist.ReduceOp.SUM, group=group)
    return t.cpu().numpy()


def generate_splitters(global_hist, P: int, m: int = 20) -> np.ndarray:
    """Phase 3 (src/domain_decomposition.hpp:227-264): bucket boundaries of P contiguous ranges,
    splitter r at the first bucket where the running count reaches r * (N / P)."""
    hist = np.asarray(global_hist, np.int64)
    num_buckets = 1 << m
    total = int(hist[:num_buckets].sum())
    target = total // P
    spl = np.zeros(P + 1, np.uint32)
    run, r = 0, 1
    cum = np.cumsum(hist[:num_buckets])
    # the first bucket at which the running count reaches target * r, for r = 1 .. P-1
    for r in range(1, P):
        j = int(np.searchsorted(cum, target * r, side="left"))
        spl[r] = j if j < num_buckets else num_buckets
    spl[P] = num_buckets
    del run
    return spl


def _lex_sort_keys(hi: np.ndarray, lo: np.ndarray) -> np.ndarray:
    return np.lexsort((lo, hi))


def get_deterministic_splitters(ctx, p, global_bbox, keys=None, group=None) -> np.ndarray:
    """Phase 3, sampling form (src/domain_decomposition.hpp:306-400): 128 stride samples of
    each rank's sorted keys (the largest key when a rank has none), pooled over ranks; with
    V valid samples, splitter i is the sample at (i V) / P.  Returns (P + 1, 2) uint64 rows of
    (high, low) sort words; row 0 is the zero key and row P the largest key."""
    torch, dist = _torch(), _dist()
    P = dist.get_world_size(group)
    hi, lo = _key_words(ctx, sfc_keys(ctx, p, global_bbox, keys))
    n = len(lo)
    MAXW = np.uint64(0xFFFFFFFFFFFFFFFF)
    samp = np.full((S_SAMPLES, 2), MAXW, np.uint64)
    if n > 0:
        order = _lex_sort_keys(hi, lo)
        stride = n // S_SAMPLES
        at = np.minimum(np.arange(S_SAMPLES) * stride, n - 1)
        samp[:, 0], samp[:, 1] = hi[order[at]], lo[order[at]]
    dev = _device(ctx, group)
    mine = torch.as_tensor(samp.view(np.int64).copy(), device=dev)
    pooled = [torch.empty_like(mine) for _ in range(P)]
    dist.all_gather(pooled, mine, group=group)
    allv = np.concatenate([t.cpu().numpy().view(np.uint64) for t in pooled])
    allv = allv[_lex_sort_keys(allv[:, 0], allv[:, 1])]
    valid = int(np.sum(~((allv[:, 0] == MAXW) & (allv[:, 1] == MAXW))))
    spl = np.zeros((P + 1, 2), np.uint64)
    spl[P] = MAXW
    for i in range(1, P):
        if valid > 0:
            spl[i] = allv[min((i * valid) // P, valid - 1)]
    return spl


def destinations(ctx, keys: np.ndarray, rank_splitters, m: int = 20, sampling: bool = False) -> np.ndarray:
    """Destination rank of each key: the largest r in [0, P) with splitter r not above it
    (the binary searches of src/domain_decomposition.hpp:446-488)."""
    spl = np.asarray(rank_splitters)
    P = len(spl) - 1
    if not sampling:
        b = bucket_ids(ctx, keys, m).astype(np.int64)
        d = np.searchsorted(spl[:P].astype(np.int64), b, side="right") - 1
        return np.clip(d, 0, P - 1).astype(np.int64)
    hi, lo = _key_words(ctx, keys)
    d = np.zeros(len(lo), np.int64)
    for r in range(1, P):
        sh, sl = spl[r, 0], spl[r, 1]
        d += ((hi > sh) | ((hi == sh) & (lo >= sl))).astype(np.int64)
    return d


def _exchange(dev, parts, send_counts, group):
    """All-to-all of several attribute arrays (already in destination order) with the given
    per-rank counts; returns the received arrays (in source-rank order) and the counts."""
    torch, dist = _torch(), _dist()
    P = len(send_counts)
    sc = torch.as_tensor(np.asarray(send_counts, np.int64), device=dev)
    rc = torch.empty_like(sc)
    dist.all_to_all_single(rc, sc, group=group)
    recv_counts = rc.cpu().numpy().astype(np.int64)
    out = []
    for a in parts:
        a = np.ascontiguousarray(a)
        wire = a.view({1: np.int8, 4: np.int32, 8: np.int64}[a.dtype.itemsize])
        src = torch.as_tensor(wire, device=dev)
        dst = torch.empty(int(recv_counts.sum()), dtype=src.dtype, device=dev)
        dist.all_to_all_single(dst, src, [int(c) for c in recv_counts], [int(c) for c in send_counts],
                               group=group)
        out.append(dst.cpu().numpy().view(a.dtype))
    del P
    return out, recv_counts


def redistribute_particles(ctx, p, rank_splitters, global_bbox, m: int = 20, keys=None, sampling: bool = False,
                           group=None):
    """Phase 4 (src/domain_decomposition.hpp:410-682): every particle goes to the rank whose SFC
    range holds its key (bucket splitters from generate_splitters, or key splitters from
    get_deterministic_splitters with sampling=True).  Returns this rank's particles: those
    received from rank 0 first, then rank 1, ..., each source's in its input order."""
    from .hlbvh import particles
    dist = _dist()
    P = dist.get_world_size(group)
    x, y, z, ids, gh = _as_particles(p, ctx.coord)
    dest = destinations(ctx, sfc_keys(ctx, p, global_bbox, keys), rank_splitters, m, sampling)
    order = np.argsort(dest, kind="stable")
    send_counts = np.bincount(dest, minlength=P)[:P].astype(np.int64)
    (rx, ry, rz, rid, rgh), _ = _exchange(_device(ctx, group), [a[order] for a in (x, y, z, ids, gh)], send_counts,
                                          group)
    return particles(rx, ry, rz, rid, rgh)


def _local_box(x, y, z, coord) -> np.ndarray:
    """The halo exchange's local box: min / max of the positions, all zeros for no particles
    (src/domain_decomposition.hpp:700-722)."""
    if len(x) == 0:
        return np.zeros(6, _np_coord(coord))
    return np.array([x.min(), x.max(), y.min(), y.max(), z.min(), z.max()], _np_coord(coord))


def exchange_halos(ctx, p, h_max, group=None):
    """Phase 5 (src/domain_decomposition.hpp:687-1030): this rank's particles followed by
    ghosts (is_ghost = 1) -- the particles of other ranks inside this rank's box widened by
    h_max.  Box widening uses the coordinate type's own arithmetic (unsigned positions wrap)."""
    from .hlbvh import particles
    torch, dist = _torch(), _dist()
    P, rank = dist.get_world_size(group), dist.get_rank(group)
    coord = ctx.coord
    dt = _np_coord(coord)
    x, y, z, ids, gh = _as_particles(p, coord)
    dev = _device(ctx, group)
    box = _local_box(x, y, z, coord)
    mine = torch.as_tensor(_to_ord(box, coord).copy(), device=dev)
    boxes = [torch.empty_like(mine) for _ in range(P)]
    dist.all_gather(boxes, mine, group=group)
    boxes = [_from_ord(b.cpu().numpy(), coord) for b in boxes]
    h = dt(h_max)
    with np.errstate(over="ignore"):
        lo_me = box[0::2] - h
        hi_me = box[1::2] + h
    neighbours = []
    for r in range(P):
        b = boxes[r]
        if r == rank or b[0] > b[1]:
            continue
        if (lo_me[0] <= b[1] and hi_me[0] >= b[0] and lo_me[1] <= b[3] and hi_me[1] >= b[2] and lo_me[2] <= b[5]
                and hi_me[2] >= b[4]):
            neighbours.append(r)
    send_counts = np.zeros(P, np.int64)
    picked = []
    for r in neighbours:
        b = boxes[r]
        with np.errstate(over="ignore"):
            lo = b[0::2] - h
            hi = b[1::2] + h
        inside = ((x >= lo[0]) & (x <= hi[0]) & (y >= lo[1]) & (y <= hi[1]) & (z >= lo[2]) & (z <= hi[2]))
        sel = np.nonzero(inside)[0]
        send_counts[r] = len(sel)
        picked.append(sel)
    sel = np.concatenate(picked) if picked else np.zeros(0, np.int64)
    sends = [x[sel], y[sel], z[sel], ids[sel], np.ones(len(sel), np.int8)]
    (rx, ry, rz, rid, rgh), _ = _exchange(dev, sends, send_counts, group)
    return particles(np.concatenate([x, rx]), np.concatenate([y, ry]), np.concatenate([z, rz]),
                     np.concatenate([ids, rid]), np.concatenate([gh, rgh]))


def decompose(ctx, p, h_max=None, m: int = 20, sampling: bool = False, group=None, keys=None):
    """The whole front end on this rank: global box, splitters (histogram or sampling),
    redistribution and, with h_max, the halo exchange.  Returns (particles, global_bbox,
    splitters)."""
    dist = _dist()
    P = dist.get_world_size(group)
    bbox = get_global_bounding_box(ctx, p, group=group)
    if sampling:
        spl = get_deterministic_splitters(ctx, p, bbox, keys=keys, group=group)
    else:
        spl = generate_splitters(get_global_histogram(ctx, p, bbox, m, keys=keys, group=group), P, m)
    q = redistribute_particles(ctx, p, spl, bbox, m, keys=keys, sampling=sampling, group=group)
    if h_max is not None:
        q = exchange_halos(ctx, q, h_max, group=group)
    return q, bbox, spl
