"""CPU oracle of the learned radius bound -- test infrastructure only (tests/ use it as the
checker of the GPU kernels in fasttree_b200/csrc/ft_learned.cu; nothing in the product
imports it).

The learned bound has no counterpart in the reference (sparxastronomy/fasttree): it is this
project's own addition, defined by its kernels' documentation.  This module restates it in
numpy:

  * features(): the 12 per-query features from a CPU-built tree (oracle.build_bvh), with the
    same definitions (ancestor box diagonals, SFC-prefix counts at window-relative levels,
    depth - log2 n, log2 k, SFC-window k-th distances) and the walk's distance formulas;
  * forward() / backward(): the 12 -> 64 -> 64 -> 1 GELU network in float64 with the GPU's
    bfloat16 rounding points (standardised inputs, weights and hidden activations);
  * adam(): one bias-corrected Adam step.
"""
from __future__ import annotations

import math

import numpy as np

from . import oracle as O

N_FEATURES, N_HID = 12, 64
OFF_W1, OFF_B1 = 0, 768
OFF_W2, OFF_B2 = 832, 4928
OFF_W3, OFF_B3 = 4992, 5056
N_PARAMS = 5057


def bf16(a) -> np.ndarray:
    """Round to bfloat16 (round to nearest even), returned as float32."""
    f = np.asarray(a, np.float32)
    u = f.view(np.uint32).astype(np.uint64)
    r = ((u + 0x7FFF + ((u >> 16) & 1)) & 0xFFFF0000).astype(np.uint32)
    return r.view(np.float32)


# ----------------------------------------------------------------------------------------
# Features
# ----------------------------------------------------------------------------------------
def _bits(coord):
    return 42 if coord == O.U64 else 21


def _dist_shift(coord):
    return 11 if coord == O.U64 else 0


def _leaf_dist(opts: O.Options, tree: O.Tree, i: np.ndarray, j: np.ndarray) -> np.ndarray:
    """Squared distance between sorted leaves i and j in the walk's units (float64)."""
    n = tree.n
    si, sj = i + n - 1, j + n - 1
    coord = opts.coord
    arrs = [(tree.min_x[si], tree.min_x[sj]), (tree.min_y[si], tree.min_y[sj]), (tree.min_z[si], tree.min_z[sj])]
    if coord in (O.F32, O.F64):
        dt = np.float32 if coord == O.F32 else np.float64
        s = None
        for a, b in arrs:
            a, b = a.astype(dt), b.astype(dt)
            d = np.maximum(b - a, np.maximum(dt(0), a - b))
            s = d * d if s is None else s + d * d
        return s.astype(np.float64)
    B, sh = _bits(coord), _dist_shift(coord)
    mask = (1 << B) - 1
    s = np.zeros(len(i), np.float64)
    for a, b in arrs:
        a = a.astype(np.uint64) & np.uint64(mask)
        b = b.astype(np.uint64) & np.uint64(mask)
        d = np.where(a > b, a - b, b - a).astype(np.uint64)
        if opts.periodic:
            d = np.minimum(d, np.uint64(1 << B) - d)
        g = (d >> np.uint64(sh)).astype(np.float64)
        s += g * g
    return s


def _common_features(opts: O.Options, tree: O.Tree, k: int, ranks: np.ndarray, window) -> np.ndarray:
    """Features of queries placed at sorted-leaf `ranks`; window(r_i, r) gives the squared
    distances (float32 values) from query r_i to its SFC-window leaves."""
    n = tree.n
    q = len(ranks)
    F = np.zeros((q, N_FEATURES), np.float64)
    isf = opts.coord in (O.F32, O.F64)
    unit = 2.0 ** -_dist_shift(opts.coord)
    lf = 2.0 ** -60 if isf else 0.5
    par = tree.parent.astype(np.int64)

    def diag(a):
        out = [(hi[a] - lo[a]).astype(np.float64)  # unsigned difference, hi >= lo in a box
               for lo, hi in ((tree.min_x, tree.max_x), (tree.min_y, tree.max_y), (tree.min_z, tree.max_z))]
        return np.sqrt(out[0] ** 2 + out[1] ** 2 + out[2] ** 2)

    slot = ranks + n - 1
    for r in range(q):
        node, depth, anc = int(slot[r]), 0, []
        while node != 0 and depth < 4096:
            p = int(par[node])
            if p < 0 or p >= n - 1:
                break
            node, depth = p, depth + 1
            if depth % 2 == 0 and depth <= 8:
                anc.append(node)
        anc = anc + [0] * (4 - len(anc))
        F[r, 0:4] = np.log2(np.maximum(diag(np.array(anc)) * unit, lf))
        F[r, 8] = depth - math.log2(n)
    F[:, 9] = math.log2(k)

    # SFC-window k-th distances
    kk = min(k, 64)
    lwk = np.zeros(q)
    for r_i, r in enumerate(ranks):
        d = np.sort(np.asarray(window(r_i, int(r)), np.float32).astype(np.float64))
        if len(d) == 0:
            wk = wk2 = 0.0
        else:
            m = min(kk, len(d))
            wk = d[m - 1]
            wk2 = d[min((kk + 1) // 2, m) - 1]
        lwk[r_i] = 0.5 * math.log2(max(wk, lf * lf))
        F[r_i, 10] = lwk[r_i]
        F[r_i, 11] = 0.5 * math.log2(max(wk2, lf * lf))

    # SFC-prefix counts at the levels whose cells are 4, 2, 1, 1/2 window distances wide
    wide = opts.coord == O.U64
    lv = 20 if wide else 21
    if isf:
        dt = np.float32 if opts.coord == O.F32 else np.float64
        side = max(float(dt(tree.max_x[0]) - dt(tree.min_x[0])), float(dt(tree.max_y[0]) - dt(tree.min_y[0])),
                   float(dt(tree.max_z[0]) - dt(tree.min_z[0])))
        base = math.log2(max(side, lf))
    else:
        base = float(_bits(opts.coord))
    lw = lwk + _dist_shift(opts.coord)
    keys = (tree.sorted_hi if wide else tree.sorted_lo)[:n].astype(np.uint64)
    for c in range(4):
        Ls = np.clip(np.floor(base - lw - (2 - c)), 0, lv).astype(np.int64)
        for L in np.unique(Ls):
            p = 3 * int(L)
            pre = np.zeros(n, np.uint64) if p == 0 else keys >> np.uint64((62 if wide else 63) - p)
            _, inv, cnt = np.unique(pre, return_inverse=True, return_counts=True)
            m = Ls == L
            F[m, 4 + c] = np.log2(cnt[inv][ranks[m]].astype(np.float64))
    return F.astype(np.float32)


def features(opts: O.Options, tree: O.Tree, k: int, leaf_ids=None) -> np.ndarray:
    """Features of self queries (every leaf, or the sorted-leaf ranks leaf_ids): the window is
    ranks r-k .. r+k without the query's own leaf."""
    n = tree.n
    ranks = np.arange(n) if leaf_ids is None else np.asarray(leaf_ids, np.int64)

    def window(_, r):
        js = np.array([j for j in range(max(0, r - k), min(n - 1, r + k) + 1) if j != r], np.int64)
        return _leaf_dist(opts, tree, np.full(len(js), r), js).astype(np.float32) if len(js) else []

    return _common_features(opts, tree, k, ranks, window)


def seed_ranks(opts: O.Options, tree: O.Tree, qx, qy, qz, bbox) -> np.ndarray:
    """Each external point's SFC rank: the first sorted key >= the point's key (keys encoded
    with the tree's build box), as an insertion point in [0, n]."""
    hi, lo = O.sfc_encode(opts, qx, qy, qz, bbox)
    n = tree.n
    shi, slo = tree.sorted_hi[:n].astype(object), tree.sorted_lo[:n].astype(object)
    comp = [(int(a) << 64) | int(b) for a, b in zip(shi, slo)]
    import bisect
    return np.array([bisect.bisect_left(comp, (int(a) << 64) | int(b)) for a, b in zip(hi, lo)], np.int64)


def features_points(opts: O.Options, tree: O.Tree, k: int, qx, qy, qz, bbox) -> np.ndarray:
    """Features of external query points: each point stands at its seed rank r (clamped to the
    last leaf), the ancestor and prefix features are those of the leaf there, and the window
    is the leaves r-k .. r+k-1 seen from the point (point-to-leaf distances)."""
    n = tree.n
    dt = O.NP_COORD[opts.coord]
    qx, qy, qz = (np.asarray(a, dt) for a in (qx, qy, qz))
    ranks = np.minimum(seed_ranks(opts, tree, qx, qy, qz, bbox), n - 1)

    def window(r_i, r):
        p3 = np.array([qx[r_i], qy[r_i], qz[r_i]], dt)
        out = []
        for j in range(max(0, r - k), min(n - 1, r + k - 1) + 1):
            s = j + n - 1
            box = np.array([tree.min_x[s], tree.max_x[s], tree.min_y[s], tree.max_y[s], tree.min_z[s],
                            tree.max_z[s]], dt)
            out.append(float(O.point_dist(opts, p3, box)))
        return out

    return _common_features(opts, tree, k, ranks, window)


def targets(opts: O.Options, dist: np.ndarray, idx: np.ndarray, k: int) -> np.ndarray:
    lf2 = 2.0 ** -120 if opts.coord in (O.F32, O.F64) else 0.25
    d = dist[:, k - 1].astype(np.float64)
    t = 0.5 * np.log2(np.maximum(d, lf2))
    t[idx[:, k - 1] == np.iinfo(np.uint64).max] = np.nan
    return t.astype(np.float32)


# ----------------------------------------------------------------------------------------
# Network
# ----------------------------------------------------------------------------------------
_erf = np.vectorize(math.erf)


def gelu(z):
    return 0.5 * z * (1.0 + _erf(z / math.sqrt(2.0)))


def gelu_grad(z):
    return 0.5 * (1.0 + _erf(z / math.sqrt(2.0))) + z * np.exp(-0.5 * z * z) / math.sqrt(2.0 * math.pi)


def unpack(params):
    p = bf16(params).astype(np.float64)
    return (p[OFF_W1:OFF_B1].reshape(N_HID, N_FEATURES), p[OFF_B1:OFF_W2], p[OFF_W2:OFF_B2].reshape(N_HID, N_HID),
            p[OFF_B2:OFF_W3], p[OFF_W3:OFF_B3], p[OFF_B3])


def _round(a, rounding):
    return bf16(a).astype(np.float64) if rounding else np.asarray(a, np.float64)


def standardise(raw, norm, rounding=True):
    """norm = (mean[12], std[12], target_mean, target_std) as the library stores it."""
    mean, std, _, _ = norm
    isd = (np.float32(1.0) / np.maximum(np.asarray(std, np.float32), np.float32(1e-3))).astype(np.float32)
    x = (np.asarray(raw, np.float32) - np.asarray(mean, np.float32)) * isd
    return _round(x, rounding)


def forward(params, raw, norm, rounding=True):
    """rounding=False keeps every value in float64 (for derivative checks of the oracle)."""
    W1, b1, W2, b2, w3, b3 = unpack(params) if rounding else unpack_exact(params)
    x = standardise(raw, norm, rounding)
    z1 = x @ W1.T + b1
    h1 = _round(gelu(z1), rounding)
    z2 = h1 @ W2.T + b2
    h2 = _round(gelu(z2), rounding)
    y = h2 @ w3 + b3
    return y, (x, z1, h1, z2, h2)


def unpack_exact(params):
    p = np.asarray(params, np.float64)
    return (p[OFF_W1:OFF_B1].reshape(N_HID, N_FEATURES), p[OFF_B1:OFF_W2], p[OFF_W2:OFF_B2].reshape(N_HID, N_HID),
            p[OFF_B2:OFF_W3], p[OFF_W3:OFF_B3], p[OFF_B3])


def predict_log2(params, raw, norm):
    """log2 k-th distance: window distance (feature 10) plus the predicted residual."""
    y, _ = forward(params, raw, norm)
    t_mean, t_std = norm[2], max(norm[3], 1e-3)
    return np.asarray(raw, np.float64)[:, 10] + y * t_std + t_mean


def loss_and_grad(params, raw, tgt, norm, rounding=True):
    """Mean squared error of the standardised residual target (log2 d_k - feature 10) and its
    gradient w.r.t. the weights.  The gradient treats the bfloat16 roundings as identity (the
    straight-through rule the GPU kernels follow)."""
    t_mean, t_std = norm[2], max(norm[3], 1e-3)
    res = np.asarray(tgt, np.float32) - np.asarray(raw, np.float32)[:, 10]
    t = (res.astype(np.float64) - t_mean) / t_std
    W1, b1, W2, b2, w3, b3 = unpack(params) if rounding else unpack_exact(params)
    y, (x, z1, h1, z2, h2) = forward(params, raw, norm, rounding)
    B = len(t)
    dy = 2.0 * (y - t) / B
    g = np.zeros(N_PARAMS, np.float64)
    g[OFF_W3:OFF_B3] = dy @ h2
    g[OFF_B3] = dy.sum()
    dz2 = dy[:, None] * w3[None, :] * gelu_grad(z2)
    g[OFF_W2:OFF_B2] = (dz2.T @ h1).reshape(-1)
    g[OFF_B2:OFF_W3] = dz2.sum(0)
    dz1 = (dz2 @ W2) * gelu_grad(z1)
    g[OFF_W1:OFF_B1] = (dz1.T @ x).reshape(-1)
    g[OFF_B1:OFF_W2] = dz1.sum(0)
    return float(np.mean((y - t) ** 2)), g


def adam(params, m, v, grad, step, lr, b1=0.9, b2=0.999, eps=1e-8):
    m = b1 * m + (1 - b1) * grad
    v = b2 * v + (1 - b2) * grad * grad
    c1, c2 = 1 - b1 ** step, 1 - b2 ** step
    return params - lr * (m / c1) / (np.sqrt(v / c2) + eps), m, v
