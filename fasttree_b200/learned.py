"""Learned radius bound for self-kNN (ft_bound_* / ft_self_knn_learned in the C ABI).

A 12 -> 64 -> 64 -> 1 GELU network predicts each self query's log2 k-th-neighbour distance
from cheap tree features; (inflation x prediction)^2 is the query's pruning bound in the fast
walk, and queries whose bound proves too small are rerun by the reference traversal, so the
output is bit-identical to self_knn_query's.  Training, inference and the features run in the
library's own CUDA kernels; this module only moves tensors.
"""
from __future__ import annotations

import ctypes
from typing import Optional

import numpy as np
import torch

from . import capi
from .capi import lib
from .hlbvh import (Context, TreeSoA, _alloc_knn_out, _as_coord, _call, _ptr, _qopts, _rows, _stream_handle,
                    build_bvh, dist_torch_dtype, particles, self_knn_query, self_knn_query_subset)

N_FEATURES = 12
N_PARAMS = 5057
FEATURE_NAMES = ["anc2_log2_diag", "anc4_log2_diag", "anc6_log2_diag", "anc8_log2_diag",
                 "prefix_4w_log2_count", "prefix_2w_log2_count", "prefix_1w_log2_count", "prefix_half_w_log2_count",
                 "leaf_depth_minus_log2_n", "log2_k", "window_kth_log2", "window_half_k_log2"]


def features(ctx: Context, tree: TreeSoA, k: int, leaf_ids=None, stream=None) -> torch.Tensor:
    """(num, 12) float32 features of self queries (every leaf, or leaf_ids)."""
    num = tree.num_leaves if leaf_ids is None else len(leaf_ids)
    out = torch.empty((num, N_FEATURES), dtype=torch.float32, device=f"cuda:{ctx.device}")
    _call(lib().ft_bound_features(ctx.handle, tree.c, _ptr(leaf_ids), num, int(k), _ptr(out) if num else None,
                                  _stream_handle(stream)))
    return out


def targets(ctx: Context, idx: torch.Tensor, dist: torch.Tensor, k: int, stream=None) -> torch.Tensor:
    """0.5 log2 of each row's k-th distance (NaN for rows with fewer than k neighbours)."""
    num = idx.numel() // k
    out = torch.empty(num, dtype=torch.float32, device=idx.device)
    _call(lib().ft_bound_targets(ctx.handle, _ptr(idx), _ptr(dist), num, int(k), _ptr(out),
                                 _stream_handle(stream)))
    return out


class BoundModel:
    """The network: fp32 master weights with bfloat16 copies, input / target standardisation."""

    def __init__(self, ctx: Context, seed: int = 0):
        self.ctx = ctx
        h = ctypes.c_void_p()
        self._h = None
        _call(lib().ft_bound_model_create(ctx.handle, ctypes.c_uint64(seed), ctypes.byref(h)))
        self._h = h
        self.norm = None

    @property
    def params(self) -> np.ndarray:
        p = np.zeros(N_PARAMS, np.float32)
        _call(lib().ft_bound_model_get_params(self.ctx.handle, self._h, p.ctypes.data))
        return p

    @params.setter
    def params(self, p):
        p = np.ascontiguousarray(p, np.float32)
        assert p.shape == (N_PARAMS,)
        _call(lib().ft_bound_model_set_params(self.ctx.handle, self._h, p.ctypes.data))

    def set_norm(self, mean, std, target_mean: float, target_std: float):
        mean = np.ascontiguousarray(mean, np.float32)
        std = np.ascontiguousarray(std, np.float32)
        _call(lib().ft_bound_model_set_norm(self.ctx.handle, self._h, mean.ctypes.data, std.ctypes.data,
                                            ctypes.c_float(target_mean), ctypes.c_float(target_std)))
        self.norm = (mean.copy(), std.copy(), float(target_mean), float(target_std))

    def fit_norm(self, feats: torch.Tensor, tgt: torch.Tensor):
        """Standardisation from a training set (the network's target is the residual
        log2 d_k - feature 10)."""
        f = feats.double()
        t = tgt.double() - f[:, 10]
        self.set_norm(f.mean(0).cpu().numpy(), f.std(0).cpu().numpy(), float(t.mean()), float(t.std()))

    def gradient(self, feats: torch.Tensor, tgt: torch.Tensor, stream=None):
        """(gradient, loss) of the mean squared error over all rows, without an update."""
        g = np.zeros(N_PARAMS, np.float32)
        loss = np.zeros(1, np.float32)
        _call(lib().ft_bound_model_gradient(self.ctx.handle, self._h, _ptr(feats), _ptr(tgt), len(tgt),
                                            g.ctypes.data, loss.ctypes.data, _stream_handle(stream)))
        return g, float(loss[0])

    def fit(self, feats: torch.Tensor, tgt: torch.Tensor, steps: int = 2000, batch: int = 8192, lr: float = 3e-3,
            seed: int = 0, record_loss: bool = True, stream=None) -> Optional[np.ndarray]:
        losses = np.zeros(max(steps, 1), np.float32) if record_loss else None
        _call(lib().ft_bound_model_fit(self.ctx.handle, self._h, _ptr(feats), _ptr(tgt), len(tgt), int(steps),
                                       int(batch), ctypes.c_float(lr), ctypes.c_uint64(seed),
                                       losses.ctypes.data if record_loss else None, _stream_handle(stream)))
        return losses[:steps] if record_loss else None

    def predict(self, feats: torch.Tensor, inflation: float = 1.15, want_bound: bool = False, stream=None):
        """Predicted log2 k-th distance per row, and optionally the bound in distance units."""
        n = feats.shape[0]
        dev = feats.device
        pred = torch.empty(n, dtype=torch.float32, device=dev)
        bound = torch.empty(n, dtype=dist_torch_dtype(self.ctx.coord), device=dev) if want_bound else None
        _call(lib().ft_bound_model_predict(self.ctx.handle, self._h, _ptr(feats), n, ctypes.c_float(inflation),
                                           _ptr(pred), _ptr(bound), _stream_handle(stream)))
        return (pred, bound) if want_bound else pred

    def free(self):
        if getattr(self, "_h", None):
            lib().ft_bound_model_destroy(self.ctx.handle, self._h)
            self._h = None

    def __del__(self):
        try:
            self.free()
        except Exception:
            pass


def training_set(ctx: Context, x, y, z, k: int, stream=None, max_samples: int = 0, seed: int = 0):
    """(features, targets) of the leaves of a training draw: the exact self-kNN's k-th
    distances and the features of the same queries.  Every leaf, or (max_samples > 0 and fewer
    than the draw's points) that many leaves drawn at random with the seed: a draw as large as
    the workload it serves keeps the workload's tree and density while the training set stays
    small."""
    n = len(x)
    tree = TreeSoA(ctx, n)
    build_bvh(ctx, particles(x, y, z), tree, stream=stream)
    ids = None
    if 0 < max_samples < n:
        g = torch.Generator(device="cpu").manual_seed(int(seed))
        ids = torch.randperm(n, generator=g)[:max_samples].sort().values.to(torch.int32).to(f"cuda:{ctx.device}")
        idx, dist = self_knn_query_subset(ctx, tree, ids, k, max_k=max(32, k), method="fast", stream=stream)
    else:
        idx, dist = self_knn_query(ctx, tree, k, max_k=max(32, k), method="fast", stream=stream)
    tgt = targets(ctx, idx.reshape(-1), dist.reshape(-1), k, stream)
    f = features(ctx, tree, k, leaf_ids=ids, stream=stream)
    del idx, dist
    tree.free()
    ok = torch.isfinite(tgt)
    return f[ok].contiguous(), tgt[ok].contiguous()


def training_set_batched(ctx: Context, set_offsets, x, y, z, k: int, stream=None):
    """(features, targets) of every leaf of a batched training draw (BatchedSets): each set's
    exact self-kNN and its features on its own tree."""
    from .hlbvh import BatchedSets
    off = np.asarray(set_offsets, np.int64)
    b = BatchedSets(ctx, int(off[-1]), len(off) - 1)
    b.build(off, x, y, z, stream=stream)
    idx, dist = b.self_knn(k, max_k=max(32, k), method="fast", stream=stream)
    tgt = targets(ctx, idx.reshape(-1), dist.reshape(-1), k, stream)
    f = b.bound_features(k, stream=stream)
    del idx, dist
    b.free()
    ok = torch.isfinite(tgt)
    return f[ok].contiguous(), tgt[ok].contiguous()


def train_bound_batched(ctx: Context, set_offsets, x, y, z, k: int, steps: int = 2000, batch: int = 8192,
                        lr: float = 3e-3, seed: int = 0, stream=None):
    """Network trained on a batched draw's exact self-kNN (training_set_batched)."""
    f, t = training_set_batched(ctx, set_offsets, x, y, z, k, stream)
    m = BoundModel(ctx, seed)
    m.fit_norm(f, t)
    losses = m.fit(f, t, steps=steps, batch=batch, lr=lr, seed=seed + 1, stream=stream)
    return m, losses


def train_bound(ctx: Context, x, y, z, k: int, steps: int = 2000, batch: int = 8192, lr: float = 3e-3,
                seed: int = 0, stream=None, max_samples: int = 0):
    """Network trained on a draw's exact self-kNN (features / targets from training_set)."""
    f, t = training_set(ctx, x, y, z, k, stream, max_samples=max_samples, seed=seed + 7)
    m = BoundModel(ctx, seed)
    m.fit_norm(f, t)
    losses = m.fit(f, t, steps=steps, batch=batch, lr=lr, seed=seed + 1, stream=stream)
    return m, losses


def self_knn_query_learned(ctx: Context, tree: TreeSoA, model: BoundModel, k: int, results=None,
                           result_dists=None, exclude_self=True, inflation: float = 1.15, leaf_ids=None,
                           max_k: int = 32, stream=None):
    """self_knn_query with the learned bound (same output); asynchronous."""
    num = tree.num_leaves if leaf_ids is None else len(leaf_ids)
    if results is None:
        results, result_dists = _alloc_knn_out(ctx, num, k)
    _call(lib().ft_self_knn_learned(ctx.handle, tree.c, model._h, _ptr(leaf_ids), num, int(k),
                                    int(bool(exclude_self)), ctypes.c_float(inflation), _ptr(results),
                                    _ptr(result_dists), ctypes.byref(_qopts(max_k, 1)), _stream_handle(stream)))
    return _rows(results, num, k), _rows(result_dists, num, k)


def features_points(ctx: Context, tree: TreeSoA, qx, qy, qz, k: int, stream=None) -> torch.Tensor:
    """(nq, 12) float32 features of external query points."""
    x, y, z = (torch.as_tensor(_as_coord(a, ctx.coord)).to(f"cuda:{ctx.device}") for a in (qx, qy, qz))
    nq = len(x)
    out = torch.empty((nq, N_FEATURES), dtype=torch.float32, device=f"cuda:{ctx.device}")
    _call(lib().ft_bound_features_points(ctx.handle, tree.c, _ptr(x), _ptr(y), _ptr(z), nq, int(k),
                                         _ptr(out) if nq else None, _stream_handle(stream)))
    return out


def knn_query_learned(ctx: Context, tree: TreeSoA, model: BoundModel, qx, qy, qz, k: int, results=None,
                      result_dists=None, inflation: float = 1.3, max_k: int = 256, stream=None):
    """knn_query<MAXK> with the learned bound (same output as knn_query); blocking."""
    x, y, z = (_as_coord(a, ctx.coord) for a in (qx, qy, qz))
    nq = len(x)
    if results is None:
        results, result_dists = _alloc_knn_out(ctx, nq, k)
    _call(lib().ft_knn_learned(ctx.handle, tree.c, model._h, _ptr(x), _ptr(y), _ptr(z), nq, int(k),
                               ctypes.c_float(inflation), _ptr(results), _ptr(result_dists),
                               ctypes.byref(_qopts(max_k, 1)), _stream_handle(stream)))
    return _rows(results, nq, k), _rows(result_dists, nq, k)
