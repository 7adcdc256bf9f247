"""Regenerates tests/golden/*.npz from the reference's own code compiled on the CPU.

    make -C oracle -f ref.mk && python tests/golden/make_golden.py

Each fixture holds one compile-time configuration of the reference: a seeded clustered input
(the shape of test/test_self_knn.cpp:291-330), the tree build_bvh makes from it, the sorted
keys, self_knn_query / self_knn_query_subset, knn_query (register and merge heap tiers) and
range_query outputs.  Small enough to commit; the reference sources are not needed to use
them.
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from oracle import oracle as O  # noqa: E402
from oracle import reference as R  # noqa: E402
from tests.gpu_util import gen, radius, to_coord  # noqa: E402

CASES = {
    "f32_morton": (O.F32, O.MORTON, False, False),
    "f64_morton": (O.F64, O.MORTON, False, False),
    "f32_ph": (O.F32, O.PEANO_HILBERT, False, False),
    "f64_ph": (O.F64, O.PEANO_HILBERT, False, False),
    "u32_ph": (O.U32, O.PEANO_HILBERT, False, False),
    "u32_ph_per": (O.U32, O.PEANO_HILBERT, True, False),
    "u64_ph": (O.U64, O.PEANO_HILBERT, False, False),
    "u64_ph_per": (O.U64, O.PEANO_HILBERT, True, False),
    "f64_morton_orig": (O.F64, O.MORTON, False, True),
    "u64_ph_per_orig": (O.U64, O.PEANO_HILBERT, True, True),
}
N = 256
NQ = 24


def make(name, cfg):
    opts = O.Options(*cfg)
    coord = cfg[0]
    x, y, z = gen("clustered", N, coord, seed=1234)
    # a few exact duplicates so ties are exercised
    x[10:14], y[10:14], z[10:14] = x[3], y[3], z[3]
    t = R.build_bvh(opts, x, y, z)
    out = {"x": x, "y": y, "z": z, "sorted_hi": t.sorted_hi, "sorted_lo": t.sorted_lo}
    for k in ("min_x", "max_x", "min_y", "max_y", "min_z", "max_z", "left_child", "right_child", "parent", "id",
              "is_ghost", "orig_idx"):
        out["tree_" + k] = getattr(t, k)
    out["self16_idx"], out["self16_dist"] = R.self_knn(opts, t, 16, True)
    sub = np.arange(0, N, 11, dtype=np.int32)
    out["subset_ids"] = sub
    out["sub40_idx"], out["sub40_dist"] = R.self_knn(opts, t, 40, False, leaf_ids=sub)
    rng = np.random.default_rng(77)
    q = rng.uniform(0, 100.0, (3, NQ))
    qx, qy, qz = (to_coord(a, coord) for a in q)
    qx[:6], qy[:6], qz[:6] = x[:6], y[:6], z[:6]
    out["qx"], out["qy"], out["qz"] = qx, qy, qz
    out["knn5_idx"], out["knn5_dist"] = R.knn(opts, t, qx, qy, qz, 5, 256)
    out["knn48_idx"], out["knn48_dist"] = R.knn(opts, t, qx, qy, qz, 48, 64)
    dt = qx.dtype
    out["rmin"] = np.array([radius(r, coord) for r in rng.uniform(0, 2, NQ)], dt)
    out["rmax"] = np.array([radius(r, coord) for r in rng.uniform(5, 15, NQ)], dt)
    res, cnt = R.range_query(opts, t, qx, qy, qz, out["rmin"], out["rmax"], 12)
    for i in range(NQ):
        res[i, min(int(cnt[i]), 12):] = -1  # unused slots are not part of the result
    out["range_res"], out["range_cnt"] = res, cnt
    out["config"] = np.array(cfg, np.int32)
    np.savez_compressed(os.path.join(HERE, f"{name}.npz"), **out)


if __name__ == "__main__":
    for name, cfg in CASES.items():
        if not R.available(O.Options(*cfg)):
            raise SystemExit(f"reference checker for {name} is not built: make -C oracle -f ref.mk")
        make(name, cfg)
        print("wrote", name)
