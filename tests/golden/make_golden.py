"""Generates the golden fixtures in this directory by running the REFERENCE's own host code
(compiled in place under oracle/_ref from the reference checkout by oracle/Makefile).

    python tests/golden/make_golden.py        # needs oracle/_ref built (reference present)

Fixtures (numpy .npz, compressed):
  poisson4096_n32_f32.npz -- the 4096 x 4096 parity workload: rows ~Poisson(16), columns uniform
                             without replacement, values U[-1,1], B 4096 x 32 U[-1,1], seed 0;
                             FP32 (the reference's test/k-32/FP32 flavour)
  small_f32.npz           -- every edge case in tests/cases.py (N = 8)
  poisson4096_n32_f64.npz, small_f64.npz
                          -- C from the reference's FP64 flavour (src/) on the same inputs
                             widened to double (every format array is then identical to the
                             FP32 one, so only C is stored)

Each FP32 file holds the inputs (rowptr, colidx, val, B), the column permutation (stable
order), every format array the reference produces (formattransation, block_catgory, balance,
row_idx_sort) and C from the reference's Swift_cpu.
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path[:0] = [os.path.join(ROOT, "oracle"), os.path.join(ROOT, "tests"),
                os.path.join(ROOT, "swift-high-performance-sparse-dense-matrix-multiplication-on-gpus_b200")]

import cases  # noqa: E402
import oracle  # noqa: E402
from swift_b200 import gen  # noqa: E402

SCALARS = ["tilenum", "regular_nnz", "reside_col", "reside_nnz", "segsum", "numblk", "nsteps"]


def record(prefix, M, K, rp, ci, val, B):
    out = oracle.pipeline(M, K, rp, ci, val, B, impl="ref")
    s = out["slide"]
    d = {f"{prefix}M": np.int64(M), f"{prefix}K": np.int64(K), f"{prefix}rowptr": rp,
         f"{prefix}colidx": ci, f"{prefix}val": val, f"{prefix}B": B, f"{prefix}perm": out["perm"],
         f"{prefix}nnzpercol": out["nnzpercol"], f"{prefix}csccolptr": out["csccolptr"],
         f"{prefix}cscrowidx": out["cscrowidx"], f"{prefix}sortnnz": out["sortnnz_tmp"],
         f"{prefix}C": out["C"]}
    for k in SCALARS:
        d[prefix + k] = np.int64(getattr(s, k))
    for k, v in s.arrays.items():
        d[prefix + k] = v
    return d


def main():
    if not oracle.ref_available():
        raise SystemExit("oracle/_ref is not built: run make -C oracle with the reference present")
    M = K = 4096
    rp, ci = gen.poisson_uniform(M, K, 16.0, seed=0)
    val = gen.uniform_values(int(rp[-1]), 1, np.float32)
    B = gen.dense_uniform(K, 32, 2, np.float32)
    np.savez_compressed(os.path.join(HERE, "poisson4096_n32_f32.npz"), **record("", M, K, rp, ci, val, B))
    c64 = oracle.pipeline(M, K, rp, ci, val.astype(np.float64), B.astype(np.float64), impl="ref")["C"]
    np.savez_compressed(os.path.join(HERE, "poisson4096_n32_f64.npz"), C=c64)
    d, d64 = {}, {}
    for name in cases.SMALL:
        m, k, r2, c2 = cases.make(name, 0)
        v2 = gen.uniform_values(int(r2[-1]), 1, np.float32)
        b2 = gen.dense_uniform(k, 8, 2, np.float32)
        d.update(record(name + "/", m, k, r2, c2, v2, b2))
        d64[name + "/C"] = oracle.pipeline(m, k, r2, c2, v2.astype(np.float64), b2.astype(np.float64), impl="ref")["C"]
    np.savez_compressed(os.path.join(HERE, "small_f32.npz"), **d)
    np.savez_compressed(os.path.join(HERE, "small_f64.npz"), **d64)
    print("fixtures written to", HERE)


if __name__ == "__main__":
    main()
