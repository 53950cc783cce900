"""Named sparse inputs shared by the oracle and GPU parity tests.

Edge cases follow the ones the Swift format has by construction: an empty matrix, no regular
tiles, no irregular remainder, one very long column (load-balance split), tiles whose rows
are all equal (format 0), K % 32 in {0, 1, 31}, and ragged dense widths."""
from __future__ import annotations

import numpy as np

from swift_b200 import gen


def _dense_col(M, K, col, extra_density, seed):
    rp, ci = gen.random_csr(M, K, extra_density, seed=seed)
    rows = np.repeat(np.arange(M), np.diff(rp))
    rows = np.concatenate([rows, np.arange(M)])
    cols = np.concatenate([ci, np.full(M, col)])
    return gen.coo_to_csr(M, rows, cols, K=K)


def _same_row_tiles(M, K, seed):
    # 64 columns that all hold rows {0..7}: depth d of every column is row d -> format-0 tiles
    rows, cols = [], []
    for c in range(64):
        rows += list(range(8))
        cols += [c] * 8
    rp, ci = gen.random_csr(M, K, 0.01, seed=seed)
    r2 = np.repeat(np.arange(M), np.diff(rp))
    return gen.coo_to_csr(M, np.concatenate([rows, r2]), np.concatenate([cols, ci]), K=K)


def make(name: str, seed: int = 0):
    """Returns (M, K, rowptr, colidx)."""
    if name == "empty":
        return 16, 40, np.zeros(17, np.int32), np.zeros(0, np.int32)
    if name == "single":
        return 5, 7, np.array([0, 0, 1, 1, 1, 1], np.int32), np.array([3], np.int32)
    if name == "tiny_k":  # fewer than 32 columns: no regular tiles at all
        M, K = 50, 20
        return (M, K) + gen.random_csr(M, K, 0.3, seed=seed)
    if name == "k32_exact":  # K % 32 == 0 with equal counts: no remainder
        M, K = 64, 64
        rows = np.concatenate([np.arange(64)] * 3)
        cols = np.concatenate([(np.arange(64) + s) % 64 for s in (0, 5, 17)])
        return (M, K) + gen.coo_to_csr(M, rows, cols, K=K)
    if name == "k_mod_1":
        M, K = 300, 321
        return (M, K) + gen.random_csr(M, K, 0.05, seed=seed)
    if name == "k_mod_31":
        M, K = 200, 223
        return (M, K) + gen.random_csr(M, K, 0.08, seed=seed, skew=1.2)
    if name == "long_col":  # one column with >> 32 entries: balance splits it
        M, K = 2000, 100
        return (M, K) + _dense_col(M, K, 37, 0.01, seed)
    if name == "same_rows":
        M, K = 100, 128
        return (M, K) + _same_row_tiles(M, K, seed)
    if name == "skewed":
        M, K = 1500, 1000
        return (M, K) + gen.random_csr(M, K, 0.01, seed=seed, skew=0.8)
    if name == "rect_wide":
        M, K = 37, 900
        return (M, K) + gen.random_csr(M, K, 0.05, seed=seed)
    if name == "rect_tall":
        M, K = 3000, 45
        return (M, K) + gen.random_csr(M, K, 0.05, seed=seed, skew=1.0)
    if name == "rmat12":
        M = K = 4096
        return (M, K) + gen.rmat(12, 16 * 4096, seed=seed)
    if name == "poisson4096":
        M = K = 4096
        return (M, K) + gen.poisson_uniform(M, K, 16.0, seed=seed)
    raise KeyError(name)


SMALL = ["empty", "single", "tiny_k", "k32_exact", "k_mod_1", "k_mod_31", "long_col",
         "same_rows", "skewed", "rect_wide", "rect_tall"]
