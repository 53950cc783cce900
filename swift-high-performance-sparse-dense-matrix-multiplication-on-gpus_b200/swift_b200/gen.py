"""Seeded synthetic inputs for the Swift SpMM workloads.

The reference measures on SuiteSparse matrices that are not available offline; these
generators stand in with the shapes, sizes and value distributions of each workload:

* ``poisson_uniform`` -- rows of ~Poisson(lam) length with columns drawn uniformly without
  replacement (the 4096 x 4096, lam = 16 parity workload);
* ``rmat``            -- R-MAT (a, b, c, d) edge draws with duplicates merged (the power-law
  scale workloads), generated with torch on any device so full-size matrices are quick;
* ``band``            -- a |i - j| < w diagonal band, merged with R-MAT for the precision
  workload;
* ``random_csr``      -- small irregular shapes for edge cases.

All return ``(rowptr, colidx)`` as int32 numpy arrays (CSR, rows sorted, columns ascending
within a row) unless noted; values are drawn separately so that the pattern and the values
can be reproduced independently.
"""
from __future__ import annotations

import numpy as np


def poisson_uniform(M: int, K: int, lam: float, seed: int = 0):
    rng = np.random.default_rng(seed)
    lens = np.minimum(rng.poisson(lam, size=M), K).astype(np.int64)
    rowptr = np.zeros(M + 1, np.int64)
    np.cumsum(lens, out=rowptr[1:])
    colidx = np.empty(int(rowptr[-1]), np.int32)
    for i in range(M):
        if lens[i]:
            colidx[rowptr[i]:rowptr[i + 1]] = np.sort(rng.choice(K, size=int(lens[i]), replace=False))
    return rowptr.astype(np.int32), colidx


def uniform_values(n: int, seed: int, dtype=np.float32, lo=-1.0, hi=1.0):
    rng = np.random.default_rng(seed)
    return rng.uniform(lo, hi, size=n).astype(dtype)


def dense_uniform(rows: int, cols: int, seed: int, dtype=np.float32):
    rng = np.random.default_rng(seed)
    return rng.uniform(-1.0, 1.0, size=(rows, cols)).astype(dtype)


def coo_to_csr(M: int, rows: np.ndarray, cols: np.ndarray, K: int | None = None):
    """Sort + merge duplicate coordinates; returns (rowptr, colidx) int32."""
    rows = np.asarray(rows, np.int64)
    cols = np.asarray(cols, np.int64)
    Kx = int(K if K is not None else (cols.max() + 1 if cols.size else 1))
    key = np.unique(rows * Kx + cols)
    r = key // Kx
    c = key % Kx
    rowptr = np.zeros(M + 1, np.int64)
    np.add.at(rowptr, r + 1, 1)
    np.cumsum(rowptr, out=rowptr)
    return rowptr.astype(np.int32), c.astype(np.int32)


def rmat(scale: int, nedges: int, a=0.57, b=0.19, c=0.19, seed=0, device="cpu", symmetric=False,
         self_loops=True):
    """R-MAT pattern on 2**scale x 2**scale with duplicates merged (torch; any device).

    Each edge draws one quadrant per level with probabilities (a, b, c, 1-a-b-c); the row bit
    is set for quadrants c and d, the column bit for b and d.  ``symmetric`` merges A and A^T
    (the graph workload); ``self_loops=False`` drops the diagonal."""
    import torch

    g = torch.Generator(device=device)
    g.manual_seed(seed)
    r = torch.zeros(nedges, dtype=torch.int64, device=device)
    cc = torch.zeros(nedges, dtype=torch.int64, device=device)
    for lvl in range(scale):
        u = torch.rand(nedges, generator=g, device=device)
        rb = (u >= a + b).to(torch.int64)
        cb = (((u >= a) & (u < a + b)) | (u >= a + b + c)).to(torch.int64)
        sh = scale - 1 - lvl
        r |= rb << sh
        cc |= cb << sh
    if symmetric:
        r, cc = torch.cat([r, cc]), torch.cat([cc, r])
    if not self_loops:
        keep = r != cc
        r, cc = r[keep], cc[keep]
    key = torch.unique(r << scale | cc)
    r = key >> scale
    cc = key & ((1 << scale) - 1)
    M = 1 << scale
    counts = torch.bincount(r, minlength=M)
    rowptr = torch.zeros(M + 1, dtype=torch.int64, device=device)
    rowptr[1:] = torch.cumsum(counts, 0)
    return rowptr.to(torch.int32).cpu().numpy(), cc.to(torch.int32).cpu().numpy()


def band(M: int, half_width: int):
    """Pattern of |i - j| < half_width on an M x M matrix (COO rows, cols)."""
    i = np.repeat(np.arange(M, dtype=np.int64), 2 * half_width - 1)
    off = np.tile(np.arange(-(half_width - 1), half_width, dtype=np.int64), M)
    j = i + off
    keep = (j >= 0) & (j < M)
    return i[keep], j[keep]


def rmat_plus_band(scale: int, nedges: int, half_width: int, seed=0, device="cpu"):
    rp, ci = rmat(scale, nedges, seed=seed, device=device)
    M = 1 << scale
    rows = np.repeat(np.arange(M, dtype=np.int64), np.diff(rp))
    bi, bj = band(M, half_width)
    return coo_to_csr(M, np.concatenate([rows, bi]), np.concatenate([ci.astype(np.int64), bj]), K=M)


def random_csr(M: int, K: int, density: float, seed: int = 0, skew: float = 0.0):
    """Small random pattern; skew > 0 concentrates nonzeros on low column indices."""
    rng = np.random.default_rng(seed)
    n = int(round(M * K * density))
    rows = rng.integers(0, max(M, 1), size=n)
    if skew > 0:
        cols = np.minimum((rng.pareto(skew, size=n) * K / 8).astype(np.int64), K - 1)
    else:
        cols = rng.integers(0, max(K, 1), size=n)
    if M == 0 or K == 0:
        return np.zeros(M + 1, np.int32), np.zeros(0, np.int32)
    return coo_to_csr(M, rows, cols, K=K)


def rmat_rect(M: int, nedges: int, seed: int = 0, device="cpu"):
    """R-MAT on the next power of two >= M with coordinates outside M x M rejected and
    duplicates merged (torch; any device)."""
    import torch

    scale = max(1, int(np.ceil(np.log2(max(M, 2)))))
    g = torch.Generator(device=device)
    g.manual_seed(seed)
    r = torch.zeros(nedges, dtype=torch.int64, device=device)
    c = torch.zeros(nedges, dtype=torch.int64, device=device)
    for lvl in range(scale):
        u = torch.rand(nedges, generator=g, device=device)
        sh = scale - 1 - lvl
        r |= (u >= 0.76).to(torch.int64) << sh
        c |= (((u >= 0.57) & (u < 0.76)) | (u >= 0.95)).to(torch.int64) << sh
    keep = (r < M) & (c < M)
    key = torch.unique(r[keep] * M + c[keep])
    counts = torch.bincount(key // M, minlength=M)
    rowptr = torch.zeros(M + 1, dtype=torch.int64, device=device)
    rowptr[1:] = torch.cumsum(counts, 0)
    return rowptr.to(torch.int32).cpu().numpy(), (key % M).to(torch.int32).cpu().numpy()


def _uniform_rows(M: int, lam: float, seed: int, device="cpu"):
    """M x M with ~Poisson(lam) row lengths and uniform columns (drawn with replacement and
    merged, which removes under 3% of the draws at lam <= 64, M >= 1024); torch, any device."""
    import torch

    g = torch.Generator(device=device)
    g.manual_seed(seed)
    lens = torch.poisson(torch.full((M,), float(lam), device=device), generator=g).to(torch.int64)
    rows = torch.repeat_interleave(torch.arange(M, device=device), lens.clamp(max=M))
    cols = torch.randint(0, M, (rows.numel(),), generator=g, device=device)
    key = torch.unique(rows * M + cols)
    rowptr = torch.zeros(M + 1, dtype=torch.int64, device=device)
    rowptr[1:] = torch.cumsum(torch.bincount(key // M, minlength=M), 0)
    return rowptr.to(torch.int32).cpu().numpy(), (key % M).to(torch.int32).cpu().numpy()


def batch_matrices(count: int, seed: int = 0, m_lo: int = 1024, m_hi: int = 65536, device="cpu"):
    """The batching workload: square matrices with M log-uniform in [m_lo, m_hi] and average
    degree U[4, 64]; the first half uniform-random (Poisson row lengths, uniform columns),
    the second half R-MAT (a, b, c, d = .57, .19, .19, .05); each with its own dense width N
    from {32, 64, 128}.  Returns a list of dicts (M, rowptr, colidx, N, kind)."""
    rng = np.random.default_rng(seed)
    out = []
    for i in range(count):
        M = int(round(np.exp(rng.uniform(np.log(m_lo), np.log(m_hi)))))
        deg = float(rng.uniform(4.0, 64.0))
        N = int(rng.choice([32, 64, 128]))
        s = int(rng.integers(0, 2**31 - 1))
        if i < count // 2:
            rp, ci = _uniform_rows(M, deg, s, device)
            kind = "uniform"
        else:
            rp, ci = rmat_rect(M, int(round(deg * M)), seed=s, device=device)
            kind = "rmat"
        out.append(dict(M=M, rowptr=rp, colidx=ci, N=N, kind=kind))
    return out


def sym_normalized_values(rowptr: np.ndarray, colidx: np.ndarray, M: int, dtype=np.float32):
    """1 / sqrt(d_i d_j) for a (symmetric) pattern -- the graph-convolution weighting."""
    deg = np.diff(rowptr).astype(np.float64)
    rows = np.repeat(np.arange(M), np.diff(rowptr))
    d = np.maximum(deg, 1.0)
    return (1.0 / np.sqrt(d[rows] * d[colidx])).astype(dtype)
