"""Block-density histogram (swift_plan_block_histogram) through the C ABI, bit-exact against
numpy on small matrices, in A's column order and in the plan's sorted column order."""
import numpy as np
import pytest

from swift_b200 import Plan, gen

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu


def reference(M, K, rp, ci, bh, bw, colpos, nbins):
    rows = np.repeat(np.arange(M, dtype=np.int64), np.diff(rp.astype(np.int64)))
    cols = colpos[ci.astype(np.int64)]
    nbc = (K + bw - 1) // bw
    _, counts = np.unique((rows // bh) * nbc + cols // bw, return_counts=True)
    f = counts / float(bh * bw)
    k = np.minimum(np.floor(-np.log2(f)).astype(np.int64), nbins - 1)
    blocks = np.bincount(k, minlength=nbins)
    nnz = np.bincount(k, weights=counts, minlength=nbins).astype(np.int64)
    return blocks, nnz


def matrices():
    yield "rmat12", 4096, 4096, *gen.rmat(12, 16 << 12, seed=2)
    M = 3000
    bi, bj = gen.band(M, 20)
    yield "band", M, M, *gen.coo_to_csr(M, bi, bj, K=M)
    yield "rect", 1500, 2300, *gen.random_csr(1500, 2300, 0.01, seed=3, skew=1.5)


@pytest.mark.parametrize("shape", [(16, 8), (128, 16), (1, 1), (7, 5)])
def test_block_histogram_matches_numpy(shape):
    bh, bw = shape
    for name, M, K, rp, ci in matrices():
        pl = Plan.from_csr(rp, ci, gen.uniform_values(len(ci), seed=1), (M, K))
        perm = pl.export_sorted()[0]
        invperm = np.empty(K, np.int64)
        invperm[perm.astype(np.int64)] = np.arange(K)
        for sorted_cols, colpos in ((False, np.arange(K)), (True, invperm)):
            blocks, nnz = pl.block_histogram(bh, bw, sorted_columns=sorted_cols, nbins=8)
            rb, rn = reference(M, K, rp, ci, bh, bw, colpos, 8)
            assert np.array_equal(blocks, rb), (name, shape, sorted_cols)
            assert np.array_equal(nnz, rn), (name, shape, sorted_cols)
            assert nnz.sum() == len(ci)
        pl.close()
