"""Pins the CPU oracle (this project's C restatement) to the reference's own host code,
compiled in place under oracle/_ref, and to the committed golden fixtures.

Bit-exact: every format array (primary contract: stable column order) and Swift_cpu's C in
FP32 and FP64.  The reference's row_idx_sort leaves the order of equal row keys unspecified
(std::sort), so val_position is compared modulo ties."""
import numpy as np
import pytest

import cases
import oracle
from swift_b200 import gen

needs_ref = pytest.mark.skipif(not oracle.ref_available(), reason="reference checkout not built here")

FORMAT_KEYS = ["tile_ptr", "tile_len", "tile_colidx", "tile_tall", "sortrowidx", "sortval",
               "reside_cscptr", "reside_cscrowidx", "reside_val", "tile_format", "segmentoffset",
               "sortrowindex", "colorblk", "blkstart", "blkstop", "blkptr"]
SCALARS = ["tilenum", "regular_nnz", "reside_col", "reside_nnz", "segsum", "numblk", "nsteps"]


def _inputs(name, dt, N=8, seed=0):
    M, K, rp, ci = cases.make(name, seed)
    val = gen.uniform_values(int(rp[-1]), seed + 1, dt)
    B = gen.dense_uniform(K, N, seed + 2, dt)
    return M, K, rp, ci, val, B


def check_val_position(keys_before, keys_after, pos, tilenum):
    """val_position maps each original slot to a slot holding the same row key."""
    nr = tilenum * 32
    for g0 in range(0, nr, 256):
        g1 = min(g0 + 256, nr)
        kb, ka, p = keys_before[g0:g1], keys_after[g0:g1], pos[g0:g1]
        assert np.array_equal(np.sort(p), np.arange(g1 - g0))
        assert np.array_equal(ka[p], kb)


@needs_ref
@pytest.mark.parametrize("dt", [np.float32, np.float64])
@pytest.mark.parametrize("name", cases.SMALL + ["rmat12"])
def test_oracle_matches_reference(name, dt):
    M, K, rp, ci, val, B = _inputs(name, dt)
    ours = oracle.pipeline(M, K, rp, ci, val, B, impl="oracle")
    ref = oracle.pipeline(M, K, rp, ci, val, B, impl="ref")
    for k in ["cscrowidx", "csccolptr", "nnzpercol", "cscval", "perm", "sortrowidx_tmp",
              "sortval_tmp", "sortnnz_tmp", "sortB"]:
        assert np.array_equal(ours[k], ref[k]), k
    so, sr = ours["slide"], ref["slide"]
    for k in SCALARS:
        assert getattr(so, k) == getattr(sr, k), k
    for k in FORMAT_KEYS:
        assert np.array_equal(so[k], sr[k]), k
    assert np.array_equal(so["rowsorted_rowidx"], sr["rowsorted_rowidx"])
    assert np.array_equal(so["val_offset"], sr["val_offset"])
    check_val_position(so["sortrowidx"], sr["rowsorted_rowidx"], sr["val_position"], so.tilenum)
    check_val_position(so["sortrowidx"], so["rowsorted_rowidx"], so["val_position"], so.tilenum)
    if dt == np.float32 and so.tilenum:
        assert so["blockratio"] == sr["blockratio"]
    # Swift_cpu: identical accumulation order -> identical bits
    assert np.array_equal(ours["C"], ref["C"])


@needs_ref
@pytest.mark.parametrize("name", ["skewed", "k_mod_31", "rmat12", "long_col"])
def test_std_sort_permutation_injected(name):
    """Secondary contract: with the reference's own (unstable) std::sort order injected,
    the arrays equal those of the reference's col_sort run as-is."""
    dt = np.float32
    M, K, rp, ci, val, B = _inputs(name, dt)
    r, p, cnt, v = oracle.csr2csc(M, K, rp, ci, val, impl="ref")
    pm = oracle.perm_std_sort(cnt, dt)
    sr_n, sv_n, sn_n, sB_n = oracle.col_sort(K, B.shape[1], cnt, None, p, r, v, B=B, impl="ref", native=True)
    sr_o, sv_o, sn_o, sB_o = oracle.col_sort(K, B.shape[1], cnt, pm, p, r, v, B=B, impl="oracle")
    assert np.array_equal(sr_n, sr_o) and np.array_equal(sv_n, sv_o)
    assert np.array_equal(sn_n, sn_o) and np.array_equal(sB_n, sB_o)
    # tie-invariant arrays agree between the stable and std::sort orders
    st = oracle.pipeline(M, K, rp, ci, val, B, impl="oracle", perm="stable")["slide"]
    sd = oracle.pipeline(M, K, rp, ci, val, B, impl="oracle", perm=pm)["slide"]
    for k in ["tile_ptr", "tile_len", "tile_colidx", "tile_tall", "reside_cscptr", "colorblk",
              "blkstart", "blkstop", "blkptr"]:
        assert np.array_equal(st[k], sd[k]), k


@pytest.mark.parametrize("name", cases.SMALL)
def test_oracle_spmm_matches_fp64_golden(name):
    """Swift_cpu over the format equals the plain CSR product (FP64, tolerance 1e-12)."""
    M, K, rp, ci, val, B = _inputs(name, np.float64, N=5)
    out = oracle.pipeline(M, K, rp, ci, val, B, impl="oracle")
    gold = oracle.csr_spmm_f64(M, K, rp, ci, val, B)
    denom = max(np.abs(gold).max(), 1e-300)
    assert np.abs(out["C"] - gold).max() / denom <= 1e-12
    s = out["slide"]
    assert s.regular_nnz + s.reside_nnz == int(rp[-1])
