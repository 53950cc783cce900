"""The reference's own GPU SpMM wrappers, compiled from its sources for sm_100a
(oracle/_ref/libswiftrefgpu_*.so, see oracle/ref_gpu.cu), run on B200 beside this library.

GPU: on R-MAT scale-13 matrices, each wrapper whose launches stay in bounds for the input
(width a multiple of 32, a reside part, Swift_GPU_4 only FP32 with tilenum % 8 == 0) passes the
reference's own check and agrees with the FP64 CSR product and with this library's product
(normwise 1e-5 FP32, 1e-12 FP64).  CPU: the entry point refuses every other input before it
touches the GPU.
"""
import numpy as np
import pytest

import oracle
from swift_b200 import Plan, gen

TOL = {np.float32: 1e-5, np.float64: 1e-12}
needs_lib = pytest.mark.skipif(not oracle.ref_gpu_available(), reason="oracle/_ref GPU build absent")


def relerr(x, ref):
    x = np.asarray(x, np.float64)
    ref = np.asarray(ref, np.float64)
    return float(np.abs(x - ref).max() / max(np.abs(ref).max(), 1e-300))


def reference_format(M, K, rp, ci, val, N):
    """The reference's own host preprocessing (csr2csc, col_sort, formattransation,
    block_catgory, balance, row_idx_sort) through oracle/_ref."""
    r, p, cnt, v = oracle.csr2csc(M, K, rp, ci, val, impl="ref")
    perm = oracle.perm_stable(cnt)
    sr, sv, sn, _ = oracle.col_sort(K, 1, cnt, perm, p, r, v, impl="ref")
    sl = oracle.build(sr, sv, sn, M, K, impl="ref", row_sort=True, N=N)
    fmt = dict(sl.arrays, tilenum=sl.tilenum, regular_nnz=sl.regular_nnz, reside_col=sl.reside_col,
               reside_nnz=sl.reside_nnz, segsum=sl.segsum, numblk=sl.numblk)
    return fmt, dict(fmt, sortrowidx=sl.arrays["rowsorted_rowidx"]), perm


@needs_lib
@pytest.mark.gpu
@pytest.mark.parametrize("dt", [np.float32, np.float64])
@pytest.mark.parametrize("seed,N", [(5, 32), (5, 64), (1, 128)])
def test_reference_wrappers_agree_with_library(seed, N, dt):
    import torch
    M = K = 1 << 13
    rp, ci = gen.rmat(13, 16 << 13, seed=seed)
    val = gen.uniform_values(len(ci), 1, dt)
    B = gen.dense_uniform(K, N, 2, dt)
    nnz = int(rp[-1])
    fmt, fmt4, perm = reference_format(M, K, rp, ci, val, N)
    ref = oracle.csr_spmm_f64(M, K, rp, ci, val, B)
    plan = Plan.from_csr(rp, ci, val, (M, K))
    ours = plan.spmm(torch.from_numpy(B).cuda(), engine="rowwise").cpu().numpy()
    plan.close()
    assert relerr(ours, ref) <= TOL[dt]
    ran = []
    for var, name in oracle.REF_GPU_VARIANTS.items():
        f = fmt4 if var == 4 else fmt
        if not oracle.ref_gpu_accepts(var, f, N, dt):
            continue
        st, ms, Cr = oracle.ref_gpu_spmm(var, f, M, K, N, nnz, B[perm], ours)
        assert st == oracle.REF_GPU_OK, name
        assert ms > 0
        assert relerr(Cr, ref) <= TOL[dt], name
        assert relerr(Cr, ours) <= 2 * TOL[dt], name
        ran.append(var)
    assert {0, 1, 2, 3} <= set(ran)
    if dt == np.float32 and fmt["tilenum"] % 8 == 0:
        assert 4 in ran


@needs_lib
def test_reference_entry_refuses_out_of_bounds_inputs_on_host():
    """Every refusal returns before the first CUDA call, so this runs without a GPU."""
    M = K = 1 << 12
    rp, ci = gen.rmat(12, 16 << 12, seed=0)
    val = gen.uniform_values(len(ci), 1, np.float32)
    fmt, fmt4, _ = reference_format(M, K, rp, ci, val, 32)
    nnz = int(rp[-1])
    for N in (0, 16, 33):  # widths the launches were not read for
        B = np.zeros((K, max(N, 1)), np.float32)
        st, _, _ = oracle.ref_gpu_spmm(0, fmt, M, K, N, nnz, B, np.zeros((M, max(N, 1)), np.float32))
        assert st == oracle.REF_GPU_REFUSED
    B = np.zeros((K, 32), np.float32)
    gold = np.zeros((M, 32), np.float32)
    no_reside = dict(fmt, reside_nnz=0)
    assert oracle.ref_gpu_spmm(3, no_reside, M, K, 32, nnz, B, gold)[0] == oracle.REF_GPU_REFUSED
    odd = dict(fmt4, tilenum=fmt4["tilenum"] // 8 * 8 - 7)  # tilenum % 8 == 1
    assert oracle.ref_gpu_spmm(4, odd, M, K, 32, nnz, B, gold)[0] == oracle.REF_GPU_REFUSED
    f64 = {k: (v.astype(np.float64) if isinstance(v, np.ndarray) and v.dtype == np.float32 else v)
           for k, v in fmt4.items()}
    f64["tilenum"] = fmt4["tilenum"] // 8 * 8
    assert oracle.ref_gpu_spmm(4, f64, M, K, 32, nnz, B.astype(np.float64),
                               gold.astype(np.float64))[0] == oracle.REF_GPU_REFUSED
    for v in (-1, 5):
        assert oracle.ref_gpu_spmm(v, fmt, M, K, 32, nnz, B, gold)[0] == oracle.REF_GPU_REFUSED
