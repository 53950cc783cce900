"""Merge-path backward kernels: SDDMM, the fused Y + dA pass and, for A == A^T with equal
values, the single pass that also produces dX = A dY.  Each output against the oracle's FP64
products (normwise 1e-4 FP32 -- dot products of up to 128 terms --, 1e-12 FP64); the fused
outputs also against the separate products; symmetry detection on symmetric and
non-symmetric patterns."""
import numpy as np
import pytest

import cases
import oracle
from swift_b200 import Plan, gen

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

TOL = {np.float32: 1e-4, np.float64: 1e-12}


def relerr(x, ref):
    x = np.asarray(x, np.float64)
    ref = np.asarray(ref, np.float64)
    if ref.size == 0:
        return 0.0
    return float(np.abs(x - ref).max() / max(np.abs(ref).max(), 1e-300))


def tdev(a):
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


def symmetric_case(scale=11, seed=0, dt=np.float32):
    rp, ci = gen.rmat(scale, 12 << scale, seed=seed, symmetric=True, self_loops=False)
    M = 1 << scale
    return M, rp, ci, gen.sym_normalized_values(rp, ci, M, dt)


@pytest.mark.parametrize("dt", [np.float32, np.float64])
@pytest.mark.parametrize("N", [1, 3, 4, 8, 20, 32, 64, 100, 128, 200])
def test_sddmm_widths(N, dt):
    M, K, rp, ci = cases.make("rmat12", 2)
    val = gen.uniform_values(int(rp[-1]), 1, dt)
    U = gen.dense_uniform(M, N, 3, dt)
    V = gen.dense_uniform(K, N, 4, dt)
    pl = Plan.from_csr(rp, ci, val, (M, K))
    out = pl.sddmm(tdev(U), tdev(V)).cpu().numpy()
    assert relerr(out, oracle.sddmm_f64(M, K, rp, ci, U, V)) <= TOL[dt]
    pl.close()


@pytest.mark.parametrize("dt", [np.float32, np.float64])
@pytest.mark.parametrize("name", ["skewed", "long_col", "same_rows", "rect_wide", "single"])
@pytest.mark.parametrize("N", [16, 64])
def test_fused_general(name, N, dt):
    M, K, rp, ci = cases.make(name, 0)
    val = gen.uniform_values(int(rp[-1]), 1, dt)
    X = gen.dense_uniform(K, N, 5, dt)
    dY = gen.dense_uniform(M, N, 6, dt)
    pl = Plan.from_csr(rp, ci, val, (M, K))
    Y, dX, dA = pl.fused_forward_backward(tdev(X), tdev(dY))
    assert relerr(Y.cpu().numpy(), oracle.csr_spmm_f64(M, K, rp, ci, val, X)) <= TOL[dt]
    assert relerr(dX.cpu().numpy(), oracle.csr_spmm_t_f64(M, K, rp, ci, val, dY)) <= TOL[dt]
    assert relerr(dA.cpu().numpy(), oracle.sddmm_f64(M, K, rp, ci, dY, X)) <= TOL[dt]
    pl.close()


@pytest.mark.parametrize("dt", [np.float32, np.float64])
@pytest.mark.parametrize("N", [8, 32, 64, 128])
def test_fused_symmetric_single_pass(N, dt):
    M, rp, ci, val = symmetric_case(dt=dt)
    X = gen.dense_uniform(M, N, 7, dt)
    dY = gen.dense_uniform(M, N, 8, dt)
    pl = Plan.from_csr(rp, ci, val, (M, M))
    assert pl.is_symmetric()
    Y, dX, dA = pl.fused_forward_backward(tdev(X), tdev(dY))
    refY = oracle.csr_spmm_f64(M, M, rp, ci, val, X)
    refdX = oracle.csr_spmm_t_f64(M, M, rp, ci, val, dY)
    refdA = oracle.sddmm_f64(M, M, rp, ci, dY, X)
    assert relerr(Y.cpu().numpy(), refY) <= TOL[dt]
    assert relerr(dX.cpu().numpy(), refdX) <= TOL[dt]
    assert relerr(dA.cpu().numpy(), refdA) <= TOL[dt]
    # the general path (transposed layout for dX) gives the same products
    pl.set_symmetry(False)
    Y2, dX2, dA2 = pl.fused_forward_backward(tdev(X), tdev(dY))
    assert relerr(dX2.cpu().numpy(), refdX) <= TOL[dt]
    assert torch.equal(Y, Y2) and torch.equal(dA, dA2)
    # deterministic
    pl.set_symmetry(True)
    Y3, dX3, dA3 = pl.fused_forward_backward(tdev(X), tdev(dY))
    assert torch.equal(Y, Y3) and torch.equal(dX, dX3) and torch.equal(dA, dA3)
    pl.close()


def test_symmetry_detection():
    M, rp, ci, val = symmetric_case(scale=9)
    assert Plan.from_csr(rp, ci, val, (M, M)).is_symmetric()
    v2 = val.copy()
    v2[3] *= 2.0  # same pattern, one value no longer mirrored
    assert not Plan.from_csr(rp, ci, v2, (M, M)).is_symmetric()
    Mr, Kr, rpr, cir = cases.make("skewed", 0)
    assert not Plan.from_csr(rpr, cir, gen.uniform_values(len(cir), 1), (Mr, Kr)).is_symmetric()
    Mg, Kg, rpg, cig = cases.make("rmat12", 0)  # square, not symmetric
    assert not Plan.from_csr(rpg, cig, gen.uniform_values(len(cig), 1), (Mg, Kg)).is_symmetric()
