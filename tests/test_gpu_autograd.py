"""torch.autograd over the Swift products (swift_b200.autograd) and value updates
(swift_plan_set_values).

* swift_plan_set_values: every engine's product after new values equals a plan built from
  scratch with those values (bit-for-bit for the row engine, which reads the same values in
  the same order), and the exported format's value arrays equal a fresh build's.
* Gradients: FP64 central finite differences (torch.autograd.gradcheck) on small graphs; FP32
  gradients on a symmetric-normalised R-MAT graph (the differentiation workload's shape at
  scale 12) against the dense torch reference dX = A^T dY, dvalues = dY[row] . X[col].
"""
import numpy as np
import pytest

from swift_b200 import Plan, gen

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu


def graph(scale, seed=0, dtype=np.float32):
    rp, ci = gen.rmat(scale, 16 << scale, seed=seed, symmetric=True, self_loops=False)
    M = 1 << scale
    return M, rp, ci, gen.sym_normalized_values(rp, ci, M, dtype)


def dense_of(M, K, rp, ci, vals):
    rows = torch.repeat_interleave(torch.arange(M, device="cuda"), torch.from_numpy(np.diff(rp)).long().cuda())
    A = torch.zeros((M, K), dtype=vals.dtype, device="cuda")
    A[rows, torch.from_numpy(ci).long().cuda()] = vals
    return A


@pytest.mark.parametrize("dt", [np.float32, np.float64])
def test_set_values_equals_fresh_build(dt):
    M, rp, ci, v0 = graph(11, dtype=dt)
    v1 = gen.uniform_values(len(ci), seed=7, dtype=dt)
    p = Plan.from_csr(rp, ci, v0, (M, M))
    p.set_values(torch.from_numpy(v1).cuda())
    q = Plan.from_csr(rp, ci, v1, (M, M))
    ea, eb = p.export(), q.export()
    for k in ("sortval", "reside_val", "sortrowidx", "tile_colidx"):
        assert np.array_equal(ea[k], eb[k]), k
    B = torch.rand((M, 64), dtype=torch.float64 if dt == np.float64 else torch.float32, device="cuda")
    for eng in ("rowwise", "tiled", "tiled_grouped"):
        Cp, Cq = p.spmm(B, engine=eng), q.spmm(B, engine=eng)
        if eng == "rowwise":
            assert torch.equal(Cp, Cq)
        else:
            assert (Cp - Cq).abs().max().item() <= 1e-5 * Cq.abs().max().item()
    Y = torch.rand_like(B)
    assert torch.equal(p.spmm_t(Y), q.spmm_t(Y))
    p.set_values(v0)  # host values
    r = Plan.from_csr(rp, ci, v0, (M, M))
    assert torch.equal(p.spmm(B, engine="rowwise"), r.spmm(B, engine="rowwise"))
    # the grouped engine's slots (built above from v1) follow the values back to v0
    Cg, Cr = p.spmm(B, engine="tiled_grouped"), r.spmm(B, engine="tiled_grouped")
    assert (Cg - Cr).abs().max().item() <= 1e-5 * Cr.abs().max().item()


@pytest.mark.parametrize("shape", [(40, 30, 0.15, 3), (64, 64, 0.3, 5)])
def test_gradcheck_fp64(shape):
    from swift_b200.autograd import swift_spmm
    M, K, dens, N = shape
    rp, ci = gen.random_csr(M, K, dens, seed=1, skew=0.5)
    vals = torch.from_numpy(gen.uniform_values(len(ci), seed=2, dtype=np.float64)).cuda().requires_grad_()
    X = torch.rand((K, N), dtype=torch.float64, device="cuda", requires_grad=True)
    plan = Plan.from_csr(rp, ci, vals.detach().cpu().numpy(), (M, K))
    assert torch.autograd.gradcheck(lambda v, x: swift_spmm(plan, v, x), (vals, X), eps=1e-6, atol=1e-6,
                                    rtol=1e-6)


def test_gradients_against_dense_reference():
    from swift_b200.autograd import SwiftSparseLinear
    M, rp, ci, v = graph(12)
    layer = SwiftSparseLinear(rp, ci, v, (M, M))
    X = torch.randn((M, 64), device="cuda", requires_grad=True)
    dY = torch.randn((M, 64), device="cuda")
    Y = layer(X)
    Y.backward(dY)
    vals = layer.values.detach().clone().double().requires_grad_()
    Xr = X.detach().double().requires_grad_()
    A = dense_of(M, M, rp, ci, vals)
    Yr = A @ Xr
    Yr.backward(dY.double())
    rel = lambda a, b: (a.double() - b).abs().max().item() / b.abs().max().item()  # noqa: E731
    assert rel(Y, Yr.detach()) <= 1e-5
    assert rel(X.grad, Xr.grad) <= 1e-5
    assert rel(layer.values.grad, vals.grad) <= 1e-5
    # an optimizer step changes the values in place; the next forward must use them
    with torch.no_grad():
        layer.values.mul_(2.0)
    Y2 = layer(X)
    assert rel(Y2, 2.0 * Yr.detach()) <= 1e-5
