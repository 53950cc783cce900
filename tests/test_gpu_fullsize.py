"""Parity at the full sizes of the five workloads (every product through the C ABI).

* 1M R-MAT (scale 20, a,b,c,d = .57,.19,.19,.05, 16,777,216 draws, duplicates merged), FP32
  and FP64 values: every format array the GPU builds is bit-exact with the reference's own
  host preprocessing run on the same matrix (csr_to_csc, col_sort with the stable column
  order, formattransation, block_catgory, balance, row_idx_sort; src/coo2csc.h:11-435,
  src/block_catgory.h:1-160, src/balance.h:1-69, src/back_process.h:23-229), and again with
  the reference's own std::sort column order injected; C of every engine matches the
  reference's Swift_cpu over its own format (test/k-32/FP32/Swift_cpu.h:2-65,
  src/Swift_cpu.h:2-78) at N = 32 and 128, normwise max|C - C_ref| / max|C_ref| <= 1e-5 (FP32)
  and <= 1e-12 (FP64), beside the error against the deterministic FP64 GPU product.
* R-MAT scale 19 (16,777,216 draws) merged with the |i - j| < 32 band: BF16 and FP16 B and C
  (FP32 accumulation), plain and per-row scaled, within 1e-2 of the FP64 product; the band
  engine (tiles of half-width 31; 16-bit tiles on the tensor cores) in FP32 within 1e-5 and in
  BF16 / FP16 within 1e-2.
* The 262,144-node symmetric-normalised R-MAT graph at N = 64: Y = A X, dX = A^T dY and
  dA = SDDMM(dY, X), plain and fused, within 1e-5 of FP64 restatements; FP64 central finite
  differences (directional, torch.autograd.gradcheck fast mode) at 1e-6 on the 4,096-node
  instance.
* The 512-matrix batch: every member of one persistent launch (plain and graph replay)
  within 1e-5 of its own FP64 product.

The inputs are the benchmark's own (bench.make_inputs and the same generators and seeds).
"""
import numpy as np
import pytest

import bench
import oracle
from swift_b200 import Plan, gen
from swift_b200.plan import Batch

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

TOL = {np.float32: 1e-5, np.float64: 1e-12}
# arrays compared with their own rule below (the row sort overwrites sortrowidx in place and
# val_position's ties are unspecified in the reference)
SPECIAL = {"sortrowidx", "rowsorted_rowidx", "val_position", "blockratio"}


def relerr(x, ref):
    x = np.asarray(x, np.float64)
    ref = np.asarray(ref, np.float64)
    return float(np.abs(x - ref).max() / max(np.abs(ref).max(), 1e-300)) if ref.size else 0.0


def trelerr(x, ref):
    return (x.double() - ref).abs().max().item() / max(ref.abs().max().item(), 1e-300)


def _quiet(fn, *a, **kw):
    # the reference's host code prints progress lines (and a spurious CSR-to-CSC message)
    with bench._StdoutToStderr():
        return fn(*a, **kw)


@pytest.fixture(scope="module")
def rmat20():
    wl = bench.WORKLOADS["rmat20_n128_f32"]
    M, K, rp, ci, val, _ = bench.make_inputs(wl, "cuda")
    return M, K, rp, ci, val.cpu().numpy()


def _reference_format(M, K, rp, ci, val, perm):
    out = _quiet(oracle.pipeline, M, K, rp, ci, val, None, impl="ref", perm=perm, row_sort=True)
    return out


def _check_format(plan, ref):
    s = ref["slide"]
    ex = plan.export(with_row_sort=True)
    for k in ("tilenum", "regular_nnz", "reside_col", "reside_nnz", "segsum", "numblk"):
        assert ex[k] == getattr(s, k), k
    assert plan.stats()["nsteps"] == s.nsteps
    compared = 0
    for k, v in s.arrays.items():
        if k in SPECIAL:
            continue
        assert k in ex, k
        assert np.array_equal(ex[k], v.astype(ex[k].dtype)), k
        compared += 1
    assert compared >= 15
    assert np.array_equal(ex["sortrowidx"], s.arrays["rowsorted_rowidx"])  # sorted keys, in place
    # val_position: a permutation of each 256-slot group mapping the sorted keys back
    nr = ex["regular_nnz"]
    vp = ex["val_position"]
    for g0 in range(0, nr, 1 << 20):  # whole groups per chunk
        g1 = min(nr, g0 + (1 << 20))
        grp = np.arange(g0, g1) // 256 * 256
        assert np.all(vp[g0:g1] >= 0) and np.all(vp[g0:g1] < np.minimum(256, nr - grp))
        assert np.array_equal(s.arrays["rowsorted_rowidx"][grp + vp[g0:g1]], s.arrays["sortrowidx"][g0:g1])
    perm, sn, _, _ = plan.export_sorted()
    assert np.array_equal(perm, ref["perm"]) and np.array_equal(sn, ref["sortnnz_tmp"])
    ex2 = plan.export(with_row_sort=False)
    assert np.array_equal(ex2["sortrowidx"], s.arrays["sortrowidx"])


@pytest.mark.parametrize("dt", [np.float32, np.float64])
def test_rmat20_format_bit_exact_vs_reference_preprocessing(rmat20, dt):
    M, K, rp, ci, val = rmat20
    v = val.astype(dt)
    ref = _reference_format(M, K, rp, ci, v, "stable")
    plan = Plan.from_csr(rp, ci, v, (M, K))
    _check_format(plan, ref)
    st = plan.stats()
    assert st["reside_nnz"] + 32 * st["tilenum"] == int(rp[-1])
    plan.close()


def test_rmat20_format_with_the_references_std_sort_order(rmat20):
    M, K, rp, ci, val = rmat20
    ref = _reference_format(M, K, rp, ci, val, "std")
    plan = Plan.from_csr(rp, ci, val, (M, K), col_perm=ref["perm"])
    _check_format(plan, ref)
    plan.close()


@pytest.mark.parametrize("N", [32, 128])
@pytest.mark.parametrize("dt", [np.float32, np.float64])
def test_rmat20_spmm_vs_full_swift_cpu(rmat20, dt, N):
    M, K, rp, ci, val = rmat20
    v = val.astype(dt)
    out = _reference_format(M, K, rp, ci, v, "stable")
    tdt = torch.float64 if dt == np.float64 else torch.float32
    g = torch.Generator(device="cuda")
    g.manual_seed(2)
    B = torch.rand((K, N), generator=g, device="cuda", dtype=tdt) * 2 - 1
    Bn = B.cpu().numpy()
    sortB = np.ascontiguousarray(Bn[out["perm"]])  # sort_dense_mtx[i,:] = B[perm[i],:]
    c_cpu = _quiet(oracle.swift_cpu, out["slide"], M, K, N, sortB, impl="ref")
    del sortB
    plan = Plan.from_csr(rp, ci, v, (M, K))
    c64 = plan.spmm_f64_reference(B.double()).cpu().numpy()
    assert relerr(c_cpu, c64) <= TOL[dt]  # the FP64 GPU oracle agrees with Swift_cpu
    for engine in ("rowwise", "tiled", "tiled_grouped", "auto"):
        Cm = plan.spmm(B, engine=engine).cpu().numpy()
        e_ref, e_64 = relerr(Cm, c_cpu), relerr(Cm, c64)
        print(f"N={N} {np.dtype(dt).name} {engine}: vs Swift_cpu {e_ref:.3e}, vs FP64 GPU product {e_64:.3e}")
        assert e_ref <= TOL[dt], (engine, e_ref)
        assert e_64 <= TOL[dt], (engine, e_64)
    plan.close()


def test_precision_band_16bit_full_size():
    wl = bench.WORKLOADS["precision_rmat19band_n128"]
    M, K, rp, ci, val, B32 = bench.make_inputs(dict(wl, kind="rmatband", dtype="f32"), "cuda")
    N = wl["N"]
    assert int(rp[-1]) > 40_000_000  # the band adds about 33M nonzeros to the R-MAT part
    plan = Plan.from_csr(torch.from_numpy(rp).cuda(), torch.from_numpy(ci).cuda(), val, (M, K))
    ref = plan.spmm_f64_reference(B32.double())
    c32 = plan.spmm(B32)
    assert trelerr(c32, ref) <= 1e-5
    m = B32.abs().amax(dim=1)
    bscale = torch.where(m > 0, torch.exp2(torch.floor(torch.log2(torch.where(m > 0, m, torch.ones_like(m)))) - 14),
                         torch.ones_like(m)).float().contiguous()
    for dt in (torch.bfloat16, torch.float16):
        C = plan.spmm(B32.to(dt))
        e64, e32 = trelerr(C, ref), trelerr(C, c32.double())
        print(f"{dt}: vs FP64 {e64:.3e}, vs FP32 path {e32:.3e}")
        assert e64 <= 1e-2 and e32 <= 1e-2
        # against FP64 on the same 16-bit-rounded B: only the accumulation and C's rounding
        assert trelerr(C, plan.spmm_f64_reference(B32.to(dt).double())) <= 1e-2
        Cs, cs = plan.spmm_scaled((B32 / bscale[:, None]).to(dt), b_scale=bscale)
        es = trelerr(Cs.double() * cs.double()[:, None], ref)
        print(f"{dt} scaled: vs FP64 {es:.3e}")
        assert es <= 1e-2
    # the band engine (dense diagonal tiles; 16-bit B on the tensor cores) at full size
    hist, w = plan.band_profile()
    assert w == 31  # the |i - j| < 32 band
    cb = plan.spmm(B32, engine="band")
    assert trelerr(cb, ref) <= 1e-5
    for dt in (torch.bfloat16, torch.float16):
        C = plan.spmm(B32.to(dt), engine="band")
        e64 = trelerr(C, ref)
        print(f"{dt} band engine: vs FP64 {e64:.3e}")
        assert e64 <= 1e-2
        assert trelerr(C, plan.spmm_f64_reference(B32.to(dt).double())) <= 1e-2
    plan.close()


def _graph(scale, dtype):
    rp, ci = gen.rmat(scale, (32 << scale) // 2, seed=0, device="cuda", symmetric=True, self_loops=False)
    M = 1 << scale
    return M, rp, ci, gen.sym_normalized_values(rp, ci, M, dtype)


def test_differentiation_graph_full_size():
    M, rp, ci, vals = _graph(18, np.float32)
    N = 64
    plan = Plan.from_csr(torch.from_numpy(rp).cuda(), torch.from_numpy(ci).cuda(), torch.from_numpy(vals).cuda(),
                         (M, M), build_transpose=True)
    g = torch.Generator(device="cuda")
    g.manual_seed(3)
    X = torch.randn((M, N), generator=g, device="cuda")
    dY = torch.randn((M, N), generator=g, device="cuda")
    Xn, dYn = X.cpu().numpy(), dY.cpu().numpy()
    y64 = oracle.csr_spmm_f64(M, M, rp, ci, vals, Xn)
    dx64 = oracle.csr_spmm_t_f64(M, M, rp, ci, vals, dYn)
    da64 = oracle.sddmm_f64(M, M, rp, ci, dYn, Xn)
    assert relerr(plan.spmm_f64_reference(X.double()).cpu().numpy(), y64) <= 1e-14
    Y, dX, dA = plan.spmm(X), plan.spmm_t(dY), plan.sddmm(dY, X)
    for name, got, want in (("Y", Y, y64), ("dX", dX, dx64), ("dA", dA, da64)):
        assert relerr(got.cpu().numpy(), want) <= 1e-5, name
    assert plan.is_symmetric()
    for sym in (True, False):
        plan.set_symmetry(sym)
        Yf, dXf, dAf = plan.fused_forward_backward(X, dY)
        for name, got, want in (("Y", Yf, y64), ("dX", dXf, dx64), ("dA", dAf, da64)):
            e = relerr(got.cpu().numpy(), want)
            print(f"fused (symmetric pass {sym}) {name}: {e:.3e}")
            assert e <= 1e-5, (sym, name)
    plan.close()
    # the autograd binding on the same layer
    from swift_b200.autograd import SwiftSparseLinear
    layer = SwiftSparseLinear(rp, ci, vals, (M, M))
    Xg = X.clone().requires_grad_()
    Yg = layer(Xg)
    Yg.backward(dY)
    assert relerr(Yg.detach().cpu().numpy(), y64) <= 1e-5
    assert relerr(Xg.grad.cpu().numpy(), dx64) <= 1e-5
    assert relerr(layer.values.grad.cpu().numpy(), da64) <= 1e-5


def test_finite_differences_fp64_on_the_4096_node_instance():
    from swift_b200.autograd import swift_spmm
    M, rp, ci, vals = _graph(12, np.float64)
    N = 64
    plan = Plan.from_csr(rp, ci, vals, (M, M), build_transpose=True)
    v = torch.from_numpy(vals).cuda().requires_grad_()
    g = torch.Generator(device="cuda")
    g.manual_seed(4)
    X = torch.randn((M, N), generator=g, device="cuda", dtype=torch.float64).requires_grad_()
    # directional central differences (u^T J w against the analytic product), several draws
    for seed in range(3):
        torch.manual_seed(seed)
        assert torch.autograd.gradcheck(lambda a, b: swift_spmm(plan, a, b), (v, X), eps=1e-6, atol=1e-6,
                                        rtol=1e-6, fast_mode=True)
    plan.close()


def test_batch512_full_size_every_member():
    mats = gen.batch_matrices(512, seed=0, device="cuda")
    g = torch.Generator(device="cuda")
    g.manual_seed(1)
    plans, Bs, Cs = [], [], []
    for m in mats:
        nnz = int(m["rowptr"][-1])
        val = torch.rand(nnz, generator=g, device="cuda") * 2 - 1
        plans.append(Plan.from_csr(torch.from_numpy(m["rowptr"]).cuda(), torch.from_numpy(m["colidx"]).cuda(),
                                   val, (m["M"], m["M"])))
        Bs.append(torch.rand((m["M"], m["N"]), generator=g, device="cuda") * 2 - 1)
        Cs.append(torch.full((m["M"], m["N"]), float("nan"), device="cuda"))
    assert sum(p.nnz for p in plans) > 200_000_000
    b = Batch(plans)
    b.set_operands(Bs, Cs)
    b.autotune()
    for c in Cs:
        c.fill_(float("nan"))
    b.run()
    torch.cuda.synchronize()
    first = [c.clone() for c in Cs]
    worst = 0.0
    for i, (p, B, C) in enumerate(zip(plans, Bs, Cs)):
        e = trelerr(C, p.spmm_f64_reference(B.double()))
        worst = max(worst, e)
        assert e <= 1e-5, (i, mats[i]["kind"], mats[i]["M"], mats[i]["N"], e)
    print(f"batch of {len(plans)}: worst member error vs FP64 {worst:.3e}")
    for c in Cs:
        c.fill_(float("nan"))
    b.run_graph()
    torch.cuda.synchronize()
    for c0, c in zip(first, Cs):
        assert torch.equal(c0, c)
    b.close()
    for p in plans:
        p.close()
