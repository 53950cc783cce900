"""GPU parity: the CUDA library (called through its C ABI) against the reference.

* Format arrays built on the GPU are bit-exact with the reference's preprocessing (committed
  fixtures made by the reference's own code, and the oracle on further cases).
* C matches the reference's Swift_cpu: normwise max|C - C_ref| / max|C_ref| <= 1e-5 (FP32),
  <= 1e-12 (FP64); the error against the deterministic FP64 GPU product is checked beside it.
"""
import numpy as np
import pytest

import cases
import golden_io
import oracle
from swift_b200 import Plan, gen

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

TOL = {np.float32: 1e-5, np.float64: 1e-12}


def relerr(x, ref):
    x = np.asarray(x, np.float64)
    ref = np.asarray(ref, np.float64)
    d = max(np.abs(ref).max(), 1e-300) if ref.size else 1.0
    return float(np.abs(x - ref).max() / d) if ref.size else 0.0


def plan_of(g, dt):
    return Plan.from_csr(g["rowptr"], g["colidx"], g["val"].astype(dt), (g["M"], g["K"]))


def tdev(a):
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


@pytest.mark.parametrize("dt", [np.float32, np.float64])
@pytest.mark.parametrize("name", golden_io.ALL)
def test_format_bit_exact_vs_reference_fixture(name, dt):
    g = golden_io.load(name, dt)
    pl = plan_of(g, dt)
    ex = pl.export(with_row_sort=True)
    for k in golden_io.SCALARS:
        if k == "nsteps":
            assert pl.stats()["nsteps"] == g[k]
        else:
            assert ex[k] == g[k], k
    for k in golden_io.ARRAYS:
        if k in ("val_position", "rowsorted_rowidx", "sortrowidx"):
            continue
        assert np.array_equal(ex[k], g[k].astype(ex[k].dtype)), k
    # export with the row sort overwrites sortrowidx with sorted keys, as the reference does
    assert np.array_equal(ex["sortrowidx"], g["rowsorted_rowidx"])
    nr = ex["regular_nnz"]
    for g0 in range(0, nr, 256):
        g1 = min(g0 + 256, nr)
        p = ex["val_position"][g0:g1]
        assert np.array_equal(np.sort(p), np.arange(g1 - g0))
        assert np.array_equal(g["rowsorted_rowidx"][g0:g1][p], g["sortrowidx"][g0:g1])
    perm, sn, sr, sv = pl.export_sorted()
    assert np.array_equal(perm, g["perm"]) and np.array_equal(sn, g["sortnnz"])
    ex2 = pl.export(with_row_sort=False)
    assert np.array_equal(ex2["sortrowidx"], g["sortrowidx"])
    pl.close()


@pytest.mark.parametrize("engine", ["tiled", "tiled_grouped", "rowwise"])
@pytest.mark.parametrize("dt", [np.float32, np.float64])
@pytest.mark.parametrize("name", golden_io.ALL)
def test_spmm_matches_swift_cpu(name, dt, engine):
    g = golden_io.load(name, dt)
    pl = plan_of(g, dt)
    B = tdev(g["B"])
    Cm = pl.spmm(B, engine=engine).cpu().numpy()
    assert Cm.dtype == dt
    assert relerr(Cm, g["C"]) <= TOL[dt], relerr(Cm, g["C"])
    c64 = pl.spmm_f64_reference(B.double()).cpu().numpy()
    assert relerr(c64, oracle.csr_spmm_f64(g["M"], g["K"], g["rowptr"], g["colidx"], g["val"], g["B"])) <= 1e-14
    assert relerr(Cm, c64) <= TOL[dt]
    pl.close()


@pytest.mark.parametrize("dt", [np.float32, np.float64])
@pytest.mark.parametrize("name", ["poisson4096", "long_col", "same_rows", "k_mod_31"])
def test_tiled_colmajor_presorted_like_reference_wrappers(name, dt):
    """The reference wrappers take the column-sorted B in column-major order and return C
    column-major (src/main.cu:338-340, src/Swift.h:390-396)."""
    g = golden_io.load(name, dt)
    pl = plan_of(g, dt)
    sortB = g["B"][g["perm"]]
    Bcm = torch.from_numpy(np.asfortranarray(sortB)).cuda().t().contiguous().t()  # column-major view
    assert Bcm.stride(0) == 1
    Cm = pl.spmm(Bcm, engine="tiled", b_presorted=True, layout="col").cpu().numpy()
    assert relerr(Cm, g["C"]) <= TOL[dt]
    # unsorted B, column-major, perm applied on the fly
    Bcm2 = torch.from_numpy(np.asfortranarray(g["B"])).cuda().t().contiguous().t()
    Cm2 = pl.spmm(Bcm2, engine="tiled", layout="col").cpu().numpy()
    assert relerr(Cm2, g["C"]) <= TOL[dt]
    pl.close()


@pytest.mark.parametrize("dt", ["f32", "f64", "bf16"])
@pytest.mark.parametrize("engine", ["auto", "rowwise"])
@pytest.mark.parametrize("N", [32, 33, 128])
@pytest.mark.parametrize("pad", [0, 5])
def test_column_major_operands_through_the_row_walk(dt, engine, N, pad):
    """Column-major B and C (leading dimensions exact or padded) run the row walk on row-major
    copies: the same bits as the row-major product, padding untouched."""
    M, K, rp, ci = cases.make("rmat12", 0)
    npdt = np.float64 if dt == "f64" else np.float32
    tdt = {"f32": torch.float32, "f64": torch.float64, "bf16": torch.bfloat16}[dt]
    val = gen.uniform_values(int(rp[-1]), 1, npdt)
    B = tdev(gen.dense_uniform(K, N, 2, npdt)).to(tdt)
    pl = Plan.from_csr(rp, ci, val, (M, K))
    Crow = pl.spmm(B, engine="rowwise")
    Bbig = torch.zeros((N, K + pad), dtype=tdt, device="cuda")
    Bbig[:, :K] = B.t()
    Cbig = torch.full((N, M + (3 if pad else 0)), 7.0, dtype=tdt, device="cuda")
    Ccm = Cbig[:, :M].t()
    pl.spmm(Bbig[:, :K].t(), C_out=Ccm, engine=engine, layout="col")
    assert torch.equal(Ccm, Crow)
    assert bool((Cbig[:, M:] == 7.0).all())
    ref = oracle.csr_spmm_f64(M, K, rp, ci, val, B.double().cpu().numpy())
    assert relerr(Ccm.double().cpu().numpy(), ref) <= (1e-2 if dt == "bf16" else TOL[npdt])
    pl.close()


@pytest.mark.parametrize("name", cases.SMALL)
@pytest.mark.parametrize("N", [4, 33])
def test_column_major_small_and_edge_shapes(name, N):
    """Column-major operands through the row walk on every small / edge shape (empty matrix,
    K < 32, rectangular, long columns): equal to the row-major product."""
    M, K, rp, ci = cases.make(name, 0)
    val = gen.uniform_values(int(rp[-1]), 1, np.float32)
    B = tdev(gen.dense_uniform(K, N, 2, np.float32))
    pl = Plan.from_csr(rp, ci, val, (M, K))
    Crow = pl.spmm(B, engine="rowwise")
    Ccm = pl.spmm(B.t().contiguous().t(), engine="auto", layout="col")
    assert Ccm.stride(0) == 1 and torch.equal(Ccm, Crow)
    assert relerr(Ccm.cpu().numpy(), oracle.csr_spmm_f64(M, K, rp, ci, val, B.cpu().numpy())) <= 1e-5
    pl.close()


@pytest.mark.parametrize("N", [1, 8, 24, 32, 33, 64, 128, 768])
@pytest.mark.parametrize("engine", ["tiled", "tiled_grouped", "rowwise"])
def test_ragged_widths(N, engine):
    M, K, rp, ci = cases.make("rmat12", 0)
    val = gen.uniform_values(int(rp[-1]), 1, np.float32)
    Bn = gen.dense_uniform(K, N, 2, np.float32)
    ref = oracle.csr_spmm_f64(M, K, rp, ci, val, Bn)
    pl = Plan.from_csr(rp, ci, val, (M, K), long_row_split=64)
    Cm = pl.spmm(tdev(Bn), engine=engine).cpu().numpy()
    assert relerr(Cm, ref) <= 1e-5
    # strided operands (leading dimension > N)
    Bp = torch.zeros((K, N + 3), dtype=torch.float32, device="cuda")
    Bp[:, :N] = tdev(Bn)
    Cp = torch.full((M, N + 5), 7.0, dtype=torch.float32, device="cuda")
    pl.spmm(Bp[:, :N], Cp[:, :N], engine=engine)
    assert relerr(Cp[:, :N].cpu().numpy(), ref) <= 1e-5
    assert torch.all(Cp[:, N:] == 7.0)
    pl.close()


@pytest.mark.parametrize("split", [16, 32, 128, 100000])
def test_long_row_split_is_deterministic(split):
    M, K, rp, ci = cases.make("rmat12", 3)
    val = gen.uniform_values(int(rp[-1]), 1, np.float32)
    Bn = gen.dense_uniform(K, 128, 2, np.float32)
    pl = Plan.from_csr(rp, ci, val, (M, K), long_row_split=split)
    st = pl.stats()
    if split < st["max_row_nnz"]:
        assert st["long_rows"] > 0
    B = tdev(Bn)
    c1 = pl.spmm(B, engine="rowwise")
    c2 = pl.spmm(B, engine="rowwise")
    assert torch.equal(c1, c2)
    assert relerr(c1.cpu().numpy(), oracle.csr_spmm_f64(M, K, rp, ci, val, Bn)) <= 1e-5
    pl.close()


@pytest.mark.parametrize("U", [7, 32, 128, 256, 1024])
@pytest.mark.parametrize("unr,vb,kern", [(4, 0, 1), (8, 0, 1), (4, 16, 2), (4, 32, 2), (16, 16, 3),
                                         (8, 32, 3), (4, 4, 0), (8, 16, 4), (16, 16, 4)])
@pytest.mark.parametrize("N", [4, 8, 32, 33, 64, 128, 300, 512])
def test_row_engine_parameters(U, unr, vb, kern, N):
    """Every task size, load depth, vector width and kernel variant gives the same
    (deterministic) product; rows split across tasks are combined in task order."""
    M, K, rp, ci = cases.make("rmat12", 1)
    val = gen.uniform_values(int(rp[-1]), 1, np.float32)
    Bn = gen.dense_uniform(K, N, 2, np.float32)
    ref = oracle.csr_spmm_f64(M, K, rp, ci, val, Bn)
    pl = Plan.from_csr(rp, ci, val, (M, K))
    pl.set_rowwise_params(U, unr, vb, kern)
    B = tdev(Bn)
    c1 = pl.spmm(B, engine="rowwise")
    c2 = pl.spmm(B, engine="rowwise")
    assert torch.equal(c1, c2)
    assert relerr(c1.cpu().numpy(), ref) <= 1e-5
    pl.close()


@pytest.mark.parametrize("dt16", ["bf16", "f16"])
def test_low_precision_operands(dt16):
    M, K, rp, ci = cases.make("rmat12", 0)
    val = gen.uniform_values(int(rp[-1]), 1, np.float32)
    Bn = gen.dense_uniform(K, 128, 2, np.float32)
    tdt = torch.bfloat16 if dt16 == "bf16" else torch.float16
    B16 = tdev(Bn).to(tdt)
    pl = Plan.from_csr(rp, ci, val, (M, K))
    C16 = pl.spmm(B16)
    assert C16.dtype == tdt
    ref = oracle.csr_spmm_f64(M, K, rp, ci, val, B16.float().cpu().numpy().astype(np.float64))
    assert relerr(C16.double().cpu().numpy(), ref) <= 1e-2
    pl.close()


def _pow2_row_scale(x):
    """Per-row powers of two putting each row's largest magnitude in [2^14, 2^15) (1 for zero rows)."""
    m = np.abs(x).max(axis=1)
    e = np.floor(np.log2(np.where(m > 0, m, 1.0)))
    return np.where(m > 0, np.exp2(e - 14), 1.0).astype(np.float32)


@pytest.mark.parametrize("dt16", ["bf16", "f16"])
@pytest.mark.parametrize("N", [8, 64, 96, 128, 200, 256, 512])
@pytest.mark.parametrize("U", [32, 512])
@pytest.mark.parametrize("vb", [0, 16])
def test_per_row_scaled_16bit_operands(dt16, N, U, vb):
    """B rows spanning 2^-40 .. 2^40 (far outside FP16's range) stored as 16-bit rows with
    per-row scales: every row of c_scale * C is within 1e-2 of the row's largest magnitude of
    the FP64 product on the dequantised B, each c_scale is a power of two putting the row's
    16-bit maximum in [2^14, 2^15], zero rows get scale 1, and rows split across tasks (U = 32)
    combine deterministically.  vb = 0 lets rows of 16-element multiples take 32-byte vectors;
    16 keeps 16-byte ones (up to N = 256)."""
    M, K, rp, ci = cases.make("rmat12", 0)
    val = gen.uniform_values(int(rp[-1]), 1, np.float32)
    rng = np.random.default_rng(7)
    Btrue = gen.dense_uniform(K, N, 2, np.float64) * np.exp2(rng.integers(-40, 41, K))[:, None]
    bs = _pow2_row_scale(Btrue)
    tdt = torch.bfloat16 if dt16 == "bf16" else torch.float16
    B16 = tdev((Btrue / bs[:, None]).astype(np.float32)).to(tdt)
    pl = Plan.from_csr(rp, ci, val, (M, K))
    pl.set_rowwise_params(U, 4, vb, 2)
    if vb == 16 and N > 256:
        from swift_b200 import _capi as capi
        with pytest.raises(capi.SwiftError):
            pl.spmm_scaled(B16, b_scale=tdev(bs))
        pl.close()
        return
    C16, cs = pl.spmm_scaled(B16, b_scale=tdev(bs))
    C16b, csb = pl.spmm_scaled(B16, b_scale=tdev(bs))
    assert torch.equal(C16, C16b) and torch.equal(cs, csb)
    Bdeq = B16.double().cpu().numpy() * bs[:, None].astype(np.float64)
    ref = oracle.csr_spmm_f64(M, K, rp, ci, val, Bdeq)
    C = C16.double().cpu().numpy()
    s = cs.cpu().numpy().astype(np.float64)
    assert np.all(np.isfinite(C))
    rmax = np.abs(ref).max(axis=1)
    err = np.abs(s[:, None] * C - ref).max(axis=1)
    assert np.all(err <= 1e-2 * rmax)
    nz = rmax > 0
    assert np.array_equal(np.exp2(np.round(np.log2(s))), s)  # powers of two
    cmax = np.abs(C).max(axis=1)
    assert np.all((cmax[nz] >= 2.0 ** 14) & (cmax[nz] <= 2.0 ** 15))
    assert np.all(s[~nz] == 1.0) and np.all(C[~nz] == 0)
    pl.close()


def test_per_row_scaled_without_b_scale_and_refusals():
    """b_scale omitted means all 1; F32 operands, widths above 256 and a missing c_scale are refused."""
    M, K, rp, ci = cases.make("rmat12", 0)
    val = gen.uniform_values(int(rp[-1]), 1, np.float32)
    Bn = gen.dense_uniform(K, 64, 2, np.float32)
    pl = Plan.from_csr(rp, ci, val, (M, K))
    B16 = tdev(Bn).to(torch.bfloat16)
    C16, cs = pl.spmm_scaled(B16)
    ref = oracle.csr_spmm_f64(M, K, rp, ci, val, B16.double().cpu().numpy())
    got = cs.cpu().numpy()[:, None].astype(np.float64) * C16.double().cpu().numpy()
    assert relerr(got, ref) <= 1e-2
    from swift_b200 import _capi as capi
    with pytest.raises(capi.SwiftError):
        pl.spmm_scaled(tdev(Bn))
    with pytest.raises(capi.SwiftError):
        pl.spmm_scaled(tdev(gen.dense_uniform(K, 264, 2, np.float32)).to(torch.bfloat16))
    st = capi.lib().swift_spmm_scaled(pl._h, 64, capi.BF16, B16.data_ptr(), 64, None, C16.data_ptr(), 64,
                                      None, None)
    assert st == capi.ERR_INVALID_ARG
    pl.close()


@pytest.mark.parametrize("dt", [np.float32, np.float64])
@pytest.mark.parametrize("name", ["rmat12", "skewed", "rect_wide", "rect_tall", "empty", "long_col"])
def test_backward_products(name, dt):
    M, K, rp, ci = cases.make(name, 0)
    val = gen.uniform_values(int(rp[-1]), 1, dt)
    N = 64
    X = gen.dense_uniform(K, N, 5, dt)
    dY = gen.dense_uniform(M, N, 6, dt)
    pl = Plan.from_csr(rp, ci, val, (M, K), long_row_split=32)
    tol = TOL[dt] * (10 if dt == np.float32 else 1)
    dX = pl.spmm_t(tdev(dY)).cpu().numpy()
    assert relerr(dX, oracle.csr_spmm_t_f64(M, K, rp, ci, val, dY)) <= tol
    dA = pl.sddmm(tdev(dY), tdev(X)).cpu().numpy()
    assert relerr(dA, oracle.sddmm_f64(M, K, rp, ci, dY, X)) <= tol
    Y, dX2, dA2 = pl.fused_forward_backward(tdev(X), tdev(dY))
    assert relerr(Y.cpu().numpy(), oracle.csr_spmm_f64(M, K, rp, ci, val, X)) <= tol
    assert relerr(dX2.cpu().numpy(), oracle.csr_spmm_t_f64(M, K, rp, ci, val, dY)) <= tol
    assert relerr(dA2.cpu().numpy(), oracle.sddmm_f64(M, K, rp, ci, dY, X)) <= tol
    pl.close()


def test_device_resident_csr_and_injected_perm():
    g = golden_io.load("skewed")
    r, p, cnt, v = oracle.csr2csc(g["M"], g["K"], g["rowptr"], g["colidx"], g["val"])
    pm = oracle.perm_stable(cnt)[::-1].copy()  # not sorted -> must be rejected
    with pytest.raises(Exception):
        Plan.from_csr(g["rowptr"], g["colidx"], g["val"], (g["M"], g["K"]), col_perm=pm)
    # a valid alternative order: ties reversed
    keys = cnt.astype(np.int64) * g["K"] + (g["K"] - 1 - np.arange(g["K"]))
    pm2 = np.argsort(keys, kind="stable").astype(np.int32)
    pl = Plan.from_csr(tdev(g["rowptr"]), tdev(g["colidx"]), tdev(g["val"]), (g["M"], g["K"]), col_perm=pm2)
    perm, *_ = pl.export_sorted()
    assert np.array_equal(perm, pm2)
    ref = oracle.pipeline(g["M"], g["K"], g["rowptr"], g["colidx"], g["val"], g["B"], perm=pm2)
    ex = pl.export()
    for k in ("sortrowidx", "sortval", "reside_cscrowidx", "reside_val", "tile_colidx", "colorblk"):
        assert np.array_equal(ex[k], ref["slide"][k]), k
    assert relerr(pl.spmm(tdev(g["B"]), engine="tiled").cpu().numpy(), ref["C"]) <= 1e-5
    pl.close()


def test_bad_csr_rejected():
    from swift_b200 import capi
    rp = np.array([0, 2, 1, 3], np.int32)
    ci = np.array([0, 1, 2], np.int32)
    with pytest.raises(capi.SwiftError) as e:
        Plan.from_csr(rp, ci, np.ones(3, np.float32), (3, 3))
    assert e.value.status == capi.ERR_BAD_CSR
    rp = np.array([0, 1, 2, 3], np.int32)
    ci = np.array([0, 1, 9], np.int32)
    with pytest.raises(capi.SwiftError):
        Plan.from_csr(tdev(rp), tdev(ci), tdev(np.ones(3, np.float32)), (3, 3))


def test_python_layer_refuses_bad_operands_before_launch():
    """Wrong shapes, dtypes and host tensors are refused on the host by every product method."""
    M, K, rp, ci = cases.make("rmat12", 0)
    val = gen.uniform_values(int(rp[-1]), 1, np.float32)
    pl = Plan.from_csr(rp, ci, val, (M, K))
    B = tdev(gen.dense_uniform(K, 32, 2, np.float32))
    with pytest.raises(ValueError, match="shape"):
        pl.spmm(B[:-1])
    with pytest.raises(ValueError, match="CUDA tensor"):
        pl.spmm(B.cpu())
    with pytest.raises(ValueError, match="dtype"):
        pl.spmm(B, C_out=torch.empty((M, 32), dtype=torch.float64, device="cuda"))
    with pytest.raises(ValueError, match="shape"):
        pl.spmm_t(B[:, :16].contiguous()[: M - 1])
    with pytest.raises(ValueError, match="shape"):
        pl.sddmm(B, B[:-1])
    with pytest.raises(ValueError, match="elements"):
        pl.spmm_scaled(B.to(torch.bfloat16), b_scale=torch.ones(K - 1, device="cuda"))
    with pytest.raises(ValueError, match="shape"):
        pl.autotune(B, torch.empty((M, 16), device="cuda"))
    C = pl.spmm(B)  # still usable
    assert relerr(C.cpu().numpy(), oracle.csr_spmm_f64(M, K, rp, ci, val, B.cpu().numpy())) <= 1e-5
    pl.close()
