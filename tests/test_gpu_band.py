"""GPU parity of the band engine (dense diagonal tiles + the row walk for the rest).

C from the BAND engine, called through the C ABI, against the reference's Swift_cpu
(restated in the oracle; FP32 normwise <= 1e-5) and against the deterministic FP64 GPU product
(16-bit B and C: <= 1e-2), on banded, mixed and band-free patterns, square and rectangular,
with partial column slices, strided operands, value updates and the shapes the engine refuses.
The |col - row| profile is checked bit-exact against numpy.
"""
import numpy as np
import pytest

import oracle
from swift_b200 import Plan, gen
from swift_b200._capi import SwiftError, ERR_UNSUPPORTED as UNSUPPORTED

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu


def relerr(x, ref):
    x = np.asarray(x, np.float64)
    ref = np.asarray(ref, np.float64)
    return float(np.abs(x - ref).max() / max(np.abs(ref).max(), 1e-300)) if ref.size else 0.0


def band_pattern(M, K, half, extra_density=0.0, seed=0):
    """|i - j| < half (clipped to K) merged with uniform extras."""
    i = np.repeat(np.arange(M, dtype=np.int64), 2 * half - 1)
    j = i + np.tile(np.arange(-(half - 1), half, dtype=np.int64), M)
    keep = (j >= 0) & (j < K)
    rows, cols = [i[keep]], [j[keep]]
    if extra_density > 0:
        rng = np.random.default_rng(seed)
        n = int(M * K * extra_density)
        rows.append(rng.integers(0, M, n))
        cols.append(rng.integers(0, K, n))
    return gen.coo_to_csr(M, np.concatenate(rows), np.concatenate(cols), K=K)


CASES = {
    # name: (M, K, pattern builder)
    "band32_plus_rmat": (4096, 4096, lambda: _rmat_band(12, 32)),
    "band4_ragged_rows": (1000, 1000, lambda: band_pattern(1000, 1000, 4, 0.002, 1)),
    "band16_wide_K": (1000, 1500, lambda: band_pattern(1000, 1500, 16, 0.003, 2)),
    "band16_narrow_K": (1500, 1000, lambda: band_pattern(1500, 1000, 16, 0.003, 3)),
    "no_band": (2048, 2048, lambda: gen.random_csr(2048, 2048, 0.004, seed=4)),
}


def _rmat_band(scale, half):
    rp, ci = gen.rmat(scale, 8 << scale, seed=0)
    M = 1 << scale
    rows = np.repeat(np.arange(M, dtype=np.int64), np.diff(rp))
    bi, bj = gen.band(M, half)
    return gen.coo_to_csr(M, np.concatenate([rows, bi]), np.concatenate([ci.astype(np.int64), bj]), K=M)


def build(name):
    M, K, f = CASES[name]
    rp, ci = f()
    val = gen.uniform_values(len(ci), seed=7)
    return M, K, rp, ci, val


@pytest.mark.parametrize("name", sorted(CASES))
def test_profile_bit_exact(name):
    M, K, rp, ci, val = build(name)
    pl = Plan.from_csr(rp, ci, val, (M, K))
    hist, w = pl.band_profile()
    rows = np.repeat(np.arange(M), np.diff(rp))
    d = np.abs(ci.astype(np.int64) - rows)
    ref = np.bincount(d[d <= 128], minlength=129)
    assert np.array_equal(hist, ref)
    # the half-width rule: the largest (within-W count - M * TW / 8) that saves a twentieth
    best, bw = 0.05 * len(ci), -1
    for cand in (3, 7, 15, 31, 47, 63):
        tw = (8 + 2 * cand + 3) // 4 * 4
        gain = ref[: cand + 1].sum() - M * tw / 8.0
        if gain > best:
            best, bw = gain, cand
    assert w == bw
    if name == "band32_plus_rmat":
        assert w == 31
    if name == "no_band":
        assert w == -1
    pl.close()


@pytest.mark.parametrize("N", [128, 132, 200, 256])
@pytest.mark.parametrize("name", sorted(CASES))
def test_band_fp32_vs_swift_cpu(name, N):
    M, K, rp, ci, val = build(name)
    B = gen.dense_uniform(K, N, seed=11)
    c_ref = oracle.pipeline(M, K, rp, ci, val, B)["C"]
    pl = Plan.from_csr(rp, ci, val, (M, K))
    Bt = torch.from_numpy(B).cuda()
    C = pl.spmm(Bt, engine="band")
    torch.cuda.synchronize()
    assert relerr(C.cpu().numpy(), c_ref) <= 1e-5
    c64 = pl.spmm_f64_reference(Bt.double()).cpu().numpy()
    assert relerr(C.cpu().numpy(), c64) <= 1e-5
    # a second product on the same plan (split and tasks reused) gives the same C
    C2 = pl.spmm(Bt, engine="band")
    assert torch.equal(C, C2)
    pl.close()


@pytest.mark.parametrize("dt", ["bfloat16", "float16"])
@pytest.mark.parametrize("name", ["band32_plus_rmat", "band4_ragged_rows", "band16_narrow_K"])
def test_band_16bit_vs_fp64(name, dt):
    M, K, rp, ci, val = build(name)
    tdt = getattr(torch, dt)
    B = torch.from_numpy(gen.dense_uniform(K, 128, seed=12)).cuda().to(tdt)
    pl = Plan.from_csr(rp, ci, val, (M, K))
    ref = pl.spmm_f64_reference(B.double()).cpu().numpy()
    C = pl.spmm(B, engine="band")
    Cr = pl.spmm(B, engine="rowwise")
    torch.cuda.synchronize()
    assert relerr(C.double().cpu().numpy(), ref) <= 1e-2
    assert relerr(C.double().cpu().numpy(), Cr.double().cpu().numpy()) <= 1e-2
    pl.close()


def test_band_strided_operands():
    M, K, rp, ci, val = build("band32_plus_rmat")
    N = 128
    Bw = torch.from_numpy(gen.dense_uniform(K, N + 8, seed=13)).cuda()
    B = Bw[:, 4:4 + N]  # ldb = N + 8, base 16 bytes into each row
    Cw = torch.full((M, N + 12), 7.0, device="cuda")
    C = Cw[:, :N]
    pl = Plan.from_csr(rp, ci, val, (M, K))
    pl.spmm(B, C_out=C, engine="band")
    c_ref = oracle.pipeline(M, K, rp, ci, val, np.ascontiguousarray(B.cpu().numpy()))["C"]
    assert relerr(C.cpu().numpy(), c_ref) <= 1e-5
    assert torch.all(Cw[:, N:] == 7.0)  # columns beyond N untouched
    pl.close()


def test_band_set_values_equals_fresh_plan():
    M, K, rp, ci, val = build("band32_plus_rmat")
    B = torch.from_numpy(gen.dense_uniform(K, 128, seed=14)).cuda()
    pl = Plan.from_csr(rp, ci, val, (M, K))
    pl.spmm(B, engine="band")  # builds the split with the old values
    v2 = gen.uniform_values(len(ci), seed=99)
    pl.set_values(v2)
    C = pl.spmm(B, engine="band")
    fresh = Plan.from_csr(rp, ci, v2, (M, K))
    Cf = fresh.spmm(B, engine="band")
    assert torch.equal(C, Cf)
    c_ref = oracle.pipeline(M, K, rp, ci, v2, B.cpu().numpy())["C"]
    assert relerr(C.cpu().numpy(), c_ref) <= 1e-5
    pl.close()
    fresh.close()


def test_band_refusals_and_auto_fallback():
    M, K, rp, ci, val = build("band4_ragged_rows")
    pl = Plan.from_csr(rp, ci, val, (M, K))
    for N in (64, 130):  # N < 128, N % 4 != 0
        B = torch.from_numpy(gen.dense_uniform(K, N, seed=15)).cuda()
        with pytest.raises(SwiftError) as ei:
            pl.spmm(B, engine="band")
        assert ei.value.status == UNSUPPORTED
    B = torch.from_numpy(gen.dense_uniform(K, 128, seed=15)).cuda()
    with pytest.raises(SwiftError) as ei:
        pl.spmm(B.t().contiguous().t(), engine="band", layout="col")  # column-major B and C
    assert ei.value.status == UNSUPPORTED
    pl.close()
    p64 = Plan.from_csr(rp, ci, val.astype(np.float64), (M, K))
    with pytest.raises(SwiftError) as ei:
        p64.spmm(B.double(), engine="band")
    assert ei.value.status == UNSUPPORTED
    p64.close()


def test_band_autotune_picks_band_and_auto_runs_it():
    M, K, rp, ci, val = build("band32_plus_rmat")
    B = torch.from_numpy(gen.dense_uniform(K, 128, seed=16)).cuda()
    C = torch.empty(M, 128, device="cuda")
    pl = Plan.from_csr(rp, ci, val, (M, K))
    eng, ms = pl.autotune(B, C)
    assert eng in ("band", "rowwise", "tiled", "tiled_grouped") and ms > 0
    Ca = pl.spmm(B)
    c_ref = oracle.pipeline(M, K, rp, ci, val, B.cpu().numpy())["C"]
    assert relerr(Ca.cpu().numpy(), c_ref) <= 1e-5
    # column-major operands under AUTO still run (row walk on row-major copies)
    Bc = B.t().contiguous().t()  # the same B, column-major
    Cc = pl.spmm(Bc, layout="col")
    assert relerr(Cc.cpu().numpy(), c_ref) <= 1e-5
    pl.close()


@pytest.mark.parametrize("dt", ["float32", "bfloat16", "float16"])
def test_band_empty_and_tiny_matrices(dt):
    """No nonzeros at all (every C row written as zeros), fewer rows than one 16-row group, and
    fewer B rows than one 64-row chunk."""
    tdt = getattr(torch, dt)
    tol = 1e-5 if dt == "float32" else 1e-2
    B = torch.from_numpy(gen.dense_uniform(300, 128, seed=21)).cuda().to(tdt)
    rp = np.zeros(501, np.int32)
    pl = Plan.from_csr(rp, np.zeros(0, np.int32), np.zeros(0, np.float32), (500, 300))
    C = torch.full((500, 128), 5.0, device="cuda", dtype=tdt)
    pl.spmm(B, C_out=C, engine="band")
    assert torch.count_nonzero(C).item() == 0
    pl.close()
    for M, K in ((5, 300), (300, 40)):
        rp, ci = band_pattern(M, K, 3)
        val = gen.uniform_values(len(ci), seed=22)
        pl = Plan.from_csr(rp, ci, val, (M, K))
        Bk = B[:K].contiguous()
        C = pl.spmm(Bk, engine="band")
        ref = pl.spmm_f64_reference(Bk.double()).cpu().numpy()
        assert relerr(C.double().cpu().numpy(), ref) <= tol, (M, K)
        if dt == "float32":
            ref = oracle.pipeline(M, K, rp, ci, val, Bk.cpu().numpy())["C"]
            assert relerr(C.cpu().numpy(), ref) <= 1e-5
        pl.close()


@pytest.mark.parametrize("dt", ["float32", "bfloat16", "float16"])
@pytest.mark.parametrize("N", [128, 136, 200, 256, 512])  # 16-bit rows a multiple of 16 bytes
@pytest.mark.parametrize("shape", [(1000, 1000, 32), (1500, 1000, 16), (777, 1200, 4), (4096, 4096, 48),
                                   (2000, 2100, 64)])
def test_band_tensor_core_exact(shape, N, dt):
    """16-bit B runs the tiles on the tensor cores (hi + lo parts), FP32 B on CUDA cores.  With
    integer A in {-1, 1} and B in {-2..2} every partial and total sum is an integer below 256,
    exact in FP32, BF16 and FP16, so C must equal the FP64 product bit for bit: a value in the
    wrong fragment slot, B row or column, or a wrong row factor would show."""
    M, K, half = shape
    rp, ci = band_pattern(M, K, half, 0.002, seed=half)
    rng = np.random.default_rng(half + N)
    val = rng.choice(np.array([-1.0, 1.0], np.float32), len(ci))
    Bi = rng.integers(-2, 3, (K, N)).astype(np.float32)
    B = torch.from_numpy(Bi).cuda().to(getattr(torch, dt))
    pl = Plan.from_csr(rp, ci, val, (M, K))
    C = pl.spmm(B, engine="band")
    torch.cuda.synchronize()
    ref = pl.spmm_f64_reference(B.double()).cpu().numpy()
    assert np.abs(ref).max() < 256
    w = pl.band_profile()[1]
    assert w >= 0  # the band engine chose a tile width
    if half == 64:
        assert w == 63  # the widest tiles (136 columns; one block per SM)
    assert np.array_equal(C.double().cpu().numpy(), ref)
    pl.close()


@pytest.mark.parametrize("dt", ["bfloat16", "float16"])
def test_band_16bit_keeps_fp32_values(dt):
    """A's FP32 values reach the tensor cores as hi + lo parts of B's type: rows holding
    1 + 3 * 2^-12 and -1 against equal B rows must give 3 * 2^-12 (the hi parts alone would give
    0 in BF16 and 2^-10 in FP16)."""
    M = K = 512
    i = np.arange(M - 1, dtype=np.int64)
    rp, ci = gen.coo_to_csr(M, np.concatenate([i, i]), np.concatenate([i, i + 1]), K=K)
    rows = np.repeat(np.arange(M), np.diff(rp))
    val = np.where(ci == rows, np.float32(1 + 3 * 2.0 ** -12), np.float32(-1.0)).astype(np.float32)
    B = torch.ones(K, 128, device="cuda", dtype=getattr(torch, dt))
    pl = Plan.from_csr(rp, ci, val, (M, K))
    C = pl.spmm(B, engine="band")
    torch.cuda.synchronize()
    expect = np.full((M, 128), 3 * 2.0 ** -12)
    expect[M - 1] = 0.0
    assert np.array_equal(C.double().cpu().numpy(), expect)
    # new values for the same pattern reach the tensor cores too (the fragments are rebuilt)
    pl.set_values(np.where(val < 0, val, np.float32(1 + 5 * 2.0 ** -12)).astype(np.float32))
    C = pl.spmm(B, engine="band")
    torch.cuda.synchronize()
    expect[:M - 1] = 5 * 2.0 ** -12
    assert np.array_equal(C.double().cpu().numpy(), expect)
    pl.close()


def test_band_fp16_rows_beyond_fp16_range():
    """FP16 B with A rows of magnitude 1e5 (beyond FP16's 65504), 1 and 0.1: each row is scaled
    by a power of two before its FP16 split, so C stays finite and within FP16 output rounding of
    the FP64 product, row by row."""
    M = K = 2048
    rp, ci = band_pattern(M, K, 16)  # every nonzero in the tiles (no rest)
    rows = np.repeat(np.arange(M), np.diff(rp))
    mag = np.where(rows % 3 == 0, 1e5, np.where(rows % 3 == 1, 1.0, 0.1)).astype(np.float32)
    val = (gen.uniform_values(len(ci), seed=5) * mag).astype(np.float32)
    B = (torch.from_numpy(gen.dense_uniform(K, 128, seed=6)).cuda() * 2.0 ** -6).half()
    pl = Plan.from_csr(rp, ci, val, (M, K))
    C = pl.spmm(B, engine="band").double().cpu().numpy()
    ref = pl.spmm_f64_reference(B.double()).cpu().numpy()
    assert np.isfinite(C).all()
    err = np.abs(C - ref).max(axis=1) / np.maximum(np.abs(ref).max(axis=1), 1e-300)
    assert err.max() <= 1e-3, err.max()
    pl.close()


def test_band_fp32_accuracy():
    """FP32 B: the tiles' product stays within a few FP32 roundings of the FP64 product (the row
    walk alone reaches about 5e-7 on this matrix)."""
    M, K, rp, ci, val = build("band32_plus_rmat")
    B = torch.from_numpy(gen.dense_uniform(K, 128, seed=17)).cuda()
    pl = Plan.from_csr(rp, ci, val, (M, K))
    C = pl.spmm(B, engine="band")
    ref = pl.spmm_f64_reference(B.double()).cpu().numpy()
    assert relerr(C.cpu().numpy(), ref) <= 2e-6
    pl.close()


@pytest.mark.parametrize("dt", ["bfloat16", "float16"])
def test_band_16bit_strided_operands(dt):
    """16-bit B and C as views with leading dimensions beyond N (rows 16-byte multiples, B 16
    bytes into each row): the TMA boxes follow the strides and the C tile store leaves the
    columns beyond N untouched."""
    M, K, rp, ci, val = build("band32_plus_rmat")
    N = 128
    tdt = getattr(torch, dt)
    Bw = torch.from_numpy(gen.dense_uniform(K, N + 16, seed=23)).cuda().to(tdt)
    B = Bw[:, 8:8 + N]
    Cw = torch.full((M, N + 24), 7.0, device="cuda", dtype=tdt)
    C = Cw[:, :N]
    pl = Plan.from_csr(rp, ci, val, (M, K))
    pl.spmm(B, C_out=C, engine="band")
    ref = pl.spmm_f64_reference(B.contiguous().double()).cpu().numpy()
    assert relerr(C.double().cpu().numpy(), ref) <= 1e-2
    assert torch.all(Cw[:, N:] == 7.0)
    Cd = pl.spmm(B.contiguous(), engine="band")
    assert torch.equal(C, Cd)  # the same product as with dense operands
    pl.close()



def test_band_bf16_and_fp16_products_alternate():
    """BF16 and FP16 products on one plan keep separate tile layouts: alternating them gives the
    results of the first products bit for bit (and rebuilds nothing)."""
    M, K, rp, ci, val = build("band32_plus_rmat")
    B32 = torch.from_numpy(gen.dense_uniform(K, 128, seed=31)).cuda()
    Bb, Bh = B32.to(torch.bfloat16), B32.half()
    pl = Plan.from_csr(rp, ci, val, (M, K))
    Cb = pl.spmm(Bb, engine="band")
    Ch = pl.spmm(Bh, engine="band")
    C32 = pl.spmm(B32, engine="band")
    for _ in range(2):
        assert torch.equal(pl.spmm(Bb, engine="band"), Cb)
        assert torch.equal(pl.spmm(Bh, engine="band"), Ch)
        assert torch.equal(pl.spmm(B32, engine="band"), C32)
    pl.close()


def test_band_no_timeouts():
    from swift_b200 import _capi as capi
    import ctypes as C
    f = C.c_int(-1)
    capi.check(capi.lib().swift_band_timeout_flag(C.byref(f), 0), "swift_band_timeout_flag")
    assert f.value == 0
