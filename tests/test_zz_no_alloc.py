"""swift_spmm_noalloc: the product entry point for callers that cannot allocate device memory
while running (allocation forbidden after start-up, or device memory owned by another
allocator).  It must give the product of the regular entry point, through the C ABI, on
consecutive calls that reuse its fixed scratch array, and refuse products beyond that array.

This file is collected last on purpose, so that a run stopping at the first failure has
already run every other test; it also passes alone in a fresh process."""
import ctypes as C

import numpy as np
import pytest

import cases
import oracle
from swift_b200 import Plan, capi, gen

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu


def _relerr(x, ref):
    x = np.asarray(x, np.float64)
    ref = np.asarray(ref, np.float64)
    return float(np.abs(x - ref).max() / max(np.abs(ref).max(), 1e-300))


_CODE = {torch.float32: capi.F32, torch.float64: capi.F64, torch.bfloat16: capi.BF16, torch.float16: capi.F16}


def _noalloc(plan, B, Cout):
    stream = C.c_void_p(torch.cuda.current_stream().cuda_stream)
    N = int(B.shape[1])
    return capi.lib().swift_spmm_noalloc(plan.handle, N, _CODE[B.dtype], B.data_ptr(), B.stride(0),
                                         Cout.data_ptr(), Cout.stride(0), stream)


@pytest.mark.parametrize("N", [32, 128])
def test_noalloc_matches_regular_entry_point_on_consecutive_calls(N):
    M, K, rp, ci = cases.make("rmat12", 2)
    val = gen.uniform_values(int(rp[-1]), 1, np.float32)
    Bn = gen.dense_uniform(K, N, 2, np.float32)
    # a small split threshold makes long rows, so the scratch array is really used
    plan = Plan.from_csr(rp, ci, val, (M, K), long_row_split=32)
    assert plan.stats()["long_pieces"] > 0
    B = torch.from_numpy(Bn).cuda()
    c_regular = plan.spmm(B, engine="rowwise").cpu().numpy()
    ref = oracle.csr_spmm_f64(M, K, rp, ci, val, Bn)
    previous = None
    for _ in range(2):
        out = torch.full((M, N), float("nan"), dtype=torch.float32, device="cuda")
        assert _noalloc(plan, B, out) == capi.OK, capi.lib().swift_last_error()
        torch.cuda.synchronize()
        got = out.cpu().numpy()
        assert _relerr(got, c_regular) <= 1e-5
        assert _relerr(got, ref) <= 1e-5
        if previous is not None:
            assert np.array_equal(got, previous)  # the partial rows add up in a fixed order
        previous = got
    plan.close()


def test_noalloc_refuses_products_beyond_its_array():
    M, K, rp, ci = cases.make("rmat12", 2)
    val = gen.uniform_values(int(rp[-1]), 1, np.float32)
    plan = Plan.from_csr(rp, ci, val, (M, K), long_row_split=16)
    pieces = plan.stats()["long_pieces"]
    N = 4096  # pieces * N * 4 bytes exceeds the 16 MiB array
    assert pieces * N * 4 > (16 << 20)
    B = torch.zeros((K, N), dtype=torch.float32, device="cuda")
    out = torch.zeros((M, N), dtype=torch.float32, device="cuda")
    assert _noalloc(plan, B, out) == capi.ERR_OVERFLOW
    assert b"long_row_split" in capi.lib().swift_last_error()
    plan.close()


# 16-bit B and C (FP32 values, FP32 accumulation) and FP64 plans against the regular entry
# point and the FP64 product on the same (rounded) B: within 1e-2 for 16-bit C, 1e-12 for FP64
@pytest.mark.parametrize("dt", ["bf16", "f16", "f64"])
@pytest.mark.parametrize("N", [32, 128])
def test_noalloc_other_operand_types(dt, N):
    M, K, rp, ci = cases.make("rmat12", 3)
    vdt = np.float64 if dt == "f64" else np.float32
    tdt = {"bf16": torch.bfloat16, "f16": torch.float16, "f64": torch.float64}[dt]
    val = gen.uniform_values(int(rp[-1]), 1, vdt)
    plan = Plan.from_csr(rp, ci, val, (M, K), long_row_split=32)
    assert plan.stats()["long_pieces"] > 0
    B = torch.from_numpy(gen.dense_uniform(K, N, 4, np.float64)).cuda().to(tdt)
    c_regular = plan.spmm(B, engine="rowwise")
    ref = oracle.csr_spmm_f64(M, K, rp, ci, val, B.double().cpu().numpy())
    tol = 1e-12 if dt == "f64" else 1e-2
    previous = None
    for _ in range(2):
        out = torch.full((M, N), float("nan"), dtype=tdt, device="cuda")
        assert _noalloc(plan, B, out) == capi.OK, capi.lib().swift_last_error()
        torch.cuda.synchronize()
        got = out.double().cpu().numpy()
        assert _relerr(got, c_regular.double().cpu().numpy()) <= tol
        assert _relerr(got, ref) <= tol
        if previous is not None:
            assert torch.equal(out, previous)
        previous = out
    # an FP64 B on an FP32 plan (or the reverse) is refused
    wrong = torch.zeros((K, N), dtype=torch.float32 if dt == "f64" else torch.float64, device="cuda")
    wout = torch.zeros((M, N), dtype=wrong.dtype, device="cuda")
    assert _noalloc(plan, wrong, wout) == capi.ERR_UNSUPPORTED
    plan.close()
