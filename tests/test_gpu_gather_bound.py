"""The gather-ceiling measurement (swift_gather_bound) through the C ABI: it gathers exactly
the B rows of A's column stream (checksum against torch), returns positive per-launch times,
and refuses the shapes it does not cover."""
import numpy as np
import pytest

from swift_b200 import Plan, gen
from swift_b200._capi import SwiftError, ERR_INVALID_ARG, ERR_UNSUPPORTED

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("N", [32, 64, 128])
def test_gather_bound_checksum_and_times(N):
    rp, ci = gen.rmat(13, 16 << 13, seed=3)
    M = 1 << 13
    val = gen.uniform_values(len(ci), seed=4)
    pl = Plan.from_csr(rp, ci, val, (M, M))
    B = torch.from_numpy(gen.dense_uniform(M, N, seed=5)).cuda()
    ms, ms_l1, chk = pl.gather_bound(B, reps=3)
    ref = B.double()[torch.from_numpy(ci.astype(np.int64)).cuda()].sum().item()
    assert ms > 0 and ms_l1 > 0
    assert abs(chk - ref) <= 1e-4 * max(1.0, B.double().abs()[torch.from_numpy(ci.astype(np.int64)).cuda()].sum().item())
    pl.close()


def test_gather_bound_refusals():
    rp, ci = gen.rmat(10, 8 << 10, seed=3)
    pl = Plan.from_csr(rp, ci, gen.uniform_values(len(ci), seed=4), (1024, 1024))
    with pytest.raises(SwiftError) as ei:
        pl.gather_bound(torch.zeros(1024, 96, device="cuda"))
    assert ei.value.status == ERR_INVALID_ARG
    pl.close()
    rp, ci = gen.random_csr(100, 100, 0.05, seed=1)
    small = Plan.from_csr(rp, ci, gen.uniform_values(len(ci), seed=2), (100, 100))
    with pytest.raises(SwiftError) as ei:
        small.gather_bound(torch.zeros(100, 32, device="cuda"))
    assert ei.value.status == ERR_UNSUPPORTED
    small.close()
