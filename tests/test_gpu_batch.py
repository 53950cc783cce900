"""Batched products in one persistent launch (swift_batch_*): every member against the
deterministic FP64 product of its own plan (normwise 1e-5), bit-identical repeats, CUDA-graph
replay equal to the plain launch, new operands picked up by a captured graph, autotuning,
the N-split (members walked as two column halves) bit-equal to the unsplit launch."""
import numpy as np
import pytest

from swift_b200 import Plan, capi, gen
from swift_b200.plan import Batch

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu


def relerr(x, ref):
    x = x.double()
    d = ref.abs().max().item() if ref.numel() else 1.0
    return (x - ref).abs().max().item() / max(d, 1e-300) if ref.numel() else 0.0


def members(count, seed, extra=True):
    ms = gen.batch_matrices(count, seed=seed, m_lo=256, m_hi=8192, device="cuda")
    if extra:  # unaligned widths (scalar path), an empty matrix, a single long row
        ms.append(dict(M=300, rowptr=gen.random_csr(300, 300, 0.05, seed=1)[0],
                       colidx=gen.random_csr(300, 300, 0.05, seed=1)[1], N=18, kind="unaligned"))
        ms.append(dict(M=64, rowptr=np.zeros(65, np.int32), colidx=np.zeros(0, np.int32), N=64, kind="empty"))
        rp = np.array([0, 4000] + [4000] * 9, np.int32)
        ms.append(dict(M=10, rowptr=rp, colidx=np.sort(np.random.default_rng(3).choice(5000, 4000, replace=False)).astype(np.int32),
                       N=128, kind="long_row"))
    for i, m in enumerate(ms):
        m.setdefault("K", m["M"] if m["kind"] != "long_row" else 5000)
        m["val"] = gen.uniform_values(len(m["colidx"]), seed=100 + i)
    return ms


def build(ms, seed):
    g = torch.Generator(device="cuda")
    g.manual_seed(seed)
    plans, Bs, Cs = [], [], []
    for m in ms:
        plans.append(Plan.from_csr(m["rowptr"], m["colidx"], m["val"], (m["M"], m["K"])))
        Bs.append(torch.rand((m["K"], m["N"]), generator=g, device="cuda") * 2 - 1)
        Cs.append(torch.full((m["M"], m["N"]), float("nan"), device="cuda"))
    return plans, Bs, Cs


def test_batch_matches_each_plan():
    ms = members(24, seed=5)
    plans, Bs, Cs = build(ms, 0)
    b = Batch(plans)
    b.set_operands(Bs, Cs)
    b.run()
    torch.cuda.synchronize()
    first = [c.clone() for c in Cs]
    for p, B, C, m in zip(plans, Bs, Cs, ms):
        ref = p.spmm_f64_reference(B.double())
        assert relerr(C, ref) <= 1e-5, m["kind"]
    b.run()
    torch.cuda.synchronize()
    for c0, c in zip(first, Cs):
        assert torch.equal(c0, c)  # deterministic: split rows combined in task order
    for c in Cs:
        c.fill_(float("nan"))
    b.run_graph()
    b.run_graph()
    torch.cuda.synchronize()
    for c0, c in zip(first, Cs):
        assert torch.equal(c0, c)
    # new operands: the captured graph reads the updated launch table
    Bs2 = [torch.rand_like(B) for B in Bs]
    Cs2 = [torch.empty_like(C) for C in Cs]
    b.set_operands(Bs2, Cs2)
    b.run_graph()
    torch.cuda.synchronize()
    for p, B, C in zip(plans, Bs2, Cs2):
        assert relerr(C, p.spmm_f64_reference(B.double())) <= 1e-5
    b.close()


def test_batch_autotune_keeps_results():
    ms = members(10, seed=9, extra=False)
    plans, Bs, Cs = build(ms, 1)
    b = Batch(plans)
    b.set_operands(Bs, Cs)
    U, ms_run = b.autotune()
    sizes = b.task_sizes()
    assert U in (128, 256, 512, 1024) and ms_run > 0
    assert sizes[2] == U and all(s in (128, 256, 512, 1024) for s in sizes)
    assert all(s in (1, 2) for s in b.n_split())
    for c in Cs:
        c.fill_(float("nan"))
    b.run()
    torch.cuda.synchronize()
    for p, B, C in zip(plans, Bs, Cs):
        assert relerr(C, p.spmm_f64_reference(B.double())) <= 1e-5
    b.close()


@pytest.mark.parametrize("splits", [(2, 2, 2), (1, 2, 1), (2, 1, 2)])
def test_batch_n_split_matches_unsplit(splits):
    """Members walked as two column halves (each its own launch entry, tasks and split-row
    scratch): every member within 1e-5 of its FP64 product and bit-equal to the unsplit batch
    (each C element is summed in the same order); members whose N is not a multiple of 8 stay
    whole; a captured graph is re-captured when the entry count changes."""
    ms = members(24, seed=6)
    plans, Bs, Cs = build(ms, 3)
    b = Batch(plans)
    b.set_operands(Bs, Cs)
    b.run_graph()
    torch.cuda.synchronize()
    whole = [c.clone() for c in Cs]
    b.set_n_split(splits)
    assert b.n_split() == list(splits)
    for c in Cs:
        c.fill_(float("nan"))
    b.run()
    torch.cuda.synchronize()
    for p, B, C, W, m in zip(plans, Bs, Cs, whole, ms):
        assert relerr(C, p.spmm_f64_reference(B.double())) <= 1e-5, m["kind"]
        assert torch.equal(C, W), m["kind"]
    for c in Cs:
        c.fill_(float("nan"))
    b.run_graph()  # the table now has more entries: the graph is captured again
    torch.cuda.synchronize()
    for C, W in zip(Cs, whole):
        assert torch.equal(C, W)
    b.set_n_split((1, 1, 1))
    b.run_graph()
    torch.cuda.synchronize()
    for C, W in zip(Cs, whole):
        assert torch.equal(C, W)
    with pytest.raises(capi.SwiftError):
        b.set_n_split((3, 1, 1))
    b.close()


def test_destroy_waits_for_its_own_streams_only():
    """Destroying a batch or a plan waits for the launches it enqueued, not for the device: with
    another stream busy (a bounded spin of about a second), both destroys return while that
    stream is still running, and the products they waited for are complete and correct."""
    ms = members(6, seed=11, extra=False)
    plans, Bs, Cs = build(ms, 4)
    b = Batch(plans)
    b.set_operands(Bs, Cs)
    work, busy = torch.cuda.Stream(), torch.cuda.Stream()
    b.run(stream=work)
    torch.cuda.synchronize()
    p0, B0 = plans[0], Bs[0]
    C0 = torch.empty_like(Cs[0])
    with torch.cuda.stream(busy):
        torch.cuda._sleep(int(2e9))  # about a second of SM clock on this stream only
    for c in Cs:
        c.fill_(float("nan"))
    b.run(stream=work)
    p0.spmm(B0, C_out=C0, stream=work)
    b.close()
    p0.close()
    assert not busy.query()  # neither destroy waited for the busy stream
    work.synchronize()
    for p, B, C in zip(plans[1:], Bs[1:], Cs[1:]):
        assert relerr(C, p.spmm_f64_reference(B.double())) <= 1e-5
    assert torch.isfinite(C0).all() and torch.isfinite(Cs[0]).all()
    torch.cuda.synchronize()
    for p in plans[1:]:
        p.close()


def test_batch_rejects_unsupported():
    m = members(2, seed=2, extra=False)
    plans, Bs, Cs = build(m, 2)
    b = Batch(plans)
    wide = [torch.rand((x["K"], 200), device="cuda") for x in m]
    with pytest.raises(capi.SwiftError) as e:
        b.set_operands(wide, [torch.empty((x["M"], 200), device="cuda") for x in m])
    assert e.value.status == capi.ERR_UNSUPPORTED
    with pytest.raises(capi.SwiftError) as e:
        b.run()  # operands never set successfully
    assert e.value.status == capi.ERR_INVALID_ARG
    b.close()
    p64 = Plan.from_csr(m[0]["rowptr"], m[0]["colidx"], m[0]["val"].astype(np.float64), (m[0]["M"], m[0]["K"]))
    with pytest.raises(capi.SwiftError) as e:
        Batch([p64])
    assert e.value.status == capi.ERR_UNSUPPORTED
