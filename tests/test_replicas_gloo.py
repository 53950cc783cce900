"""The multi-process path of bench.py on CPU: two gloo ranks, as `torchrun --nproc-per-node 2`
would start them.  The product has no exchange step, so the only cross-rank logic is timing:
every rank's device time is reduced to the maximum (the job is as slow as its slowest
replica) and the whole-job rate counts every replica's work."""
import os
import socket

import pytest

torch = pytest.importorskip("torch")
import torch.distributed as dist  # noqa: E402
import torch.multiprocessing as mp  # noqa: E402


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, q):
    import datetime
    import sys
    sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
    import bench
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        ms = 10.0 + 5.0 * rank  # rank 1 is the slower replica
        slowest = bench.max_over_ranks(ms, dist, device="cpu")
        rate = bench.whole_job_rate(100.0, world, slowest / 1e3)
        dist.barrier()
        q.put((rank, slowest, rate))
    finally:
        dist.destroy_process_group()


def test_two_replicas_report_the_slowest_time_and_the_summed_work():
    world, port = 2, _free_port()
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_rank_main, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=120)
    assert all(p.exitcode == 0 for p in procs), [p.exitcode for p in procs]
    got = sorted(q.get(timeout=10) for _ in range(world))
    for rank, slowest, rate in got:
        assert slowest == 15.0
        assert rate == pytest.approx(world * 100.0 / 0.015)


def test_single_process_needs_no_group():
    import sys
    sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
    import bench
    assert bench.max_over_ranks(3.5, None) == 3.5
    assert bench.whole_job_rate(10.0, 1, 2.0) == 5.0


def test_profile_summaries_map_to_their_own_workload():
    """Each committed ncu summary is found for its own workload only (a workload name that ends
    another one's must not pick up the other's DRAM traffic)."""
    import glob
    import sys
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    sys.path.insert(0, root)
    import bench
    seen = 0
    for path in glob.glob(os.path.join(root, "profiles", "*.txt")):
        with open(path) as f:
            wl = next((ln.split(":", 1)[1].split()[0] for ln in f if ln.startswith("workload:")), None)
        if wl is None:
            continue
        seen += 1
        assert wl in bench.WORKLOADS, wl
        assert bench.profile_summary(wl)["file"] == os.path.relpath(path, root)
    assert seen >= 2
