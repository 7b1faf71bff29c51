"""The multi-GPU path of bench.py is replicas only (independent solves, no data exchange): its
host logic — the max-over-ranks timing reduction and the per-rank permeability seeds — runs here
as two gloo ranks on the CPU, with the same functions the NCCL ranks call."""
import os
import socket
import sys

import pytest

torch = pytest.importorskip("torch")
import torch.distributed as dist  # noqa: E402
import torch.multiprocessing as mp  # noqa: E402

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, out):
    sys.path.insert(0, ROOT)
    import datetime

    import bench
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        # each rank times a different value; every rank receives the largest
        got = bench.max_over_ranks(10.0 * (rank + 1), dist)
        seeds = [None] * world
        dist.all_gather_object(seeds, bench.replica_seed(2026, rank))
        out.put((rank, got, seeds))
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_reduce_the_max_and_use_distinct_seeds():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = sorted(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert [r[1] for r in res] == [20.0, 20.0]
    seeds = res[0][2]
    assert len(set(seeds)) == 2 and res[1][2] == seeds


def test_single_process_needs_no_process_group():
    sys.path.insert(0, ROOT)
    import bench
    assert bench.max_over_ranks(3.5, None) == 3.5


def test_reference_arm_other_ranks_do_no_work(capsys):
    """Under torchrun only rank 0 runs and prints the reference arm; the others return at once."""
    sys.path.insert(0, ROOT)
    import bench
    bench.reference_arm(None, rank=1)
    assert capsys.readouterr().out == ""
