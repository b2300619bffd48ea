"""The multi-rank logic of bench.py on CPU: two gloo ranks over 127.0.0.1.

bench.py runs one replica of the workload per GPU ("replicas only": no data
collective).  Across ranks it needs exactly two decisions, which these tests
drive through the same helpers the bench calls: the timed seconds are the
slowest rank's, and a capacity retry or a hard failure on any rank is taken
by every rank, so that all ranks issue the same collectives in the same order.
"""
import os
import socket
import sys

import pytest

torch = pytest.importorskip("torch")
import torch.distributed as dist  # noqa: E402
import torch.multiprocessing as mp  # noqa: E402

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, out):
    import datetime
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    sys.path.insert(0, ROOT)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        import bench
        dev = torch.device("cpu")
        res = {"max": bench.max_over_ranks(1.5 + rank, world, dev)}
        res["clean"] = bench.retry_verdict(0, False, world, dev)
        # rank 0 overflowed and grew its capacity, rank 1 was clean: both time again
        res["grow"] = bench.retry_verdict(3 if rank == 0 else 0, rank == 0, world, dev)
        # rank 1 failed for good, rank 0 grew: both stop
        res["fail"] = bench.retry_verdict(3, rank == 0, world, dev)
        out[rank] = res
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_agree_on_timing_and_retries():
    world = 2
    port = _free_port()
    with mp.Manager() as mgr:
        out = mgr.dict()
        mp.start_processes(_rank_main, args=(world, port, out), nprocs=world, join=True, start_method="spawn")
        res = dict(out)
    assert sorted(res) == [0, 1]
    for r in range(world):
        assert res[r]["max"] == pytest.approx(2.5)  # the slower rank's seconds
        assert res[r]["clean"] == 0
        assert res[r]["grow"] == 1
        assert res[r]["fail"] == 2


def test_single_rank_needs_no_process_group():
    sys.path.insert(0, ROOT)
    import bench
    dev = torch.device("cpu")
    assert bench.max_over_ranks(0.25, 1, dev) == 0.25
    assert bench.retry_verdict(0, False, 1, dev) == 0
    assert bench.retry_verdict(3, True, 1, dev) == 1
    assert bench.retry_verdict(4, False, 1, dev) == 2
