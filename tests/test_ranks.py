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


def _ranked_main(rank, world, port, out):
    """bench.run_ranked, the bench's own rank entry, with a CPU body: each rank
    times a different replica; rank 0 alone prints the line."""
    import io
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world))
    sys.path.insert(0, ROOT)
    import bench
    buf = io.StringIO()

    def body(r, w):
        secs = bench.max_over_ranks(0.5 * (r + 1), w, torch.device("cpu"))
        return {"rank": r, "n_gpus": w, "seconds": secs}

    line = bench.run_ranked(body, rank, world, backend="gloo", out=buf)
    out[rank] = (line, buf.getvalue(), dist.is_initialized())


def test_bench_rank_entry_two_gloo_ranks():
    world = 2
    port = _free_port()
    with mp.Manager() as mgr:
        out = mgr.dict()
        mp.start_processes(_ranked_main, args=(world, port, out), nprocs=world, join=True, start_method="spawn")
        res = dict(out)
    assert sorted(res) == [0, 1]
    for r in range(world):
        line, printed, still_joined = res[r]
        assert line["seconds"] == pytest.approx(1.0)  # the slower rank's time on both
        assert not still_joined  # the group is left
        assert (printed != "") == (r == 0)  # one JSON line, from rank 0
    import json
    assert json.loads(res[0][1]) == {"rank": 0, "n_gpus": 2, "seconds": 1.0}


def test_gpus_flag_resolves_world_size():
    sys.path.insert(0, ROOT)
    import bench
    assert bench.resolve_world(1, {}) == (0, 1, False)
    assert bench.resolve_world(4, {}) == (0, 1, True)  # relaunch under torchrun
    assert bench.resolve_world(2, {"WORLD_SIZE": "2", "RANK": "1"}) == (1, 2, False)
    with pytest.raises(SystemExit):
        bench.resolve_world(8, {"WORLD_SIZE": "1"})  # would time one GPU as eight
    with pytest.raises(SystemExit):
        bench.resolve_world(0, {})
    cmd = bench.torchrun_command(4, 29511, ["--steps", "20"])
    assert cmd[1:3] == ["-m", "torch.distributed.run"]
    assert "--nproc-per-node=4" in cmd and cmd[cmd.index("--master-addr") + 1] == "127.0.0.1"
    assert cmd[-3].endswith("bench.py") and cmd[-2:] == ["--steps", "20"]
