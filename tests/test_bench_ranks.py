"""Host logic of `bench.py --gpus N` on CPU: N ranks as gloo processes
(world size 2).  Each rank times its own replica; the reported times are the
maximum over the ranks, which every rank receives from one collective."""
import multiprocessing as mp
import os
import socket
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, q):
    sys.path.insert(0, ROOT)
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    import datetime
    import torch.distributed as dist
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    import bench
    # rank r is slowest on value r
    times = [1.0 + (rank == 0), 1.0 + 2 * (rank == 1), 0.5]
    q.put((rank, bench.max_over_ranks(times, world, "cpu")))
    dist.barrier()
    dist.destroy_process_group()


def test_max_over_ranks_gloo_two_ranks():
    pytest.importorskip("torch")
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    got = dict(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert got[0] == got[1] == [2.0, 3.0, 0.5]


def test_max_over_ranks_single_rank_is_identity():
    sys.path.insert(0, ROOT)
    import bench
    assert bench.max_over_ranks([1, 2.5], 1, "cpu") == [1.0, 2.5]


def test_reference_arm_other_ranks_exit_quietly(capsys, monkeypatch):
    """Under torchrun only rank 0 runs and prints the reference arm."""
    sys.path.insert(0, ROOT)
    import bench
    monkeypatch.setenv("RANK", "1")
    monkeypatch.setenv("WORLD_SIZE", "2")
    monkeypatch.setattr(sys, "argv", ["bench.py", "--impl", "reference", "--gpus", "2"])
    bench.main()
    assert capsys.readouterr().out == ""
