"""Replica timing over a world-size-2 gloo process group on CPU: the time is
the maximum over ranks and the throughput counts every rank's units."""
import os
import socket

import pytest

torch = pytest.importorskip("torch")
import torch.distributed as dist  # noqa: E402
import torch.multiprocessing as mp  # noqa: E402


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _rank(rank, world, port, q):
    import datetime
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    from mbx_b200 import replicas
    mine = [1.0 + rank, 5.0 - rank, 2.5]
    got = replicas.max_over_ranks(mine, dist, "cpu")
    q.put((rank, got, replicas.throughput(1000, got[0], world)))
    dist.barrier()
    dist.destroy_process_group()


def test_max_over_two_ranks():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = [q.get(timeout=120) for _ in procs]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for rank, got, tput in res:
        assert got == [2.0, 5.0, 2.5]
        assert tput == 2 * 1000 / 2e-3


def test_single_process_passthrough():
    from mbx_b200 import replicas
    assert replicas.max_over_ranks([3.0, 4.0]) == [3.0, 4.0]
