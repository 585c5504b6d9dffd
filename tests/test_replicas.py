"""The N > 1 path of bench.py (replicas): two gloo ranks on CPU agree on the
slowest rank's time and count both ranks' steps."""
import os
import socket

import pytest
import torch.distributed as dist
import torch.multiprocessing as mp

from nonstationary_mra_b200 import replicas


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    ms = [100.0 + 50.0 * rank, 200.0 - 10.0 * rank]   # rank 1 slower in the first, faster in the second
    got = replicas.max_over_ranks(ms)
    out[rank] = (got, replicas.job_throughput(5, world, got[0]))
    dist.barrier()
    dist.destroy_process_group()


def test_two_ranks_take_the_max_and_count_all_steps():
    port = _free_port()
    with mp.Manager() as m:
        out = m.dict()
        mp.spawn(_rank, args=(2, port, out), nprocs=2, join=True)
        res = dict(out)
    for rank in (0, 1):
        got, thr = res[rank]
        assert got == [150.0, 200.0]
        assert thr == pytest.approx(2 * 5 / 0.150)


def test_single_process_is_identity():
    assert replicas.max_over_ranks([3.0, 4.0]) == [3.0, 4.0]
    assert replicas.job_throughput(10, 1, 500.0) == pytest.approx(20.0)
