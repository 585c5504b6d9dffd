"""Sub-tree sharding on the GPU (mra_shard_*): the sharded log-likelihood is
bitwise the whole evaluation's.  Two contexts in one process stand for two
ranks, and then two gloo processes run the real exchange (shard.loglik); the
ranks share one GPU, which is safe because no kernel waits on another rank:
the exchange happens on the host between launches."""
import os
import socket

import numpy as np
import pytest
import torch.distributed as dist
import torch.multiprocessing as mp

from nonstationary_mra_b200 import api, capi, shard

from test_gpu_parity import random_case

pytestmark = pytest.mark.gpu

CASE = (6, 4, 5, 16, 3000, 0, True, 3, True)      # clustered, M = 5: split levels 1 and 2


def _whole(st, md):
    ctx = api.Context(st, md)
    ctx.set_theta()
    d, ll = ctx.loglik()
    ctx.close()
    return d, ll


@pytest.mark.parametrize("split", [1, 2])
def test_two_contexts_give_the_whole_loglik_bitwise(split):
    api.set_device(0)
    st, md = random_case(*CASE)
    d0, ll0 = _whole(st, md)
    n_sub = st.J ** split
    owner = np.arange(n_sub) % 2
    a, b = api.Context(st, md), api.Context(st, md)
    for ctx in (a, b):
        ctx.set_theta()
    a.shard_set(split, owner == 0)
    b.shard_set(split, owner == 1)
    a.shard_subtrees()
    b.shard_subtrees()
    for q in np.nonzero(owner == 1)[0]:
        a.shard_import(int(q), b.shard_export(int(q)))
    d, ll = a.shard_top()
    assert d == d0 and ll == ll0
    # whole-tree calls are refused while sharded, and work again once cleared
    with pytest.raises(capi.MRAError) as e:
        a.loglik()
    assert e.value.status == capi.MRA_ERR_STATE
    a.shard_set(split, None)
    assert a.loglik()[0] == d0
    a.close()
    b.close()


def test_shard_arguments_are_checked():
    api.set_device(0)
    st, md = random_case(*CASE)
    ctx = api.Context(st, md)
    for bad in (0, st.M - 2):
        with pytest.raises(capi.MRAError):
            ctx.shard_set(bad, np.ones(st.J ** max(bad, 1), dtype=bool))
    ctx.shard_set(1, np.ones(st.J, dtype=bool))
    with pytest.raises(capi.MRAError):
        ctx.shard_import(0, np.zeros(3))      # wrong record size
    ctx.close()


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    api.set_device(0)
    st, md = random_case(*CASE)
    sp = shard.plan(st, world, split=2)
    ctx = api.Context(st, md)
    ctx.set_theta()
    d, ll = shard.loglik(ctx, sp, rank, world)
    ctx.close()
    out[rank] = (d, ll, int((sp.owner == rank).sum()))
    dist.barrier()
    dist.destroy_process_group()


def test_two_gloo_ranks_match_the_whole_evaluation():
    st, md = random_case(*CASE)
    api.set_device(0)
    d0, ll0 = _whole(st, md)
    port = _free_port()
    # every helper process is spawned, none forked: this process already uses the GPU
    with mp.get_context("spawn").Manager() as m:
        out = m.dict()
        mp.spawn(_rank, args=(2, port, out), nprocs=2, join=True)
        res = dict(out)
    for rank in (0, 1):
        assert res[rank][0] == d0 and res[rank][1] == ll0
    assert res[0][2] + res[1][2] == st.J ** 2 and min(res[0][2], res[1][2]) > 0
