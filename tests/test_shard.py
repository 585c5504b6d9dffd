"""Sub-tree sharding, host side (nonstationary_mra_b200/shard.py): the LPT plan,
and the exchange protocol between two gloo ranks on CPU with a stand-in
context that records what each rank computes, exports and imports."""
import os
import socket

import numpy as np
import pytest
import torch.distributed as dist
import torch.multiprocessing as mp

from nonstationary_mra_b200 import partition, shard


def _structure(seed=3, n=4000, J=4, M=6, r=9):
    rng = np.random.default_rng(seed)
    c = rng.random((2, 4))
    xy = np.clip(c[:, rng.integers(0, 4, n)] + 0.05 * rng.standard_normal((2, n)), 0, 1)
    return partition.build_by_program(xy[0], xy[1], rng.standard_normal(n), J, M, r, np.exp(1) / 100,
                                      distance=2, all_lon=xy[0], all_lat=xy[1])


def test_plan_assigns_every_subtree_once_and_balances():
    st = _structure()
    for world in (1, 2, 3, 4):
        sp = shard.plan(st, world)
        assert 1 <= sp.split <= st.M - 3
        assert sp.owner.shape == (st.J ** sp.split,)
        assert set(np.unique(sp.owner)) <= set(range(world))
        loads = np.array([sp.cost[sp.owner == k].sum() for k in range(world)])
        np.testing.assert_allclose(loads, sp.load)
        # LPT bound: no rank above the mean by more than the largest sub-tree
        assert loads.max() <= loads.mean() + sp.cost.max() + 1e-9
        assert np.array_equal(sp.owner, shard.plan(st, world).owner)   # deterministic


def test_split_level_choice():
    assert shard.choose_split(4, 10, 1) == 1
    assert shard.choose_split(4, 10, 8) == 3      # 64 sub-trees >= 4 per rank
    assert shard.choose_split(2, 5, 8) == 2       # capped at M-3
    with pytest.raises(ValueError):
        shard.choose_split(4, 3, 2)


def test_costs_follow_the_observations():
    st = _structure()
    c = shard.subtree_costs(st, 1)
    n = np.diff(st.obs_offset).reshape(st.J, -1).sum(axis=1)
    assert np.argmax(c) == np.argmax(n) and np.argmin(c) == np.argmin(n)


class FakeContext:
    """Stand-in for api.Context: a sub-tree's record is a function of its index;
    the top evaluation sums every record in sub-tree order, so rank 0 returns
    exactly the single-context value only if it received every record once."""

    def __init__(self, n_sub, log):
        self.n_sub, self.log, self.owned, self.imported, self.ran = n_sub, log, None, {}, False

    def shard_set(self, split, owned):
        self.owned = None if owned is None else np.asarray(owned, dtype=bool)

    def shard_subtrees(self):
        self.ran = True
        self.log.append(("subtrees", int(self.owned.sum())))

    @staticmethod
    def record(q):
        return np.array([q, 0.5 * q, (q + 1) ** 2], dtype=np.float64)

    def shard_export(self, q):
        assert self.ran and self.owned[q]
        return self.record(q)

    def shard_import(self, q, rec):
        assert not self.owned[q] and q not in self.imported
        np.testing.assert_array_equal(rec, self.record(q))
        self.imported[q] = rec

    def shard_top(self):
        assert len(self.imported) + int(self.owned.sum()) == self.n_sub
        d = sum(float(self.record(q).sum()) for q in range(self.n_sub))
        return d, -0.5 * d


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, owner, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    sp = shard.ShardPlan(split=2, owner=np.asarray(owner), cost=np.ones(len(owner)), load=np.zeros(world))
    log = []
    ctx = FakeContext(len(owner), log)
    d, ll = shard.loglik(ctx, sp, rank, world)
    out[rank] = (d, ll, len(ctx.imported), log, ctx.owned is None)
    dist.barrier()
    dist.destroy_process_group()


def test_two_gloo_ranks_exchange_every_record_once():
    owner = [0, 1, 1, 0, 1, 0, 0, 1, 1, 1, 0, 0, 1, 0, 1, 0]
    port = _free_port()
    with mp.Manager() as m:
        out = m.dict()
        mp.spawn(_rank, args=(2, port, owner, out), nprocs=2, join=True)
        res = dict(out)
    expect = sum(float(FakeContext.record(q).sum()) for q in range(len(owner)))
    for rank in (0, 1):
        d, ll, n_imported, log, cleared = res[rank]
        assert d == expect and ll == -0.5 * expect          # every rank gets rank 0's result
        assert log == [("subtrees", owner.count(rank))]
        assert cleared                                       # the context is returned to whole evaluations
    assert res[0][2] == owner.count(1) and res[1][2] == 0    # only rank 0 imports
