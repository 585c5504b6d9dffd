"""Sub-tree sharding of one exact log-likelihood over several GPUs.

One process per GPU, each with a context on the same structure.  The tree is
split at a level s into J^s sub-trees, which are independent below level s: the
prior of each only needs its ancestors' factors (levels < s, cheap, computed on
every rank) and its posterior only its own observations.  This is the
reference's MPI decomposition (src/class_partition.cpp:1188-1280 assigns whole
sub-trees to ranks by a cost model; src/class_approximation.cpp:186-264 sums the
children's contributions on the parent's rank).

  plan(st, world)            split level and an LPT assignment of the
                             sub-trees to ranks by their estimated work
  loglik(ctx, plan, ...)     every rank evaluates its sub-trees, exports one
                             record per owned sub-tree (its output to the parent
                             and its log-likelihood terms), rank 0 gathers and
                             imports the others' records, evaluates the levels
                             above s and the sum, and broadcasts the result

The exchange is one gather of the records (a few hundred KB at r = 64) and one
broadcast of (d, log-likelihood); rank 0's result is bitwise the single-context
evaluation's, since every term is computed by the same kernel code and summed
in the same order.
"""
from __future__ import annotations

from dataclasses import dataclass

import numpy as np


@dataclass
class ShardPlan:
    split: int              # split level s (1 <= s <= M-3)
    owner: np.ndarray       # [J^s] rank of each level-s sub-tree
    cost: np.ndarray        # [J^s] estimated multiply-adds of each sub-tree
    load: np.ndarray        # [world] estimated multiply-adds per rank


def finest_cost(n: np.ndarray, r: int, L: int) -> np.ndarray:
    """Multiply-adds of the finest-level work of regions with n observations
    (the reference algorithm's count: conditioning on L ancestor levels, the
    Cholesky factorization, B^ and its A~ / w~ products)."""
    n = np.asarray(n, dtype=np.float64)
    R = float(r)
    return (R * R * n * L * (L - 1) / 2 + L * R * R * n / 2 + L * R * n * n / 2 + n ** 3 / 6 + n * n / 2 +
            L * n * n * R / 2 + L * R * n + L * R * R * n / 2 + L * (L - 1) / 2 * R * R * n)


def subtree_costs(st, split: int) -> np.ndarray:
    """Estimated multiply-adds of each level-`split` sub-tree: its finest regions'
    work by their observation counts, plus its interior regions (the same number
    in every sub-tree) at the canonical r^3 count of a region of their level."""
    J, M, r = st.J, st.M, st.r
    n = np.diff(np.asarray(st.obs_offset))
    per = J ** (M - 1 - split)           # finest regions per sub-tree (heap order: contiguous)
    fin = finest_cost(n, r, M - 1).reshape(-1, per).sum(axis=1)
    R3 = float(r) ** 3
    interior = sum(J ** (m - split) * R3 * (m * (m - 1) + 2 * m + 1.0 / 3 + 1.0 / 6) for m in range(split, M - 1))
    return fin + interior


def choose_split(J: int, M: int, world: int) -> int:
    """The shallowest level with at least 4 sub-trees per rank (enough to balance
    uneven sub-trees), within [1, M-3]."""
    if M < 4:
        raise ValueError("sub-tree sharding needs M >= 4")
    s = 1
    while s < M - 3 and J ** s < 4 * world:
        s += 1
    return s


def plan(st, world: int, split: int | None = None) -> ShardPlan:
    """LPT assignment (longest sub-tree first to the least-loaded rank, ties to the
    lowest rank) of the level-`split` sub-trees to `world` ranks."""
    if world < 1:
        raise ValueError("world must be >= 1")
    s = choose_split(st.J, st.M, world) if split is None else int(split)
    if not 1 <= s <= st.M - 3:
        raise ValueError("the split level must be in [1, M-3]")
    cost = subtree_costs(st, s)
    owner = np.zeros(cost.shape[0], dtype=np.int64)
    load = np.zeros(world)
    for q in np.argsort(-cost, kind="stable"):
        k = int(np.argmin(load))
        owner[q] = k
        load[k] += cost[q]
    return ShardPlan(split=s, owner=owner, cost=cost, load=load)


def loglik(ctx, sp: ShardPlan, rank: int = 0, world: int = 1, group=None):
    """(d, log-likelihood) of the whole tree, every rank returning rank 0's
    result.  `ctx` is this rank's context (api.Context or anything with the same
    shard_* methods); with world > 1 torch.distributed must be initialised."""
    owned = sp.owner == rank
    ctx.shard_set(sp.split, owned)
    try:
        ctx.shard_subtrees()
        launches = ctx.stats()["kernel_launches"] if hasattr(ctx, "stats") else 0
        records = {int(q): ctx.shard_export(int(q)) for q in np.nonzero(owned)[0]}
        if world > 1:
            import torch.distributed as dist
            gathered = [None] * world if rank == 0 else None
            dist.gather_object(records, gathered, dst=0, group=group)
        else:
            gathered = [records]
        result = [None, None]
        if rank == 0:
            for k in range(1, world):
                for q, rec in sorted(gathered[k].items()):
                    if sp.owner[q] != k:
                        raise RuntimeError(f"rank {k} sent sub-tree {q} that it does not own")
                    ctx.shard_import(q, rec)
            got = set(records) | {q for k in range(1, world) for q in gathered[k]}
            if got != set(range(len(sp.owner))):
                raise RuntimeError("a sub-tree record is missing")
            result = list(ctx.shard_top())
            launches += ctx.stats()["kernel_launches"] if hasattr(ctx, "stats") else 0
        ctx.shard_launches = launches  # kernels this rank launched for the evaluation
        if world > 1:
            import torch.distributed as dist
            dist.broadcast_object_list(result, src=0, group=group)
        return result[0], result[1]
    finally:
        ctx.shard_set(sp.split, None)
