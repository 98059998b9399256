"""Multi-GPU sharding of a search: independent query-reference pairs.

The reference spreads query blocks over devices and streams every reference
chunk to every device (src/libmycu/cuproc/JobDispatcher.cpp:1019-1048,
1111-1123); no data moves between devices.  Here one process per GPU owns a
share of the REFERENCES, balanced by the estimated cost sum(Lq * Lr)
(longest-processing-time-first), aligns every query with its share, and the
per-pair result records are gathered to rank 0 in the original reference
order.  The only collective is that final gather of results (and the
barriers around timing); the search itself has no data-path exchange.
"""
from __future__ import annotations

import heapq
from typing import Callable, List, Sequence, Tuple

import numpy as np

from .synth import SoA


def lpt_shards(rlens: Sequence[int], qlens: Sequence[int], nranks: int) -> List[np.ndarray]:
    """Split reference indices into nranks shards of near-equal cost.

    Cost of a reference = its length x the total query length (the DP and
    refinement work of its pairs scales with Lq * Lr).  Each shard is
    returned sorted by reference index.
    """
    rl = np.asarray(rlens, dtype=np.int64)
    qsum = int(np.sum(qlens)) if len(qlens) else 1
    cost = rl * max(qsum, 1)
    order = np.argsort(-cost, kind="stable")
    heap = [(0, r) for r in range(nranks)]
    heapq.heapify(heap)
    parts: List[List[int]] = [[] for _ in range(nranks)]
    for i in order:
        c, r = heapq.heappop(heap)
        parts[r].append(int(i))
        heapq.heappush(heap, (c + int(cost[i]), r))
    return [np.array(sorted(p), dtype=np.int64) for p in parts]


def subset(s: SoA, idx: np.ndarray) -> SoA:
    """SoA block of the structures idx (in that order)."""
    lens = s.lens[idx].astype(np.int32)
    offs = np.zeros_like(lens)
    if len(lens) > 1:
        offs[1:] = np.cumsum(lens[:-1])
    sel = np.concatenate([np.arange(s.offs[i], s.offs[i] + s.lens[i]) for i in idx]) if len(idx) else np.zeros(0, np.int64)
    return SoA(lens, offs, s.x[sel].copy(), s.y[sel].copy(), s.z[sel].copy(),
               s.rsd[sel].copy(), s.mol[idx].astype(np.int32))


ProcessFn = Callable[[SoA, SoA], Tuple[np.ndarray, np.ndarray]]


class ShardPlan:
    """This rank's share of a reference block, made once and reused for every
    query block (the reference streams each reference chunk to every device
    for every query block; here a rank keeps its share)."""

    def __init__(self, refs: SoA, qlens: Sequence[int], rank: int, world: int):
        self.rank, self.world, self.nref = rank, world, refs.n
        self.shards = lpt_shards(refs.lens, qlens, world)
        self.mine = self.shards[rank]
        self.refs = refs if world == 1 else subset(refs, self.mine)


def search_sharded(queries: SoA, refs: SoA, process: ProcessFn, rank: int, world: int,
                   group=None, plan: "ShardPlan" = None):
    """Align all queries with this rank's reference shard and gather the
    (nq, nr, 16) result records and (nq, nr, 12) transforms on rank 0.

    `process(queries, refs_shard)` returns (alndata, tfm) for the shard.
    Returns the full arrays on rank 0 and None elsewhere.  Uses
    torch.distributed (gloo or nccl) when world > 1.  `plan` (a ShardPlan
    of `refs`) saves re-splitting the references on every call.
    """
    if plan is None:
        plan = ShardPlan(refs, queries.lens, rank, world)
    mine = plan.mine
    if len(mine):
        aln, tfm = process(queries, plan.refs)
    else:
        aln = np.zeros((queries.n, 0, 16), np.float32)
        tfm = np.zeros((queries.n, 0, 12), np.float32)
    if world == 1:
        return aln, tfm
    import torch.distributed as dist
    payload = (mine, np.ascontiguousarray(aln), np.ascontiguousarray(tfm))
    got = [None] * world if rank == 0 else None
    dist.gather_object(payload, got, dst=0, group=group)
    if rank != 0:
        return None
    full_aln = np.zeros((queries.n, refs.n, 16), np.float32)
    full_tfm = np.zeros((queries.n, refs.n, 12), np.float32)
    for idx, a, t in got:
        if len(idx):
            full_aln[:, idx, :] = a
            full_tfm[:, idx, :] = t
    return full_aln, full_tfm
