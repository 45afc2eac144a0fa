"""Multi-GPU sharding of one DB: each rank (one process per GPU) holds a
contiguous, residue-balanced slice of the records, searches it, and the
ranks exchange only their k best hits.

This replaces WorkerPool's split of one DB across its workers
(src/WorkerPool.cpp:10-82: every worker pulls chunks from the shared
DataPool, then getResult merges the workers' ResultLists, :99-105).  Here
the split is static (records do not move after load) and the merge is one
all-gather of k (score, index) pairs per query, ordered by score
descending, then record index ascending.
"""
from __future__ import annotations

import numpy as np


def shard_bounds(offsets: np.ndarray, world: int) -> list:
    """Contiguous record ranges [(begin, end), ...], one per rank, with about
    the same number of residues each."""
    off = np.asarray(offsets, dtype=np.int64)
    n = len(off) - 1
    total = int(off[-1] - off[0])
    cuts = [0]
    for r in range(1, world):
        target = off[0] + total * r // world
        cuts.append(int(min(max(np.searchsorted(off, target, side="left"), cuts[-1]), n)))
    cuts.append(n)
    return [(cuts[r], cuts[r + 1]) for r in range(world)]


def local_records(residues: np.ndarray, offsets: np.ndarray, begin: int, end: int):
    """A shard's records as (residues, offsets rebased to 0)."""
    off = np.asarray(offsets, dtype=np.uint64)
    lo, hi = int(off[begin]), int(off[end])
    return np.asarray(residues)[lo:hi], (off[begin:end + 1] - off[begin]).astype(np.uint64)


def merge_hits(lists, k: int) -> list:
    """Merged top-k of per-shard hit lists [(score, global index), ...]
    under the search's order: score descending, then index ascending."""
    allh = [h for lst in lists for h in lst if h[0] > 0]
    allh.sort(key=lambda h: (-h[0], h[1]))
    return allh[:k]


def gather_topk(local_hits, base: int, k: int, group=None) -> list:
    """All ranks' hits (local record indices + their shard's first record
    `base`) merged into the global top-k; every rank gets the same list."""
    import torch.distributed as dist
    mine = [(int(s), int(i) + base) for (s, i) in local_hits]
    world = dist.get_world_size(group)
    got = [None] * world
    dist.all_gather_object(got, mine, group=group)
    return merge_hits(got, k)


class ShardedSearch:
    """One rank's part of a sharded search: loads this rank's slice of the DB
    into a context on its GPU; search() returns the global top-k."""

    def __init__(self, ctx, residues, offsets, rank: int, world: int, group=None):
        self.ctx = ctx
        self.group = group
        self.begin, self.end = shard_bounds(offsets, world)[rank]
        res, off = local_records(residues, offsets, self.begin, self.end)
        ctx.load_db(res, off)

    def search(self, query) -> list:
        hits, _ = self.ctx.search(query)
        return gather_topk(hits, self.begin, self.ctx.params.top_k, self.group)
