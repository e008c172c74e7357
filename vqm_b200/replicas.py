"""Scoring one list of pairs on several GPUs as independent replicas.

Pairs are independent, so the multi-GPU form of the scorer has no data-path
collective: every rank (one process per GPU, torch.distributed for the
plumbing) takes a shard of the list, scores it on its own GPU with its own
batch scorer, and the ranks exchange only the results (108 norms and a score
per pair) to give every rank the whole list in input order. Shards of a
list of pairs balance pixels, longest pair first, since a pair's cost grows
with its pixel count; the frames of a video take contiguous ranges instead
(one size, and each rank reads and scores its range in order).
"""

from __future__ import annotations

from typing import Callable, Sequence


def shard(pixels: Sequence[int], world: int) -> list[list[int]]:
    """Indices of the pairs each rank scores: pairs by descending pixel count
    (then index), each to the rank with the fewest pixels so far (then the
    lowest rank). Each shard keeps its indices in ascending order."""
    if world < 1:
        raise ValueError("world must be at least 1")
    load = [0] * world
    out: list[list[int]] = [[] for _ in range(world)]
    for i in sorted(range(len(pixels)), key=lambda k: (-pixels[k], k)):
        r = min(range(world), key=lambda q: (load[q], q))
        out[r].append(i)
        load[r] += int(pixels[i])
    return [sorted(s) for s in out]


def contiguous(count: int, world: int) -> list[range]:
    """Rank r's frames [r * count // world, (r + 1) * count // world): in
    order, sizes differing by at most one."""
    if world < 1:
        raise ValueError("world must be at least 1")
    return [range(r * count // world, (r + 1) * count // world) for r in range(world)]


def gather_ordered(local: list, first: int, count: int, group=None) -> list:
    """Every rank's results for its contiguous range (starting at `first`),
    reassembled in order on every rank."""
    import torch.distributed as dist

    world = dist.get_world_size(group)
    gathered: list = [None] * world
    dist.all_gather_object(gathered, (first, list(local)), group=group)
    out: list = [None] * count
    for start, part in gathered:
        out[start:start + len(part)] = part
    return out


def score_sharded(pairs: Sequence, score: Callable[[list], list], group=None) -> list:
    """Scores `pairs` (the same list on every rank) across the ranks of
    `group` and returns every pair's result, in input order, on every rank.

    `score(sub_list)` runs on this rank's GPU and returns one result per
    pair (for example ``Ssimulacra2Batch(...).compute_many``). Results are
    exchanged with ``all_gather_object``, so they must be picklable."""
    import torch.distributed as dist

    world = dist.get_world_size(group)
    rank = dist.get_rank(group)
    pixels = [o.width * o.height for o, _ in pairs]
    shards = shard(pixels, world)
    mine = shards[rank]
    local = score([pairs[i] for i in mine]) if mine else []
    if len(local) != len(mine):
        raise RuntimeError("the scorer returned a different number of results")
    gathered: list = [None] * world
    dist.all_gather_object(gathered, list(zip(mine, local)), group=group)
    out: list = [None] * len(pairs)
    for part in gathered:
        for i, r in part:
            out[i] = r
    return out
