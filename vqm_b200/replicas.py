"""Scoring one list of pairs on several GPUs as independent replicas.

Pairs are independent, so the multi-GPU form of the scorer has no data-path
collective: every rank (one process per GPU, torch.distributed for the
plumbing) takes a shard of the list, scores it on its own GPU with its own
batch scorer, and the ranks exchange only the results (108 norms and a score
per pair) to give every rank the whole list in input order. Shards balance
pixels, longest pair first, since a pair's cost grows with its pixel count.
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
