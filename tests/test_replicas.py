"""The multi-GPU replica path (vqm_b200/replicas.py) on CPU: sharding by
pixel count, and a world-size-2 gloo run that scores each rank's shard with
a stand-in scorer and gathers every result, in order, on both ranks."""

import os
import socket
from dataclasses import dataclass

import pytest

from vqm_b200 import replicas


def test_shard_balances_pixels_and_covers_every_pair():
    pixels = [1920 * 1080, 640 * 360, 3840 * 2160, 1280 * 720, 640 * 360, 1920 * 1080, 320 * 180]
    shards = replicas.shard(pixels, 2)
    assert sorted(i for s in shards for i in s) == list(range(len(pixels)))
    loads = [sum(pixels[i] for i in s) for s in shards]
    assert max(loads) - min(loads) <= max(pixels)
    # Deterministic: every rank computes the same split.
    assert replicas.shard(pixels, 2) == shards
    assert replicas.shard(pixels, 1) == [list(range(len(pixels)))]
    assert replicas.shard([], 3) == [[], [], []]
    with pytest.raises(ValueError):
        replicas.shard(pixels, 0)


@dataclass
class _Img:
    width: int
    height: int
    tag: int


def _score(sub):
    return [(o.tag, o.width * o.height + d.tag) for o, d in sub]


def _worker(rank, world, port, out_dir):
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        sizes = [(64, 32), (640, 360), (320, 180), (1920, 1080), (8, 8), (100, 50)]
        pairs = [(_Img(w, h, i), _Img(w, h, 100 + i)) for i, (w, h) in enumerate(sizes)]
        calls = []

        def score(sub):
            calls.append(len(sub))
            return _score(sub)

        out = replicas.score_sharded(pairs, score)
        with open(os.path.join(out_dir, f"rank{rank}.txt"), "w") as f:
            f.write(repr((out, calls)))
    finally:
        dist.destroy_process_group()


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def test_score_sharded_two_gloo_ranks(tmp_path):
    import torch.multiprocessing as mp
    world = 2
    mp.spawn(_worker, args=(world, _free_port(), str(tmp_path)), nprocs=world, join=True)
    results = [eval((tmp_path / f"rank{r}.txt").read_text()) for r in range(world)]
    sizes = [(64, 32), (640, 360), (320, 180), (1920, 1080), (8, 8), (100, 50)]
    expected = [(i, w * h + 100 + i) for i, (w, h) in enumerate(sizes)]
    for out, calls in results:
        assert out == expected
        assert sum(calls) <= len(sizes)
    # Each pair was scored exactly once, across the two ranks.
    assert sum(sum(c) for _, c in results) == len(sizes)


def test_contiguous_ranges_cover_the_clip_in_order():
    for count in (0, 1, 5, 240, 241):
        for world in (1, 2, 3, 8):
            ranges = replicas.contiguous(count, world)
            assert [i for r in ranges for i in r] == list(range(count))
            sizes = [len(r) for r in ranges]
            assert max(sizes) - min(sizes) <= 1
    with pytest.raises(ValueError):
        replicas.contiguous(5, 0)


def _gather_worker(rank, world, port, out_dir):
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        count = 7
        mine = replicas.contiguous(count, world)[rank]
        local = [(i, i * i) for i in mine]
        out = replicas.gather_ordered(local, mine.start, count)
        with open(os.path.join(out_dir, f"g{rank}.txt"), "w") as f:
            f.write(repr(out))
    finally:
        dist.destroy_process_group()


def test_gather_ordered_two_gloo_ranks(tmp_path):
    import torch.multiprocessing as mp
    mp.spawn(_gather_worker, args=(2, _free_port(), str(tmp_path)), nprocs=2, join=True)
    for r in range(2):
        assert eval((tmp_path / f"g{r}.txt").read_text()) == [(i, i * i) for i in range(7)]
