"""Serving loop (vqm_cu_ss2_server_*): continuous batching of single-pair
requests, admission by a device-memory budget, and every request's result
the same whether it is scored alone or in a mix of other requests: bit for
bit with a fixed blur kernel, and within 1e-6 relative per feature (well
inside the 1e-4 parity bound) when each batch picks its strip length from
its size, which regroups the compensated partial sums."""

import threading

import numpy as np
import pytest

from tests import helpers
from tests import synthetic
from vqm_b200 import ss2


def test_server_needs_a_device_or_reports_why():
    import torch
    if torch.cuda.is_available():
        pytest.skip("covered by the GPU tests")
    with pytest.raises(ss2.CudaError):
        ss2.Ssimulacra2Server()


def _mix():
    """RGB 8-bit and 10-bit 4:2:0 pairs of several sizes, odd ones in RGB."""
    sizes = [(640, 360), (1280, 720), (333, 187), (1920, 1080), (322, 182), (1000, 563)]
    pairs = []
    for i, (w, h) in enumerate(sizes * 3):
        if i % 2:
            pairs.append(synthetic.yuv_pair(w & ~1, h & ~1, 100 + i)[:2])
        else:
            pairs.append(synthetic.rgb_pair(w, h, 100 + i)[:2])
    return pairs


# Blur kernels: None lets every batch pick its 32x32 strip length from its
# tile count; 9 is the 8-tile strip kernel, fixed.
@pytest.mark.gpu
@pytest.mark.parametrize("variant", [None, 9])
def test_results_same_alone_and_in_the_mix(variant):
    import torch
    pairs = _mix()
    # One pair as caller-owned device buffers too.
    o, d = helpers.plain_256_pair()
    to = torch.from_numpy(o.data).cuda()
    td = torch.from_numpy(d.data).cuda()
    pairs.append((ss2.DeviceImage.packed(256, 256, o.format, to.data_ptr(), to),
                  ss2.DeviceImage.packed(256, 256, d.format, td.data_ptr(), td)))
    if variant is not None:
        assert ss2.blur_variants()[variant][3] == 8  # an 8-tile strip kernel
    batch = ss2.Ssimulacra2Batch(variant=variant)
    alone = [batch.compute_many([p])[0] for p in pairs]
    batch.close()

    server_variant = 0 if variant is None else variant + 1
    with ss2.Ssimulacra2Server(workers=2, max_batch_pairs=8, variant=server_variant) as server:
        tickets = [None] * len(pairs)

        def produce(indices):
            for i in indices:
                tickets[i] = server.submit(*pairs[i])

        threads = [threading.Thread(target=produce, args=(range(k, len(pairs), 2),))
                   for k in range(2)]
        for t in threads:
            t.start()
        for t in threads:
            t.join()
        results = [server.wait(t) for t in tickets]
        stats = server.stats()

    for i, ((r, latency), a) in enumerate(zip(results, alone)):
        if variant is None:
            assert not helpers.feature_mismatch(r.norms, a.norms, rtol=1e-6, atol=1e-12), i
        else:
            assert np.array_equal(r.norms, a.norms), i
            assert r.device_score == a.device_score, i
        assert latency > 0.0
    assert stats.submitted == stats.completed == len(pairs)
    assert stats.failed == 0 and stats.queued == 0 and stats.bytes_in_flight == 0
    # Requests that queued while both workers were busy shared launches.
    assert stats.batches < len(pairs) and stats.largest_batch > 1
    # And they match the CPU oracle.
    for (r, _), (o, d) in list(zip(results, pairs))[:4]:
        norms, score = helpers.oracle_compute(o, d)
        assert not helpers.feature_mismatch(r.norms, norms)
        assert abs(r.score() - score) <= helpers.SCORE_TOL


@pytest.mark.gpu
def test_budget_caps_the_memory_the_workers_hold():
    """A mixed stream under a tight budget: the device memory all workers
    hold together (their own count of what they allocated, growth included)
    never exceeds the budget, idle workers give memory back when a request
    needs it, and every result equals the pair scored alone."""
    import torch
    sizes = [(3840, 2160), (640, 360), (1920, 1080), (2560, 1440), (1280, 720), (3840, 2160),
             (333, 187), (1920, 1080)]
    pairs = [(synthetic.yuv_pair if i % 2 else synthetic.rgb_pair)(w, h, 400 + i)[:2]
             for i, (w, h) in enumerate(sizes * 2)]
    batch = ss2.Ssimulacra2Batch()
    alone = [batch.compute_many([p])[0] for p in pairs]
    need_4k = batch.device_bytes_after([pairs[0]])
    batch.close()
    torch.cuda.synchronize()
    free_before, _ = torch.cuda.mem_get_info()
    # Room for one 4K pair and a little more, over three workers: the old
    # per-worker split (a third each) could not have admitted a 4K pair.
    budget = int(need_4k * 1.3)
    with ss2.Ssimulacra2Server(memory_budget=budget, workers=3, max_batch_pairs=8) as server:
        tickets = [server.submit(o, d) for o, d in pairs]
        results = [server.wait(t)[0] for t in tickets]
        stats = server.stats()
        free_after, _ = torch.cuda.mem_get_info()
    assert stats.budget_bytes == budget
    assert 0 < stats.peak_device_bytes <= budget
    assert stats.device_bytes <= budget
    assert stats.trims > 0  # idle workers' memory was freed to admit the 4K pairs
    assert free_before - free_after <= budget + (64 << 20)  # the driver agrees
    assert stats.completed == len(pairs) and stats.failed == 0
    for i, (r, a) in enumerate(zip(results, alone)):
        assert not helpers.feature_mismatch(r.norms, a.norms, rtol=1e-6, atol=1e-12), i


@pytest.mark.gpu
def test_budget_is_clamped_to_free_device_memory():
    import torch
    free, _ = torch.cuda.mem_get_info()
    with ss2.Ssimulacra2Server(memory_budget=1 << 50, workers=1) as server:
        assert server.stats().budget_bytes <= free


@pytest.mark.gpu
def test_request_up_to_the_whole_budget_is_admitted():
    o, d = synthetic.rgb_pair(1920, 1080, 300)[:2]
    # A 1080p pair from host memory needs ~41 MB: above half of a 60 MB
    # budget (a worker's share), below the whole of it.
    with ss2.Ssimulacra2Server(memory_budget=60_000_000, workers=2) as server:
        r, _ = server.wait(server.submit(o, d))
        assert r.norms.shape == (6, 18)
        assert server.stats().peak_device_bytes <= 60_000_000
    with ss2.Ssimulacra2Server(memory_budget=30_000_000, workers=2) as server:
        with pytest.raises(ss2.InvalidArgument, match="the budget is"):
            server.submit(o, d)
        small_o, small_d = synthetic.rgb_pair(320, 180, 301)[:2]
        r, _ = server.wait(server.submit(small_o, small_d))
        assert r.norms.shape == (6, 18)
        with pytest.raises(ss2.InvalidArgument, match="ticket"):
            server.wait(12345)


@pytest.mark.gpu
def test_batch_counts_its_own_memory():
    """device_bytes_after predicts exactly what a submit leaves the batch
    holding (growth included); trim frees it and scoring goes on."""
    b = ss2.Ssimulacra2Batch()
    small = [synthetic.rgb_pair(640, 360, 11)[:2]]
    large = [synthetic.yuv_pair(1920, 1080, 12)[:2]] * 2
    first = None
    try:
        assert b.device_bytes() == 0
        for ps in (small, large, small, large + small):
            want = b.device_bytes_after(ps)
            got = b.compute_many(ps)
            first = first or got[0]
            assert b.device_bytes() == want
        held = b.device_bytes()
        assert b.device_bytes_after(small) == held  # nothing grows for a smaller batch
        b.trim()
        assert b.device_bytes() == 0
        assert np.array_equal(b.compute_many(small)[0].norms, first.norms)
    finally:
        b.close()
