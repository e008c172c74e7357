"""Serving loop (vqm_cu_ss2_server_*): continuous batching of single-pair
requests, admission by a device-memory budget, and every request's result
bit-identical whether it is scored alone or in a mix of other requests."""

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


@pytest.mark.gpu
def test_results_same_alone_and_in_the_mix():
    import torch
    pairs = _mix()
    # One pair as caller-owned device buffers too.
    o, d = helpers.plain_256_pair()
    to = torch.from_numpy(o.data).cuda()
    td = torch.from_numpy(d.data).cuda()
    pairs.append((ss2.DeviceImage.packed(256, 256, o.format, to.data_ptr(), to),
                  ss2.DeviceImage.packed(256, 256, d.format, td.data_ptr(), td)))
    batch = ss2.Ssimulacra2Batch()
    alone = [batch.compute_many([p])[0] for p in pairs]
    batch.close()

    with ss2.Ssimulacra2Server(workers=2, max_batch_pairs=8) as server:
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
def test_budget_bounds_each_batch():
    pairs = [synthetic.rgb_pair(1920, 1080, 200 + i)[:2] for i in range(5)]
    # A 1080p pair from host memory needs ~41 MB on the device: 60 MB per
    # worker admits one pair per batch, never two.
    budget = 2 * 60_000_000
    with ss2.Ssimulacra2Server(memory_budget=budget, workers=2, max_batch_pairs=8) as server:
        tickets = [server.submit(o, d) for o, d in pairs]
        results = [server.wait(t)[0] for t in tickets]
        stats = server.stats()
    assert stats.largest_batch == 1 and stats.batches == len(pairs)
    assert 0 < stats.peak_bytes <= budget
    batch = ss2.Ssimulacra2Batch()
    for r, p in zip(results, pairs):
        assert np.array_equal(r.norms, batch.compute_many([p])[0].norms)
    batch.close()


@pytest.mark.gpu
def test_request_larger_than_a_worker_is_rejected():
    o, d = synthetic.rgb_pair(1920, 1080, 300)[:2]
    with ss2.Ssimulacra2Server(memory_budget=2 * 30_000_000, workers=2) as server:
        with pytest.raises(ss2.InvalidArgument, match="worker's budget"):
            server.submit(o, d)
        small_o, small_d = synthetic.rgb_pair(320, 180, 301)[:2]
        r, _ = server.wait(server.submit(small_o, small_d))
        assert r.norms.shape == (6, 18)
        with pytest.raises(ss2.InvalidArgument, match="ticket"):
            server.wait(12345)
