"""The opt-in recursive Gaussian blur mode on the GPU.

Graded against its own references, never against VQM (whose scores the
mode does not reproduce, docs/divergence.md:22):

- the FP32 oracle in the same mode (the kernels' arithmetic): every feature
  within 1e-4 relative, pruned features exactly 0, score within 1e-2;
- the FP64 recursion itself: score within 1e-2 and every feature within
  1e-2 relative plus 5e-5 absolute, the bound the CPU tests state;
- identity exactly 100; batch, pool, server and half planes carry the mode.
"""

import numpy as np
import pytest

from tests import helpers
from tests import synthetic
from tests.test_recursive_blur import FEATURE_ATOL64, FEATURE_RTOL64, SCORE_TOL64
from vqm_b200 import ss2

pytestmark = pytest.mark.gpu

REC = ss2.Ssimulacra2Blur.RECURSIVE


def check_recursive(result, o, d, label, precision=32, rtol=helpers.FEATURE_RTOL):
    norms, score = helpers.oracle_compute(o, d, precision=precision, blur=REC)
    bad = helpers.feature_mismatch(result.norms, norms, rtol=rtol)
    assert not bad, (label, bad[:8])
    assert np.all(result.norms[helpers.pruned_mask(result.norms.shape[0])] == 0.0), label
    s = result.score()
    assert abs(s - score) <= helpers.SCORE_TOL, (label, s, score)
    if precision != 32:
        return s
    n64, s64 = helpers.oracle_compute(o, d, precision=64, blur=REC)
    bad = helpers.feature_mismatch(result.norms, n64, rtol=FEATURE_RTOL64, atol=FEATURE_ATOL64)
    assert not bad, (label, "fp64", bad[:8])
    assert abs(s - s64) <= SCORE_TOL64, (label, s, s64)
    m = n64 != 0
    rel = np.max(np.abs(result.norms[m] - n64[m]) / np.abs(n64[m]))
    print(f"{label}: cuda {s:.8f} oracle32 {score:.8f} fp64 recursion {s64:.8f} "
          f"|d64| {abs(s - s64):.2e} max feature rel {rel:.2e}")
    return s


@pytest.mark.parametrize("make", [
    lambda: helpers.plain_256_pair(),
    lambda: synthetic.rgb_pair(333, 187, 71)[:2],
    lambda: synthetic.rgb_pair(1920, 1080, 72)[:2],
    lambda: synthetic.yuv_pair(1280, 720, 73)[:2],
    lambda: synthetic.yuv_pair(3840, 2160, 74)[:2],
])
def test_pipeline_recursive_parity(make):
    o, d = make()
    with ss2.Ssimulacra2Pipeline(o.width, o.height, blur=REC) as p:
        r = p.compute(o, d)
        again = p.compute(o, d)
        assert np.array_equal(r.norms, again.norms)
        assert p.compute(o, o).score() == 100.0
    check_recursive(r, o, d, f"{o.width}x{o.height}")


def test_modes_differ_on_the_same_pair():
    o, d = helpers.plain_256_pair()
    with ss2.Ssimulacra2Pipeline(256, 256) as sampled, \
            ss2.Ssimulacra2Pipeline(256, 256, blur=REC) as recursive:
        a, b = sampled.compute(o, d), recursive.compute(o, d)
    _, s_sampled = helpers.oracle_compute(o, d)
    assert abs(a.score() - s_sampled) <= helpers.SCORE_TOL
    assert abs(a.score() - b.score()) > 1e-2


def uneven_pairs():
    jobs = [(1, 2, 640, 360, 81), (0, 1, 333, 187, 82), (1, 2, 1921, 1081, 83),
            (0, 1, 97, 61, 84), (1, 2, 1280, 719, 85), (0, 1, 1920, 1080, 86)]
    out = []
    for yuv, _, w, h, seed in jobs:
        out.append((synthetic.yuv_pair if yuv else synthetic.rgb_pair)(w, h, seed)[:2])
    return out


def test_batch_pool_and_server_carry_the_mode():
    pairs = uneven_pairs()
    batch = ss2.Ssimulacra2Batch(blur=REC)
    got = batch.compute_many(pairs)
    batch.close()
    for r, (o, d) in zip(got, pairs):
        check_recursive(r, o, d, f"batch {o.width}x{o.height}")
    # The pool's chunks are the same submissions: bit for bit.
    pool = ss2.Ssimulacra2Pool(workers=2, chunk=len(pairs), blur=REC)
    pooled = pool.compute_many(pairs)
    pool.close()
    for a, b in zip(pooled, got):
        assert np.array_equal(a.norms, b.norms)
    with ss2.Ssimulacra2Server(workers=2, max_batch_pairs=4, blur=REC) as server:
        tickets = [server.submit(o, d) for o, d in pairs]
        served = [server.wait(t)[0] for t in tickets]
    for s, b in zip(served, got):
        assert not helpers.feature_mismatch(s.norms, b.norms, rtol=1e-6, atol=1e-12)


def test_half_planes_in_recursive_mode():
    o, d = synthetic.rgb_pair(333, 187, 91)[:2]
    with ss2.Ssimulacra2Pipeline(o.width, o.height, half_planes=True, blur=REC) as p:
        r = p.compute(o, d)
        assert p.compute(o, o).score() == 100.0
    check_recursive(r, o, d, "half planes", precision=16)
