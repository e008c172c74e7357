"""Half planes (ssimulacra2.h:41-46): binary16 pyramid planes with FP32
arithmetic. Parity is against the oracle's half-plane restatement (planes and
level averages rounded to binary16, ssimu2_common.glsl:45-91) at the same bar
as full planes; the distance to full planes is VQM's own bound for the mode
(tests/metrics/ssimulacra2/pipeline_test.cc:785-834: score 0.1, norms 2e-4)."""

import numpy as np
import pytest

from tests import helpers
from tests import synthetic
from vqm_b200 import ss2

pytestmark = pytest.mark.gpu


def _check_half(result, o, d, label):
    norms, score = helpers.oracle_compute(o, d, precision=16)
    bad = helpers.feature_mismatch(result.norms, norms)
    assert not bad, (label, bad[:8])
    assert np.all(result.norms[helpers.pruned_mask(result.norms.shape[0])] == 0.0)
    assert abs(result.score() - score) <= helpers.SCORE_TOL, (label, result.score(), score)


def test_vqm_half_plane_bounds_on_the_gradient_pairs():
    orig = helpers.gradient(0)
    with ss2.Ssimulacra2Pipeline(32, 32) as exact, \
            ss2.Ssimulacra2Pipeline(32, 32, half_planes=True) as half:
        for v in (1, 2):
            dist = helpers.gradient(v)
            e, h = exact.compute(orig, dist), half.compute(orig, dist)
            assert h.norms.shape == e.norms.shape
            assert abs(h.score() - e.score()) <= 0.1
            assert np.max(np.abs(h.norms - e.norms)) <= 2e-4
            _check_half(h, orig, dist, f"gradient {v}")
        assert half.compute(orig, orig).score() == 100.0


@pytest.mark.parametrize("make", [
    lambda: helpers.plain_256_pair(),
    lambda: synthetic.rgb_pair(333, 187, 61)[:2],
    lambda: synthetic.rgb_pair(101, 57, 62)[:2],
    lambda: synthetic.yuv_pair(322, 182, 63)[:2],
])
def test_half_plane_parity(make):
    o, d = make()
    with ss2.Ssimulacra2Pipeline(o.width, o.height, half_planes=True) as p:
        r = p.compute(o, d)
    _check_half(r, o, d, f"{o.width}x{o.height}")


def test_half_plane_batch_matches_pipeline_for_every_variant():
    pairs = [synthetic.rgb_pair(333, 187, 64)[:2], synthetic.yuv_pair(640, 360, 65)[:2],
             synthetic.rgb_pair(97, 61, 66)[:2]]
    ref = []
    for o, d in pairs:
        with ss2.Ssimulacra2Pipeline(o.width, o.height, half_planes=True) as p:
            ref.append(p.compute(o, d).norms)
    for v in range(len(ss2.blur_variants())):
        b = ss2.Ssimulacra2Batch(variant=v, half_planes=True)
        got = b.compute_many(pairs)
        b.close()
        for g, r, (o, d) in zip(got, ref, pairs):
            bad = helpers.feature_mismatch(g.norms, r)
            assert not bad, (v, bad[:4])
