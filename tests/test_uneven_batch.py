"""The uneven batch at its own scale: the first 16 10-bit 4:2:0 pairs of the
benchmark's uneven draw (sizes up to 3840x2160) and its 8 odd-sized 8-bit RGB
pairs, scored in one Ssimulacra2Batch with the autotuned blur variant.

Every pair must match the FP32 oracle (each of the 108 features within 1e-4
relative, pruned features exactly 0, score within 1e-2), and what the
one-pair pipeline returns for it alone within 1e-6 relative per feature (the
two may group the compensated partial sums differently: a batch this size
runs 8-tile blur strips, one pair alone one tile per CTA). The batch semantics
follow Ssimulacra2Pool::ComputeMany (src/pool.cc:44-72): one result per pair,
in input order.
"""

import os

import numpy as np
import pytest

import workloads
from oracle import binding as ob
from tests import helpers, synthetic
from vqm_b200 import autotune, ss2

pytestmark = pytest.mark.gpu

YUV_PAIRS = 16


def _jobs():
    jobs = workloads.uneven_jobs()
    yuv = [j for j in jobs if j[0] == "yuv"][:YUV_PAIRS]
    rgb = [j for j in jobs if j[0] == "rgb"]
    return yuv + rgb


@pytest.fixture(scope="module")
def uneven_pairs():
    from concurrent.futures import ProcessPoolExecutor
    import multiprocessing as mp
    jobs = _jobs()
    with ProcessPoolExecutor(min(len(jobs), os.cpu_count() or 1),
                             mp_context=mp.get_context("spawn")) as ex:
        planar = list(ex.map(workloads.make_pair, jobs))
    return [(synthetic.image(o), synthetic.image(d)) for o, d in planar]


def _device(pairs):
    import torch
    keep, dev = [], []
    for o, d in pairs:
        to, td = torch.from_numpy(o.data).cuda(), torch.from_numpy(d.data).cuda()
        keep += [to, td]
        dev.append((ss2.DeviceImage.packed(o.width, o.height, o.format, to.data_ptr(), to),
                    ss2.DeviceImage.packed(d.width, d.height, d.format, td.data_ptr(), td)))
    return dev, keep


def test_draw_covers_the_configuration(uneven_pairs):
    sizes = [(o.width, o.height) for o, _ in uneven_pairs]
    kinds = [o.format.family for o, _ in uneven_pairs]
    assert len(uneven_pairs) == 24
    assert any(w % 2 and h % 2 for w, h in sizes[YUV_PAIRS:])  # odd RGB geometry
    assert all(w % 2 == 0 and h % 2 == 0 for w, h in sizes[:YUV_PAIRS])
    assert kinds[:YUV_PAIRS] == [ss2.ColorFamily.Yuv] * YUV_PAIRS
    assert max(w * h for w, h in sizes) > 4_000_000


def test_uneven_batch_matches_oracle_and_pipeline(uneven_pairs):
    dev, _keep = _device(uneven_pairs)
    tuned = autotune.tune(dev, use_cache=False, repeats=1)
    with_batch = ss2.Ssimulacra2Batch(max_pairs=len(dev), variant=tuned.variant)
    results = with_batch.compute_many(dev)
    again = with_batch.compute_many(dev)
    with_batch.close()
    assert len(results) == len(uneven_pairs)

    op = [(helpers.to_oracle(o), helpers.to_oracle(d)) for o, d in uneven_pairs]
    norms, scales, scores = ob.compute_many(op, precision=32)
    _, _, scores64 = ob.compute_many(op, precision=64)
    worst_rel, worst_score, worst64 = 0.0, 0.0, 0.0
    for i, (r, (o, _)) in enumerate(zip(results, uneven_pairs)):
        label = f"pair {i} {o.width}x{o.height} family {o.format.family}"
        want = norms[i, : 18 * int(scales[i])].reshape(int(scales[i]), 18)
        bad = helpers.feature_mismatch(r.norms, want)
        assert not bad, (label, bad[:6])
        mask = helpers.pruned_mask(r.norms.shape[0])
        assert np.all(r.norms[mask] == 0.0), label
        assert abs(r.score() - scores[i]) <= helpers.SCORE_TOL, (label, r.score(), scores[i])
        assert np.array_equal(r.norms, again[i].norms), label  # repeatable
        nz = want != 0
        worst_rel = max(worst_rel, float(np.max(np.abs(r.norms[nz] - want[nz]) /
                                                np.abs(want[nz]))))
        worst_score = max(worst_score, abs(r.score() - scores[i]))
        worst64 = max(worst64, abs(r.score() - scores64[i]))
    print(f"uneven batch of {len(results)} (blur variant {tuned.variant}): max rel feature "
          f"error {worst_rel:.2e}, max score error {worst_score:.2e} (FP64 oracle {worst64:.2e})")

    # The same pairs one per call through the fixed-size pipeline.
    for i, ((o, d), r) in enumerate(zip(dev, results)):
        with ss2.Ssimulacra2Pipeline(o.width, o.height) as pipe:
            alone = pipe.compute(o, d)
        assert not helpers.feature_mismatch(alone.norms, r.norms, rtol=1e-6, atol=1e-12), \
            f"pair {i} alone != in the batch"
