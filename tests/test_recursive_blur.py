"""The opt-in recursive Gaussian blur mode, on the CPU.

The mode has no counterpart in VQM: it is the third-order recursive
Gaussian (sigma 1.5) of Cloudinary's ssimulacra2, which VQM replaced with a
13-tap sampled Gaussian on purpose (docs/divergence.md:22). Neither
Cloudinary's ssimulacra2 nor libjxl is present here, so the filter is pinned
by its defining properties and by its own FP64 evaluation, never by VQM:

- the oracle derives the coefficients from closed forms, the library from
  numeric sums; their float taps must be equal bit for bit;
- unit gain, variance sigma^2 = 2.25, support |m| < N = 5, symmetry, and the
  coefficients nearest the Gaussian's cosine-series coefficients;
- the FP64 recursion equals the FP64 convolution with the taps (so the
  kernels' direct evaluation is that recursive filter) on random planes of
  ragged sizes and on an impulse;
- the FP32 restatement of the whole metric in this mode (the CUDA kernels'
  arithmetic) stays within the stated bound of the FP64 recursion: score
  within 1e-2, every feature within 1e-2 relative plus 5e-5 absolute.
  Measured on these pairs and the GPU tests' pairs: at most 8.8e-3 in the
  score (a 1922x1082 10-bit 4:2:0 pair) and 1.3e-5 absolute in a feature;
  features below 1e-4 can differ by tens of percent, in either blur mode,
  from the FP32 cancellation in sigma^2 = blur(x^2) - mu^2.
"""

import numpy as np
import pytest

from oracle import binding as ob
from tests import helpers
from tests import synthetic
from vqm_b200 import ss2

SCORE_TOL64 = 1e-2
FEATURE_RTOL64 = 1e-2
FEATURE_ATOL64 = 5e-5


def test_parameters_and_defining_properties():
    radius, freqs, beta, taps = ob.recursive_gaussian()
    assert radius == 5  # round(3.2795 * 1.5 + 0.2546)
    assert np.allclose(freqs, [(2 * k + 1) * np.pi / 10 for k in range(3)], rtol=0, atol=1e-15)
    m = np.arange(-6, 7)
    assert np.array_equal(taps, taps[::-1])
    assert np.all(taps[np.abs(m) >= radius] == 0.0)
    assert np.all(taps[np.abs(m) < radius] > 0.0)
    assert abs(taps.sum() - 1.0) < 1e-14
    assert abs((m * m * taps).sum() - 2.25) < 1e-12
    # The impulse response is the cosine sum with these coefficients.
    cos = np.cos(np.outer(freqs, m[np.abs(m) < radius]))
    assert np.allclose(beta @ cos, taps[np.abs(m) < radius], rtol=0, atol=1e-15)
    # Nearest point to the Gaussian's cosine-series coefficients on the two
    # constraints: beta - rho lies in the span of the constraint rows.
    w = np.arange(-radius, radius + 1)
    rows = np.cos(np.outer(freqs, w))
    p = np.vstack([rows.sum(1), (rows * w * w).sum(1)])
    rho = np.exp(-0.5 * 2.25 * freqs ** 2) / radius
    coef, *_ = np.linalg.lstsq(p.T, beta - rho, rcond=None)
    assert np.allclose(p.T @ coef, beta - rho, rtol=0, atol=1e-14)


def test_library_taps_equal_oracle_taps():
    _, _, _, taps = ob.recursive_gaussian()
    assert np.array_equal(ss2.blur_taps(ss2.Ssimulacra2Blur.RECURSIVE), taps.astype(np.float32))
    assert np.array_equal(ss2.blur_taps(ss2.Ssimulacra2Blur.SAMPLED), ob.gaussian())
    with pytest.raises(ss2.InvalidArgument):
        ss2.blur_taps(2)


def direct(plane, taps):
    """Zero-padded separable convolution in double, rows then columns."""
    h, w = plane.shape
    pad = np.pad(plane, 6)
    rows = sum(taps[k] * pad[6:6 + h, k:k + w] for k in range(13))
    rows = np.pad(rows, ((6, 6), (0, 0)))
    return sum(taps[k] * rows[k:k + h, :] for k in range(13))


@pytest.mark.parametrize("shape", [(8, 8), (9, 31), (37, 53), (128, 97), (3, 200)])
def test_recursion_equals_convolution(shape):
    _, _, _, taps = ob.recursive_gaussian()
    rng = np.random.default_rng(shape[0] * 1000 + shape[1])
    x = rng.random(shape) * 2 - 0.5
    rec = ob.blur_plane(x, blur=1, precision=64)
    assert np.max(np.abs(rec - direct(x, taps))) < 1e-13
    # The FP32 evaluation the kernels use: float taps, 13 ascending FMAs.
    f32 = ob.blur_plane(x, blur=1, precision=32)
    assert np.max(np.abs(f32 - rec)) < 2e-6


def test_impulse_response():
    _, _, _, taps = ob.recursive_gaussian()
    x = np.zeros((21, 21))
    x[10, 10] = 1.0
    rec = ob.blur_plane(x, blur=1, precision=64)
    assert np.allclose(rec[4:17, 4:17], np.outer(taps, taps), rtol=0, atol=1e-15)
    # An impulse at the border: zero padding, nothing wraps or reflects.
    x = np.zeros((16, 16))
    x[0, 0] = 1.0
    rec = ob.blur_plane(x, blur=1, precision=64)
    assert np.allclose(rec[:7, :7], np.outer(taps[6:], taps[6:]), rtol=0, atol=1e-15)
    assert np.all(np.abs(rec[7:, :]) < 1e-15) and np.all(np.abs(rec[:, 7:]) < 1e-15)


def pairs():
    out = [helpers.plain_256_pair()]
    for w, h, seed in ((333, 187, 1), (640, 360, 2)):
        out.append(synthetic.rgb_pair(w, h, seed)[:2])
    out.append(synthetic.yuv_pair(480, 270, 4)[:2])
    out.append(synthetic.yuv_pair(1280, 720, 73)[:2])
    return out


def test_fp32_metric_within_bound_of_fp64_recursion():
    for o, d in pairs():
        n32, s32 = helpers.oracle_compute(o, d, blur=1)
        n64, s64 = helpers.oracle_compute(o, d, blur=1, precision=64)
        assert abs(s32 - s64) <= SCORE_TOL64, (o.width, s32, s64)
        bad = helpers.feature_mismatch(n32, n64, rtol=FEATURE_RTOL64, atol=FEATURE_ATOL64)
        assert not bad, (o.width, bad[:4])


def test_mode_moves_scores_and_keeps_identity():
    o, d = helpers.plain_256_pair()
    _, sampled = helpers.oracle_compute(o, d, precision=64)
    _, recursive = helpers.oracle_compute(o, d, precision=64, blur=1)
    assert abs(sampled - recursive) > 1e-2  # a different metric, not VQM's scores
    for precision in (32, 64):
        norms, score = helpers.oracle_compute(o, o, precision=precision, blur=1)
        assert score == 100.0 and np.all(norms == 0.0)


def test_unknown_mode_is_rejected():
    o, d = helpers.plain_256_pair()
    with pytest.raises(ob.OracleError):
        helpers.oracle_compute(o, d, blur=2)
    # The library rejects it before touching a device.
    with pytest.raises(ss2.InvalidArgument):
        ss2.Ssimulacra2Pipeline(64, 64, blur=2)
    with pytest.raises(ss2.InvalidArgument):
        ss2.Ssimulacra2Batch(max_pairs=1, blur=2)
