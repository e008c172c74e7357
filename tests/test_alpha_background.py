"""ComputeWorstBackground (include/vqm_alpha.h:12-28) as VQM's alpha tests
state it (tests/core/alpha_test.cc:23-131, the SSIMULACRA 2 half): opaque
pairs are scored once at the default background; a pair with alpha on
either side is scored over 0.1 and 0.9 and the lower score is kept, for
packed images and plane views alike."""

import numpy as np
import pytest

from tests import helpers
from vqm_b200 import ss2

pytestmark = pytest.mark.gpu


def _view(img: ss2.Image) -> ss2.HostImage:
    """Plane views over the packed image's bytes, one row of w bytes per
    row (alpha_test.cc:39-49, 84-96)."""
    n = img.width * img.height
    count = 4 if img.format.alpha != ss2.AlphaType.None_ else 3
    planes = [img.data[p * n:(p + 1) * n].reshape(img.height, img.width) for p in range(count)]
    strides = [img.width] * count + [0] * (4 - count)
    return ss2.HostImage(img.width, img.height, img.format, planes + [None] * (4 - count),
                         tuple(strides))


def test_worst_background_helper():
    """alpha_test.cc:23-72."""
    o = helpers.ramp_image(32, 32, True, ss2.PixelType.Byte)
    data = o.data.copy()
    data[:128] ^= 0x55
    d = ss2.Image(32, 32, o.format, data)
    with ss2.Ssimulacra2Pipeline(32, 32) as p:
        dark = p.compute(o, d, 0.1).score()
        bright = p.compute(o, d, 0.9).score()
        assert dark != bright
        assert ss2.compute_worst_background(p, o, d).score() == min(dark, bright)
        assert ss2.compute_worst_background(p, _view(o), _view(d)).score() == min(dark, bright)
        opaque, other = helpers.gradient(0), helpers.gradient(1)
        assert (ss2.compute_worst_background(p, opaque, other).score()
                == p.compute(opaque, other).score())
    for bg, want in ((0.1, dark), (0.9, bright)):
        assert abs(helpers.oracle_compute(o, d, bg)[1] - want) <= helpers.SCORE_TOL


def test_worst_background_with_alpha_on_either_side():
    """alpha_test.cc:74-131: a flat opaque image against the same pixels
    fully transparent (a zero alpha plane), in both orders."""
    opaque = helpers.ramp_image(32, 32, False, ss2.PixelType.Byte)
    opaque = ss2.Image(32, 32, opaque.format, np.full_like(opaque.data, 128))
    fmt = opaque.format.copy(alpha=ss2.AlphaType.Straight)
    data = np.zeros(ss2.required_bytes(fmt, 32, 32), np.uint8)
    data[:opaque.data.nbytes] = opaque.data
    transparent = ss2.Image(32, 32, fmt, data)
    with ss2.Ssimulacra2Pipeline(32, 32) as p:
        for o, d in ((opaque, transparent), (transparent, opaque)):
            dark = p.compute(o, d, 0.1).score()
            bright = p.compute(o, d, 0.9).score()
            expected = min(dark, bright)
            assert expected < 90.0
            assert ss2.compute_worst_background(p, o, d).score() == expected
            assert ss2.compute_worst_background(p, _view(o), _view(d)).score() == expected
            assert abs(helpers.oracle_compute(o, d, 0.1 if dark <= bright else 0.9)[1]
                       - expected) <= helpers.SCORE_TOL
