"""The decode pinned to the reference's independent FP64 model of the input
conversions (tests/input/input_reference.h of the reference), not to this
repository's own restatement of the shaders: for every A/B case of the
reference's input-format tests, (A, B) must score like (B, B) within the
reference's bounds, on the CPU oracle and on the CUDA pipeline (see
tests/input_ab.py)."""

import numpy as np
import pytest

from tests import helpers, input_ab
from vqm_b200 import ss2

VALUES = input_ab.load_fixture()
CASES = input_ab.cases(VALUES)
IDS = [c.name for c in CASES]


def test_fixture_matches_the_reference_model():
    ref = input_ab.live_reference()
    if ref is None:
        pytest.skip("oracle/_ref/libvqm_ref.so (reference checkout) is not built")
    live = input_ab.reference_values(ref)
    assert sorted(live) == sorted(VALUES)
    for k, v in live.items():
        assert np.array_equal(v, VALUES[k]), k


def test_case_count_covers_the_reference_suite():
    # 5 datatype/range, 18 transfer + 1 chromatic HLG, 11 matrix, 10
    # primaries, 1 full-range byte chroma, 11 subsampling, 3 CL, 2 ICtCp,
    # 2 alpha backgrounds.
    assert len(CASES) == 64


@pytest.mark.parametrize("case", CASES, ids=IDS)
def test_oracle_decodes_like_the_reference_model(case):
    pair, _ = helpers.oracle_compute(case.a, case.b, case.background, case.chroma_filter)
    same, _ = helpers.oracle_compute(case.b, case.b, case.background, case.chroma_filter)
    delta = input_ab.max_norm_delta(pair, same)
    assert delta <= case.tolerance, f"{case.name}: {delta:.3e} > {case.tolerance:.1e}"


@pytest.mark.gpu
@pytest.mark.parametrize("case", CASES, ids=IDS)
def test_cuda_decodes_like_the_reference_model(case):
    with ss2.Ssimulacra2Pipeline(input_ab.SIDE, input_ab.SIDE,
                                 chroma_filter=case.chroma_filter) as pipe:
        pair = pipe.compute(case.a, case.b, case.background).norms
        same = pipe.compute(case.b, case.b, case.background).norms
    delta = input_ab.max_norm_delta(pair, same)
    assert delta <= case.tolerance, f"{case.name}: {delta:.3e} > {case.tolerance:.1e}"


def _zero_premultiplied():
    fmt = helpers.pinned_format(alpha=ss2.AlphaType.Premultiplied)
    zero = [np.zeros((input_ab.SIDE, input_ab.SIDE), np.float32)] * 4
    return helpers.pack_planes(fmt, input_ab.SIDE, input_ab.SIDE, zero)


def test_oracle_zero_alpha_is_finite():
    """Premultiplied with zero alpha must not divide by zero
    (input_format_chroma_test.cc:380-393)."""
    img = _zero_premultiplied()
    norms, score = helpers.oracle_compute(img, img)
    assert np.all(np.isfinite(norms)) and np.isfinite(score) and score <= 100.0


@pytest.mark.gpu
def test_cuda_zero_alpha_is_finite():
    img = _zero_premultiplied()
    with ss2.Ssimulacra2Pipeline(input_ab.SIDE, input_ab.SIDE) as pipe:
        r = pipe.compute(img, img)
    assert np.all(np.isfinite(r.norms)) and np.isfinite(r.score()) and r.score() <= 100.0
