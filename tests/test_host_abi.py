"""The C ABI without a GPU: the library loads, exports every function the
header declares, and its host-side rules (formats, scale plan, decode
constants, score) match the oracle and the reference's own host code."""

import ctypes
import math
import os
import re

import numpy as np
import pytest

from oracle import binding as ob
from tests import helpers
from tests.test_oracle import _formats, needs_ref, ref
from vqm_b200 import ss2

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_functions():
    names = []
    for header in os.listdir(os.path.join(ROOT, "include")):
        if not header.endswith(".h"):
            continue
        text = open(os.path.join(ROOT, "include", header)).read()
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
        names += re.findall(r"^\s*(?:const\s+)?[\w\s\*]+?\b(vqm_cu_\w+)\s*\(", text, flags=re.M)
    return sorted(set(names))


def test_library_exports_every_declared_symbol():
    lib = ctypes.CDLL(ss2.library_path())
    names = declared_functions()
    assert len(names) >= 30
    for name in names:
        assert hasattr(lib, name), name
    # And the Python binding covers all of them.
    assert set(names) <= set(ss2.EXPORTED_SYMBOLS), set(names) - set(ss2.EXPORTED_SYMBOLS)


def test_version():
    assert ss2._lib.vqm_cu_version() >> 16 == 1


def _to_ss2(f: ob.Format) -> ss2.ImageFormat:
    return ss2.ImageFormat(f.type, f.family, f.alpha, f.range, f.matrix, f.transfer,
                           f.primaries, f.chroma_location, f.subsample_w, f.subsample_h,
                           f.depth)


def test_required_bytes_pins():
    # pipeline_test.cc:573 and :692.
    assert ss2.required_bytes(helpers.pinned_format(type=ss2.PixelType.Byte), 33, 17) == 1692
    grey = helpers.pinned_format(type=ss2.PixelType.Byte).copy(
        family=ss2.ColorFamily.Grey, matrix=ss2.MatrixCoefficients.Unspecified)
    assert ss2.required_bytes(grey, 8, 8) == 64


def test_required_bytes_and_constants_match_oracle():
    for f in _formats():
        for w, h in ((33, 17), (64, 30)):
            assert ss2.required_bytes(_to_ss2(f), w, h) == ob.required_bytes(f, w, h)
        try:
            want = ob.source_desc(f, 0)
        except ob.OracleError:
            continue
        try:
            ss2.validate_format(_to_ss2(f), 64, 64)
        except ss2.InvalidArgument:
            continue
        got = ss2.source_constants(_to_ss2(f), 0)
        assert np.array_equal(got, want), bytes(f)


@needs_ref
def test_validation_messages_match_reference():
    bad = []
    F = ob.Format
    base = F()
    base.type, base.family, base.range, base.matrix, base.transfer, base.primaries = 0, 1, 1, 0, 13, 1
    variants = [
        dict(type=7), dict(range=5), dict(alpha=9), dict(chroma_location=9), dict(matrix=3),
        dict(matrix=99), dict(primaries=3), dict(primaries=99), dict(depth=12),
        dict(subsample_w=3), dict(subsample_w=1), dict(family=2), dict(family=2, matrix=2),
        dict(family=2, matrix=1, subsample_w=1, subsample_h=1),
        dict(family=0, matrix=0), dict(family=0, matrix=2, subsample_w=1),
        dict(transfer=2), dict(transfer=3), dict(primaries=2), dict(family=5),
        dict(family=2, matrix=10), dict(family=2, matrix=14, transfer=16, primaries=1),
        dict(family=2, matrix=11), dict(family=2, matrix=12, primaries=10),
        dict(family=2, matrix=1, transfer=18, primaries=10), dict(range=0, type=0, depth=4),
        dict(type=1, depth=10, range=0), dict(family=2, matrix=9, transfer=14, primaries=9),
    ]
    for sizes in ((32, 32), (33, 17)):
        for v in variants:
            f = ob.Format.from_buffer_copy(bytes(base))
            for k, val in v.items():
                setattr(f, k, val)
            status = ref.vqmref_validate(ctypes.c_char_p(bytes(f)), *sizes)
            ref_msg = ref.vqmref_last_error().decode() if status else None
            try:
                ss2.validate_format(_to_ss2(f), *sizes)
                ours = None
            except ss2.InvalidArgument as e:
                ours = str(e)
            if ours != ref_msg:
                bad.append((v, sizes, ours, ref_msg))
    assert not bad, bad


def test_plan_scales_matches_oracle():
    for w, h in ((8, 8), (13, 9), (32, 32), (64, 64), (65, 65), (129, 97), (1920, 1080),
                 (3840, 2160), (321, 181), (3839, 2159), (8, 4000)):
        assert ss2.plan_scales(w, h) == ob.plan_scales(w, h)
    with pytest.raises(ss2.InvalidArgument, match="8x8"):
        ss2.plan_scales(4, 8)


@needs_ref
def test_channel_pruning_matches_reference():
    """Ssimulacra2ChannelPruned through the C ABI against score.cc compiled
    from the reference's sources, for every plan length."""
    for scales in range(1, 7):
        for s in range(scales):
            for c in range(3):
                assert ss2.channel_pruned(c, s, scales) == bool(
                    ref.vqmref_channel_pruned(c, s, scales)), (c, s, scales)
    for bad in ((3, 0, 6), (0, 6, 6), (0, 0, 7), (0, 0, 0)):
        with pytest.raises(ss2.InvalidArgument):
            ss2.channel_pruned(*bad)
    # 1080p keeps 11 of 18 planes: Y at L0, X and Y at L1-L2, X, Y and B at
    # L3-L4, nothing at L5.
    assert ss2.kept_pixels(1920, 1080) == 3_491_280


def test_host_score_bit_exact():
    rng = np.random.default_rng(3)
    for scales in range(1, 7):
        n = rng.uniform(0, 0.2, size=(scales, 18))
        assert ss2.score(n) == ob.score(n, scales)
    n = np.zeros((6, 18))
    n[0, 3] = math.nan
    with pytest.raises(ss2.InvalidArgument):
        ss2.score(n)
    with pytest.raises(ss2.InvalidArgument):
        ss2.score(np.zeros((7, 18)))


def test_pipeline_without_device_raises_runtime_error():
    from tests.conftest import cuda_available
    if cuda_available():
        pytest.skip("a device is present")
    with pytest.raises(ss2.CudaError):
        ss2.Ssimulacra2Pipeline(64, 64)
    with pytest.raises(ss2.InvalidArgument, match="8x8"):
        ss2.Ssimulacra2Pipeline(4, 8)


def test_automatic_strip_length():
    """The blur kernel a batch without a variant takes: for one pair, the
    strip length whose measured blur time on a B200 was least (1080p 2,
    1440p and 4K 4), for large batches the longest strip."""
    shapes = ss2.blur_variants()
    strip = lambda sizes: shapes[ss2.auto_blur_variant(sizes, sms=148)][3]  # noqa: E731
    assert strip([(1920, 1080)]) == 2
    assert strip([(2560, 1440)]) == 4
    assert strip([(3840, 2160)]) == 4
    assert strip([(1920, 1080)] * 64) == 16
    assert strip([(3840, 2160)] * 8) == 16
    assert strip([(256, 256)]) == 1
    # Every choice is a plain strip kernel of the default tile.
    for sizes in ([(1280, 720)], [(640, 360)] * 3, [(333, 187), (3840, 2160)]):
        w, h, threads, _, persistent = shapes[ss2.auto_blur_variant(sizes)]
        assert (w, h, threads, persistent) == (32, 32, 128, 0)
    with pytest.raises(ss2.InvalidArgument):
        ss2.auto_blur_variant([(4, 4)])
