"""Parity of the CUDA scorer with the CPU oracle, through the C ABI.

Bar: every one of the 108 features within 1e-4 relative (absolute floor
1e-9) of the FP32 oracle, which the oracle tests pin to VQM's goldens;
pruned features exactly 0; score within 1e-2; identity exactly 100; repeated
calls bit-identical. The FP64 oracle error of each score is reported.
"""

import ctypes
import math

import numpy as np
import pytest

from tests import helpers
from tests import synthetic
from vqm_b200 import ss2

pytestmark = pytest.mark.gpu


def check_parity(result, o, d, background=0.5, chroma_filter=0, label=""):
    norms, score = helpers.oracle_compute(o, d, background, chroma_filter)
    got = result.norms
    assert got.shape == norms.shape, label
    bad = helpers.feature_mismatch(got, norms)
    assert not bad, (label, bad[:8])
    mask = helpers.pruned_mask(got.shape[0])
    assert np.all(got[mask] == 0.0), label
    s = result.score()
    assert abs(s - score) <= helpers.SCORE_TOL, (label, s, score)
    _, score64 = helpers.oracle_compute(o, d, background, chroma_filter, precision=64)
    print(f"{label}: cuda {s:.8f} oracle32 {score:.8f} oracle64 {score64:.8f} "
          f"|d32| {abs(s - score):.2e} |d64| {abs(s - score64):.2e}")
    return s


@pytest.fixture(scope="module")
def pipe32():
    p = ss2.Ssimulacra2Pipeline(32, 32)
    yield p
    p.close()


def test_vqm_gradient_goldens(pipe32):
    # pipeline_test.cc:146-174.
    o = helpers.gradient(0)
    for v, gold in ((1, 93.17505696), (2, 92.12553218)):
        d = helpers.gradient(v)
        r = pipe32.compute(o, d)
        assert len(r.scales) == 4
        assert abs(r.score() - gold) <= 5e-3
        check_parity(r, o, d, label=f"gradient 0/{v}")


def test_identity_exactly_100(pipe32):
    img = helpers.gradient(0)
    r = pipe32.compute(img, img)
    assert r.score() == 100.0
    assert np.all(r.norms == 0.0)


@pytest.mark.parametrize("w,h,scales", [(8, 8, 2), (13, 9, 2), (64, 64, 5), (65, 65, 5),
                                        (129, 97, 5)])
def test_small_geometries(w, h, scales):
    # pipeline_test.cc:760-783: identity, scale count, repeatability.
    img = helpers.ramp_image(w, h, False)
    with ss2.Ssimulacra2Pipeline(w, h) as p:
        first = p.compute(img, img)
        assert len(first.scales) == scales
        assert first.score() == 100.0
        second = p.compute(img, img)
        assert np.array_equal(first.norms, second.norms)
        # A distorted ramp against the oracle at the same odd sizes.
        d = helpers.ramp_image(w, h, False)
        arr = d.data.view("<f4").copy()
        arr[::7] = np.clip(arr[::7] * 0.9 + 0.03, 0, 1)
        d.data = arr.view(np.uint8)
        check_parity(p.compute(img, d), img, d, label=f"ramp {w}x{h}")


def _pyramid_cases():
    return {
        "rgb8_256": lambda: helpers.plain_256_pair(),
        "rgb8_odd": lambda: synthetic.rgb_pair(333, 187, 5)[:2],
        "yuv420p10": lambda: synthetic.yuv_pair(322, 182, 6)[:2],
        "float_ramp": lambda: (helpers.ramp_image(65, 33, False), helpers.ramp_image(65, 33, False)),
        "rgb8_alpha": lambda: (helpers.ramp_image(40, 24, True, ss2.PixelType.Byte),) * 2,
    }


@pytest.mark.parametrize("case", list(_pyramid_cases()))
def test_pyramid_planes_bit_exact(case):
    """The XYB planes equal the oracle's bit for bit: decode, transfer, cube
    root and the box pyramid all round identically on both sides."""
    from oracle import binding as ob
    o, d = _pyramid_cases()[case]()
    with ss2.Ssimulacra2Pipeline(o.width, o.height) as p:
        p.compute(o, d, 0.3)
        scales = len(ss2.plan_scales(o.width, o.height))
        for image, img in enumerate((o, d)):
            want = ob.pyramid(helpers.to_oracle(img), 0.3)
            for level in range(scales):
                for c in range(3):
                    if ob.channel_pruned(c, level, scales):
                        continue
                    got = p.debug_plane(image, level, c)
                    assert np.array_equal(got.view(np.uint32), want[level][c].view(np.uint32)), \
                        (case, image, level, c, np.abs(got - want[level][c]).max())


def _yuv_fast_formats():
    F, T = ss2.ImageFormat, ss2.TransferCharacteristics

    def yuv(**kw):
        base = dict(type=ss2.PixelType.Word, depth=10, family=ss2.ColorFamily.Yuv,
                    range=ss2.PixelRange.Limited, matrix=ss2.MatrixCoefficients.Bt709,
                    transfer=T.Bt709, primaries=ss2.ColorPrimaries.Bt709, subsample_w=1,
                    subsample_h=1)
        base.update(kw)
        return F(**base)

    L = ss2.ChromaLocation
    return {
        "420p10_left": yuv(chroma_location=L.Left),
        "420p10_center": yuv(chroma_location=L.Center),
        "420p10_topleft": yuv(chroma_location=L.TopLeft),
        "420p10_top": yuv(chroma_location=L.Top),
        "420p10_bottomleft": yuv(chroma_location=L.BottomLeft),
        "420p10_bottom": yuv(chroma_location=L.Bottom),
        "422p8": yuv(type=ss2.PixelType.Byte, depth=0, subsample_h=0),
        "444p10": yuv(subsample_w=0, subsample_h=0),
        "440p10": yuv(subsample_w=0),
        "420p12_bt2020": yuv(depth=12, matrix=ss2.MatrixCoefficients.Bt2020Ncl,
                             transfer=T.Bt2020_12, primaries=ss2.ColorPrimaries.Bt2020),
        "420p8_gamma22": yuv(type=ss2.PixelType.Byte, depth=0, transfer=T.Bt470M),
        "420p16_gamma28_full": yuv(depth=16, range=ss2.PixelRange.Full, transfer=T.Bt470Bg),
    }


@pytest.mark.parametrize("name,w,h", [(n, 200, 134) for n in _yuv_fast_formats()] +
                         [("444p10", 201, 133), ("422p8", 200, 133), ("440p10", 201, 134)])
def test_yuv_fast_path_planes_bit_exact(name, w, h):
    """Integer YUV with a power-law transfer takes the fast decode (staged
    chroma window, per-parity taps); its planes equal the oracle's generic
    decode bit for bit, inside the image and along its edges. An image of
    odd width or height runs the generic prepare kernel instead (the YUV
    kernel takes whole 2x2 blocks only), with the same planes."""
    from oracle import binding as ob
    fmt = _yuv_fast_formats()[name]
    assert ss2.decode_path(fmt) == "yuv"
    ov = _values(fmt, w, h, 21)
    rng = np.random.default_rng(4)
    dv = [None if v is None else np.clip(v + rng.normal(0, 0.03, v.shape),
                                         -0.5 if i in (1, 2) else 0, 1)
          for i, v in enumerate(ov)]
    imgs = (helpers.pack_planes(fmt, w, h, ov), helpers.pack_planes(fmt, w, h, dv))
    with ss2.Ssimulacra2Pipeline(w, h) as p:
        p.compute(*imgs)
        scales = len(ss2.plan_scales(w, h))
        for image, img in enumerate(imgs):
            want = ob.pyramid(helpers.to_oracle(img), 0.5)
            for level in range(scales):
                for c in range(3):
                    if ob.channel_pruned(c, level, scales):
                        continue
                    got = p.debug_plane(image, level, c)
                    assert np.array_equal(got.view(np.uint32), want[level][c].view(np.uint32)), \
                        (name, image, level, c, np.abs(got - want[level][c]).max())


def test_plain_256_pair():
    o, d = helpers.plain_256_pair()
    with ss2.Ssimulacra2Pipeline(256, 256) as p:
        r = p.compute(o, d)
        check_parity(r, o, d, label="256x256 noise+quant")
        again = p.compute(o, d)
        assert np.array_equal(r.norms, again.norms)


@pytest.mark.parametrize("w,h", [(1920, 1080), (333, 187), (1001, 77), (640, 361),
                                 (2000, 9), (8, 1500)])
def test_rgb8_sizes(w, h):
    o, d, kind = synthetic.rgb_pair(w, h, seed=w * 7 + h)
    with ss2.Ssimulacra2Pipeline(w, h) as p:
        check_parity(p.compute(o, d), o, d, label=f"rgb8 {w}x{h} {kind}")


@pytest.mark.parametrize("w,h", [(1920, 1080), (3840, 2160), (322, 182), (1278, 720)])
def test_yuv420_10bit(w, h):
    o, d, kind = synthetic.yuv_pair(w, h, seed=w + 3 * h)
    with ss2.Ssimulacra2Pipeline(o.width, o.height) as p:
        check_parity(p.compute(o, d), o, d, label=f"yuv420p10 {w}x{h} {kind}")


def _variants():
    F = ss2.ImageFormat
    return {
        "float": F(type=ss2.PixelType.Float),
        "half": F(type=ss2.PixelType.Half),
        "word16": F(type=ss2.PixelType.Word),
        "word10_limited_rgb": F(type=ss2.PixelType.Word, depth=10, range=ss2.PixelRange.Limited),
        "grey8": F(type=ss2.PixelType.Byte, family=ss2.ColorFamily.Grey,
                   matrix=ss2.MatrixCoefficients.Unspecified),
        "yuv444_bt2020": F(type=ss2.PixelType.Word, family=ss2.ColorFamily.Yuv, depth=10,
                           range=ss2.PixelRange.Limited, matrix=ss2.MatrixCoefficients.Bt2020Ncl,
                           transfer=ss2.TransferCharacteristics.Bt2020_10,
                           primaries=ss2.ColorPrimaries.Bt2020),
        "yuv422_bt601": F(type=ss2.PixelType.Byte, family=ss2.ColorFamily.Yuv,
                          range=ss2.PixelRange.Limited, matrix=ss2.MatrixCoefficients.St170M,
                          transfer=ss2.TransferCharacteristics.Bt601,
                          primaries=ss2.ColorPrimaries.St170M, subsample_w=1),
        "yuv420_pq": F(type=ss2.PixelType.Word, family=ss2.ColorFamily.Yuv, depth=10,
                       range=ss2.PixelRange.Limited, matrix=ss2.MatrixCoefficients.Bt2020Ncl,
                       transfer=ss2.TransferCharacteristics.St2084,
                       primaries=ss2.ColorPrimaries.Bt2020, subsample_w=1, subsample_h=1,
                       chroma_location=ss2.ChromaLocation.TopLeft),
        "ictcp_hlg": F(type=ss2.PixelType.Word, family=ss2.ColorFamily.Yuv, depth=12,
                       range=ss2.PixelRange.Limited, matrix=ss2.MatrixCoefficients.Bt2100ICtCp,
                       transfer=ss2.TransferCharacteristics.AribB67,
                       primaries=ss2.ColorPrimaries.Bt2020),
        "cl_2020": F(type=ss2.PixelType.Word, family=ss2.ColorFamily.Yuv, depth=10,
                     range=ss2.PixelRange.Limited, matrix=ss2.MatrixCoefficients.Bt2020Cl,
                     transfer=ss2.TransferCharacteristics.Bt2020_10,
                     primaries=ss2.ColorPrimaries.Bt2020),
        "rgb8_alpha": F(type=ss2.PixelType.Byte, alpha=ss2.AlphaType.Straight),
        "rgbf_premul": F(type=ss2.PixelType.Float, alpha=ss2.AlphaType.Premultiplied),
        "xvycc": F(type=ss2.PixelType.Byte, family=ss2.ColorFamily.Yuv,
                   range=ss2.PixelRange.Limited, matrix=ss2.MatrixCoefficients.Bt709,
                   transfer=ss2.TransferCharacteristics.Iec61966_2_4,
                   primaries=ss2.ColorPrimaries.Bt709),
    }


def _values(fmt, w, h, seed):
    rng = np.random.default_rng(seed)
    base = synthetic.texture(w, h, rng) / 255.0
    layout = ss2.plane_layout(fmt, w, h)
    vals = []
    for p in range(4):
        if layout[p] is None:
            vals.append(None)
            continue
        _, pw, ph, _ = layout[p]
        src = base[min(p, 2)]
        if (pw, ph) != (w, h):
            src = src[: ph * (h // ph): h // ph, : pw * (w // pw): w // pw][:ph, :pw]
        if p in (1, 2) and fmt.family == ss2.ColorFamily.Yuv:
            src = (src - 0.5) * 0.6
        if p == 3:
            src = 0.2 + 0.8 * src
        vals.append(src)
    return vals


@pytest.mark.parametrize("name", list(_variants()))
@pytest.mark.parametrize("chroma_filter", [0, 1, 2])
def test_input_formats(name, chroma_filter):
    fmt = _variants()[name]
    sub = fmt.subsample_w or fmt.subsample_h
    if chroma_filter and not sub:
        pytest.skip("chroma filter only applies to subsampled chroma")
    w, h = 96, 66
    ov = _values(fmt, w, h, 11)
    dv = [None if v is None else np.clip(v + np.random.default_rng(5).normal(0, 0.02, v.shape),
                                         -0.5 if i in (1, 2) and fmt.family == 2 else 0, 1)
          for i, v in enumerate(ov)]
    o = helpers.pack_planes(fmt, w, h, ov)
    d = helpers.pack_planes(fmt, w, h, dv)
    with ss2.Ssimulacra2Pipeline(w, h, chroma_filter=chroma_filter) as p:
        for bg in ((0.1, 0.9) if fmt.alpha else (0.5,)):
            check_parity(p.compute(o, d, bg), o, d, bg, chroma_filter,
                         label=f"{name} filter {chroma_filter} bg {bg}")


@pytest.mark.parametrize("name", ["rgb8_limited", "rgb8_bt2020", "grey8"])
def test_table_decode_full_code_range(name):
    """8-bit table decode over every code 0..255: limited range puts codes
    below 16 at negative light (mixes that clamp to 0 and take the cube
    root's checked path), BT.2020 primaries go through a matrix (checked
    path), full-range grey stays non-negative (unchecked path)."""
    F = ss2.ImageFormat
    fmt = {"rgb8_limited": F(type=ss2.PixelType.Byte, range=ss2.PixelRange.Limited),
           "rgb8_bt2020": F(type=ss2.PixelType.Byte, primaries=ss2.ColorPrimaries.Bt2020),
           "grey8": F(type=ss2.PixelType.Byte, family=ss2.ColorFamily.Grey,
                      matrix=ss2.MatrixCoefficients.Bt709)}[name]
    w, h = 160, 96
    rng = np.random.default_rng(77)
    planes = 1 if fmt.family == ss2.ColorFamily.Grey else 3
    ramp = np.tile(np.arange(w, dtype=np.int64) * 256 // w, (h, 1))
    o = np.stack([(ramp + 37 * c + rng.integers(0, 9, (h, w))) % 256 for c in range(planes)])
    o[:, :24, :40] = 0  # a block of code 0 in every plane
    d = np.clip(o + rng.integers(-6, 7, o.shape), 0, 255)
    oi = ss2.Image(w, h, fmt, o.astype(np.uint8).reshape(-1).copy())
    di = ss2.Image(w, h, fmt, d.astype(np.uint8).reshape(-1).copy())
    with ss2.Ssimulacra2Pipeline(w, h) as p:
        check_parity(p.compute(oi, di), oi, di, label=name)


def test_mixed_format_pair():
    o, _, _ = synthetic.rgb_pair(320, 180, seed=1)
    _, d, _ = synthetic.yuv_pair(320, 180, seed=1)
    with ss2.Ssimulacra2Pipeline(320, 180) as p:
        check_parity(p.compute(o, d), o, d, label="rgb8 vs yuv420p10")


def test_batch_matches_pipeline():
    pairs = [synthetic.rgb_pair(333, 187, 1)[:2], synthetic.yuv_pair(640, 360, 2)[:2],
             synthetic.rgb_pair(8, 8, 3)[:2], synthetic.rgb_pair(1920, 1080, 4)[:2],
             synthetic.yuv_pair(1000, 563, 5)[:2], helpers.plain_256_pair()]
    b = ss2.Ssimulacra2Batch()
    results = b.compute_many(pairs)
    for (o, d), r in zip(pairs, results):
        with ss2.Ssimulacra2Pipeline(o.width, o.height) as p:
            single = p.compute(o, d)
        # The two may pick different strip lengths (they regroup the
        # compensated partial sums), so they agree to rounding.
        assert not helpers.feature_mismatch(single.norms, r.norms, rtol=1e-6, atol=1e-12)
        assert abs(r.device_score - r.score()) <= 1e-9
        check_parity(r, o, d, label=f"batch {o.width}x{o.height}")
    # A second, smaller batch on the same scorer reuses its memory (it may
    # pick a shorter strip, so it agrees to rounding).
    again = b.compute_many(pairs[:2])
    assert not helpers.feature_mismatch(again[1].norms, results[1].norms, rtol=1e-6,
                                        atol=1e-12)
    assert np.array_equal(b.compute_many(pairs[:2])[1].norms, again[1].norms)


def test_table_prepare_of_large_launches_is_bit_exact():
    """Large launches of the 8-bit table decode run 128-thread CTAs, small
    ones 256-thread CTAs; both write the same planes, so with the same blur
    kernel a pair scores bit for bit the same alone and in a batch of
    three ~1080p pairs, one of odd size (3,060 tiles of 64x64, the
    128-thread form on any device of up to 306 SMs)."""
    pairs = [synthetic.rgb_pair(1920, 1080, 60 + i)[:2] for i in range(2)]
    pairs.append(synthetic.rgb_pair(1919, 1077, 62)[:2])  # partial tiles, odd sizes
    b = ss2.Ssimulacra2Batch(variant=0)
    together = b.compute_many(pairs)
    for (o, d), r in zip(pairs, together):
        alone = b.compute_many([(o, d)])[0]
        assert np.array_equal(alone.norms, r.norms) and alone.device_score == r.device_score
        check_parity(r, o, d, label="1080p in a batch of three")
    b.close()


def test_yuv_prepare_of_large_launches_is_bit_exact():
    """Large YUV launches whose images all have 4:2:0 chroma run 128-thread
    CTAs with a 4:2:0 chroma window; other YUV launches run 256-thread CTAs
    with a window for any subsampling. Both write the same planes: 720p
    pairs score bit for bit the same alone (480 tiles, 256 threads) and
    beside a 4K pair (5,040 tiles, 128 threads), and a 4:2:2 image keeps its
    launch on the 256-thread kernel (the 4K pair then scores as before) and
    matches the oracle."""
    big = synthetic.yuv_pair(3840, 2160, 80)[:2]
    small = [synthetic.yuv_pair(1280, 720, 81 + i)[:2] for i in range(2)]
    b = ss2.Ssimulacra2Batch(variant=0)
    try:
        together = b.compute_many(small + [big])
        for (o, d), r in zip(small, together[:2]):
            alone = b.compute_many([(o, d)])[0]
            assert np.array_equal(alone.norms, r.norms) and alone.device_score == r.device_score
            check_parity(r, o, d, label="720p 4:2:0 beside a 4K pair")
        check_parity(together[2], *big, label="4K 4:2:0 in a large launch")
        fmt = _variants()["yuv422_bt601"]
        w, h = 640, 360
        ov = _values(fmt, w, h, 82)
        dv = [None if v is None else np.clip(v * 0.97 + 0.01, -0.5 if i in (1, 2) else 0, 1)
              for i, v in enumerate(ov)]
        o422, d422 = helpers.pack_planes(fmt, w, h, ov), helpers.pack_planes(fmt, w, h, dv)
        mixed = b.compute_many([big, (o422, d422)])
        assert np.array_equal(mixed[0].norms, together[2].norms)
        check_parity(mixed[1], o422, d422, label="4:2:2 in a large YUV launch")
    finally:
        b.close()


@pytest.mark.parametrize("variant", range(len(ss2.blur_variants())))
def test_every_blur_variant(variant):
    """Every compiled blur kernel gives the oracle's features; they differ
    from each other only in how their partials group the sums (per tile, or
    per strip of tiles), so they agree to rounding."""
    pairs = [synthetic.rgb_pair(333, 187, 41)[:2], synthetic.yuv_pair(1280, 720, 42)[:2],
             synthetic.rgb_pair(8, 8, 43)[:2], synthetic.rgb_pair(97, 2000, 44)[:2]]
    b = ss2.Ssimulacra2Batch(variant=variant)
    ref = ss2.Ssimulacra2Batch(variant=0).compute_many(pairs)
    # Variants with variant 0's tile and one tile per partial (persistent
    # CTAs) reduce every tile as it does, so they agree with it bit for bit.
    shape, shape0 = ss2.blur_variants()[variant], ss2.blur_variants()[0]
    same_grouping = shape[:2] == shape0[:2] and shape[3] == 1
    again = b.compute_many(pairs)
    for (o, d), r, r0, r1 in zip(pairs, b.compute_many(pairs), ref, again):
        check_parity(r, o, d, label=f"variant {variant} {o.width}x{o.height}")
        assert np.array_equal(r.norms, r1.norms)  # each kernel repeats itself exactly
        if same_grouping:
            assert np.array_equal(r.norms, r0.norms) and r.device_score == r0.device_score
        else:
            assert not helpers.feature_mismatch(r.norms, r0.norms, rtol=1e-6, atol=1e-12)


def test_pool_score_many_in_order():
    pairs = [synthetic.rgb_pair(200 + 10 * i, 120, i)[:2] for i in range(5)]
    pool = ss2.Ssimulacra2Pool(workers=2, chunk=2)
    scores = pool.score_many(pairs)
    for (o, d), s in zip(pairs, scores):
        _, want = helpers.oracle_compute(o, d)
        assert abs(s - want) <= helpers.SCORE_TOL


def test_pool_streams_lists_in_any_order():
    """Lists submitted back to back (the second before the first's results
    are taken) give the same results as one list at a time, in either order
    of taking them."""
    a = [synthetic.rgb_pair(200 + 10 * i, 120, 70 + i)[:2] for i in range(5)]
    b = [synthetic.yuv_pair(160, 90 + 2 * i, 80 + i)[:2] for i in range(3)]
    pool = ss2.Ssimulacra2Pool(workers=2, chunk=2)
    want_a, want_b = pool.compute_many(a), pool.compute_many(b)
    ta, tb = pool.submit_many(a), pool.submit_many(b)
    got_b, got_a = pool.results(tb), pool.results(ta)
    for got, want in ((got_a, want_a), (got_b, want_b)):
        assert len(got) == len(want)
        for g, w in zip(got, want):
            assert np.array_equal(g.norms, w.norms) and g.device_score == w.device_score
    assert pool.results(pool.submit_many([])) == []
    with pytest.raises(ss2.InvalidArgument):
        pool.results(ta)  # already taken
    pool.close()


def test_resident_and_streaming_agree_bitwise():
    o, d = helpers.plain_256_pair()
    with ss2.Ssimulacra2Pipeline(256, 256, gpu_resident_images=2) as p:
        streamed = p.compute(o, d)
        a, b = p.upload(o), p.upload(d)
        assert np.array_equal(p.compute(a, b).norms, streamed.norms)
        assert np.array_equal(p.compute(a, d).norms, streamed.norms)
        with pytest.raises(ss2.InvalidArgument):
            p.upload(o)  # both slots in use
        p.release(a)
        with pytest.raises(ss2.InvalidArgument, match="not a live resident image"):
            p.compute(a, b)
        p.release(a)  # stale release is ignored
        c = p.upload(d)
        assert c.slot != a.slot
        assert p.compute(c, b).score() == 100.0


def test_reference_pyramid_reuse():
    """vulkan.cc:238-243, 714-736: the same resident original with the same
    background skips its prepare; results stay bit-identical."""
    o, d1, _ = synthetic.rgb_pair(320, 180, 71)
    _, d2, _ = synthetic.rgb_pair(320, 180, 72)
    with ss2.Ssimulacra2Pipeline(320, 180, gpu_resident_images=3) as p:
        ref = [p.compute(o, d).norms for d in (d1, d2)]
        ref_bg = p.compute(o, d2, 0.2).norms
        assert p.reference_reuses() == 0
        a, b1, b2 = p.upload(o), p.upload(d1), p.upload(d2)
        assert np.array_equal(p.compute(a, b1).norms, ref[0])
        assert np.array_equal(p.compute(a, b2).norms, ref[1])
        assert p.reference_reuses() == 1
        assert np.array_equal(p.compute(a, d1).norms, ref[0])  # streamed distorted
        assert p.reference_reuses() == 2
        assert np.array_equal(p.compute(a, b2, 0.2).norms, ref_bg)  # new background
        assert p.reference_reuses() == 2
        p.compute(o, d1)  # a streamed original replaces the cached planes
        assert np.array_equal(p.compute(a, b2).norms, ref[1])
        assert p.reference_reuses() == 2
        p.set_graphs(False)
        assert np.array_equal(p.compute(a, b1).norms, ref[0])
        assert p.reference_reuses() == 3
        p.release(b1)
        p.release(a)  # forgets the cached original
        a2 = p.upload(d1)
        assert np.array_equal(p.compute(a2, b2).norms, p.compute(d1, d2).norms)
        assert p.reference_reuses() == 3


def test_mixed_resident_reference_with_alpha():
    """pipeline_test.cc:47-118 (the SSIMULACRA 2 half): a resident original
    with straight alpha against streamed distorted images at two
    backgrounds. With alpha the background changes the planes, so a cached
    reference pyramid must be re-prepared when it changes; every resident
    result equals the streamed one bit for bit (VQM: within 1e-12)."""
    o = helpers.ramp_image(32, 32, True, ss2.PixelType.Byte)
    d_data = o.data.copy()
    d_data[:32 * 32] = 0
    other_data = o.data.copy()
    other_data[32 * 32:2 * 32 * 32] = 0
    d = ss2.Image(32, 32, o.format, d_data)
    other = ss2.Image(32, 32, o.format, other_data)
    with ss2.Ssimulacra2Pipeline(32, 32) as p:
        dark = p.compute(o, d, 0.1)
        bright = p.compute(o, d, 0.9)
        other_dark = p.compute(o, other, 0.1)
        assert dark.score() != bright.score()  # the background matters here
        ref = p.upload(o)
        assert np.array_equal(p.compute(ref, d, 0.1).norms, dark.norms)
        assert np.array_equal(p.compute(ref, d, 0.1).norms, dark.norms)
        assert np.array_equal(p.compute(ref, other, 0.1).norms, other_dark.norms)
        assert np.array_equal(p.compute(ref, d, 0.9).norms, bright.norms)
        tok = p.submit(ref, d)
        with pytest.raises(ss2.LogicError):
            p.submit(ref, d)
        p.finish(tok)
        short = ss2.Image(32, 32, o.format, d.data[:-1])
        with pytest.raises(ss2.InvalidArgument):
            p.submit(ref, short)
        p.release(ref)
        with pytest.raises(ss2.InvalidArgument):
            p.compute(ref, d)
        replacement = p.upload(d)
        assert np.array_equal(p.compute(replacement, d).norms, p.compute(d, d).norms)
    for bg, want in ((0.1, dark), (0.9, bright)):
        _, score = helpers.oracle_compute(o, d, bg)
        assert abs(want.score() - score) <= helpers.SCORE_TOL
    with ss2.Ssimulacra2Pipeline(32, 32, streaming_inputs=False) as p:
        ref = p.upload(o)
        with pytest.raises(ss2.InvalidArgument):
            p.compute(ref, d)


def test_invalid_formats_rejected_on_every_path():
    """pipeline_test.cc:218-274 (the SSIMULACRA 2 half): a format VQM rejects
    raises InvalidArgument from compute on packed images and on plane views,
    from upload and from allocate_image, and takes nothing from the
    caller-owned input pool."""
    base = ss2.ImageFormat()
    for w, h in ((32, 32), (33, 17)):
        image_bytes = ss2.required_bytes(base, w, h)
        invalid = [base.copy(subsample_w=1),  # RGB with subsampled planes
                   base.copy(family=ss2.ColorFamily.Yuv)]  # YUV with the RGB matrix
        if w % 2 or h % 2:
            invalid.append(base.copy(family=ss2.ColorFamily.Yuv,
                                     matrix=ss2.MatrixCoefficients.Bt709,
                                     subsample_w=1, subsample_h=1))
        invalid += [base.copy(range=255), base.copy(alpha=255)]
        with ss2.Ssimulacra2Pipeline(w, h, input_bytes=2 * image_bytes + 63) as p:
            for bad in invalid:
                packed = ss2.Image(w, h, bad, np.zeros(image_bytes, np.uint8))
                planes = [np.zeros(4 * w * h, np.uint8) for _ in range(4)]
                view = ss2.HostImage(w, h, bad, planes)
                with pytest.raises(ss2.InvalidArgument):
                    p.compute(packed, packed)
                with pytest.raises(ss2.InvalidArgument):
                    p.compute(view, view)
                with pytest.raises(ss2.InvalidArgument):
                    p.upload(packed)
                with pytest.raises(ss2.InvalidArgument):
                    p.allocate_image(bad)
            a, b = p.allocate_image(base), p.allocate_image(base)
            assert a.bytes + b.bytes == 2 * image_bytes


def test_streaming_submission_validation():
    """pipeline_test.cc:359-446 (the SSIMULACRA 2 half): bad streamed inputs
    raise InvalidArgument; while a submission is in flight every call that
    would touch the pipeline's inputs raises LogicError and the pending pair
    is left as it was; after Finish, handle 0 (a default handle) raises
    InvalidArgument in a submission and releases as a no-op."""
    o, d = helpers.gradient(0), helpers.gradient(1)
    w, h = o.width, o.height
    oversized = ss2.Image(w, h, d.format, np.zeros(20 * w * h, np.uint8))
    short = ss2.Image(w, h, o.format, o.data[:1])
    wrong_size = ss2.Image(w - 1, h, o.format,
                           np.zeros(ss2.required_bytes(o.format, w - 1, h), np.uint8))
    no_image = ss2.UploadedImage(0, (w, h))
    no_buffer = ss2.ImageBuffer(0, (w, h), 0)
    with ss2.Ssimulacra2Pipeline(w, h) as p:
        resident, resident_d = p.upload(o), p.upload(d)
        with pytest.raises(ss2.InvalidArgument):
            p.upload(o)  # both resident slots are taken
        for bad in ((o, oversized), (short, d), (wrong_size, d)):
            with pytest.raises(ss2.InvalidArgument):
                p.submit(*bad)
        expected = p.compute(o, d)
        tok = p.submit(o, d)
        in_flight = [
            lambda: p.submit(o, o), lambda: p.submit(o, oversized),
            lambda: p.compute(o, oversized), lambda: p.upload(o),
            lambda: p.upload(oversized), lambda: p.release(resident),
            lambda: p.release(no_image), lambda: p.submit(resident, resident_d),
            lambda: p.submit(no_image, resident), lambda: p.compute(no_image, resident),
            lambda: p.allocate_image(o.format), lambda: p.map_image(no_buffer),
            lambda: p.release(no_buffer), lambda: p.submit(no_buffer, no_buffer),
            lambda: p.compute(no_buffer, no_buffer)]
        for call in in_flight:
            with pytest.raises(ss2.LogicError):
                call()
        assert np.array_equal(p.finish(tok).norms, expected.norms)
        with pytest.raises(ss2.InvalidArgument):
            p.finish(tok)
        with pytest.raises(ss2.InvalidArgument):
            p.submit(no_image, resident)
        with pytest.raises(ss2.InvalidArgument):
            p.submit(no_buffer, no_buffer)
        p.release(no_image)
        p.release(no_buffer)
        p.release(resident)
        p.release(resident_d)


def test_resident_handle_contracts():
    """pipeline_test.cc:478-513: a released handle does not alias the image
    that reuses its slot, and a replacement scores like its pixels."""
    o, d = helpers.gradient(0), helpers.gradient(1)
    with ss2.Ssimulacra2Pipeline(o.width, o.height) as p:
        old, other = p.upload(o), p.upload(d)
        before = p.compute(old, other).score()
        with pytest.raises(ss2.InvalidArgument):
            p.upload(o)
        wrong = ss2.UploadedImage(other.slot, (o.width - 1, o.height))
        wrong_img = ss2.Image(o.width - 1, o.height, d.format,
                              np.zeros(ss2.required_bytes(d.format, o.width - 1, o.height),
                                       np.uint8))
        with pytest.raises(ss2.InvalidArgument):
            p.submit(old, wrong_img)
        p.release(old)
        replacement = p.upload(d)
        with pytest.raises(ss2.InvalidArgument):
            p.submit(old, other)
        expected = p.compute(d, d).score()
        after = p.compute(replacement, other).score()
        assert after == expected == 100.0
        assert abs(before - after) > 1e-5
        del wrong
    # One slot: a second upload has nowhere to go until the first is released
    # (pipeline_test.cc:451-476).
    with ss2.Ssimulacra2Pipeline(o.width, o.height, gpu_resident_images=1) as single:
        first = single.upload(o)
        with pytest.raises(ss2.InvalidArgument):
            single.upload(d)
        single.release(first)
        single.upload(d)


def test_submit_finish_contracts():
    o, d = helpers.plain_256_pair()
    with ss2.Ssimulacra2Pipeline(256, 256) as p:
        expected = p.compute(o, d)
        tok = p.submit(o, d)
        with pytest.raises(ss2.LogicError):
            p.submit(o, o)
        with pytest.raises(ss2.LogicError):
            p.upload(o)
        r = p.finish(tok)
        assert np.array_equal(r.norms, expected.norms)
        with pytest.raises(ss2.InvalidArgument):
            p.finish(tok)
        short = ss2.Image(256, 256, o.format, o.data[:-1])
        with pytest.raises(ss2.InvalidArgument):
            p.compute(short, d)
        wrong = synthetic.rgb_pair(128, 256, 0)[0]
        with pytest.raises(ss2.InvalidArgument, match="geometry"):
            p.compute(wrong, d)


def test_streaming_disabled():
    o, d = helpers.plain_256_pair()
    with ss2.Ssimulacra2Pipeline(256, 256, streaming_inputs=False) as p:
        with pytest.raises(ss2.InvalidArgument):
            p.compute(o, d)
        a, b = p.upload(o), p.upload(d)
        _, want = helpers.oracle_compute(o, d)
        assert abs(p.compute(a, b).score() - want) <= helpers.SCORE_TOL


def _cudart():
    for name in ("libcudart.so.12", "libcudart.so"):
        try:
            return ctypes.CDLL(name)
        except OSError:
            continue
    import torch  # the torch wheel ships a cudart
    import glob
    import os
    libs = glob.glob(os.path.join(os.path.dirname(torch.__file__), "..", "nvidia",
                                  "cuda_runtime", "lib", "libcudart.so*"))
    return ctypes.CDLL(libs[0])


def test_device_buffers_and_caller_pool():
    import torch
    o, d = helpers.plain_256_pair()
    nbytes = o.data.nbytes
    with ss2.Ssimulacra2Pipeline(256, 256, input_bytes=2 * ((nbytes + 63) // 64 * 64)) as p:
        want = p.compute(o, d)
        # Caller-owned device memory read in place.
        to = torch.from_numpy(o.data).cuda()
        td = torch.from_numpy(d.data).cuda()
        do = ss2.DeviceImage.packed(256, 256, o.format, to.data_ptr(), to)
        dd = ss2.DeviceImage.packed(256, 256, d.format, td.data_ptr(), td)
        assert np.array_equal(p.compute(do, dd).norms, want.norms)
        # AllocateImage / MapImage pool.
        a = p.allocate_image(o.format)
        b = p.allocate_image(d.format)
        assert a.bytes == nbytes and b.bytes == nbytes
        with pytest.raises(ss2.InvalidArgument):
            p.allocate_image(o.format)  # pool full
        # Written like VQM's mapped arena: a host copy into the mapping.
        for buf, img in ((a, o), (b, d)):
            ctypes.memmove(p.map_image(buf), img.data.ctypes.data, nbytes)
        assert np.array_equal(p.compute(a, b).norms, want.norms)
        # Or by the copy engine from device memory (unified addressing).
        rt = _cudart()
        for buf, t in ((a, td), (b, to)):
            assert rt.cudaMemcpy(ctypes.c_void_p(p.map_image(buf)), ctypes.c_void_p(t.data_ptr()),
                                 ctypes.c_size_t(nbytes), 4) == 0
        assert np.array_equal(p.compute(b, a).norms, want.norms)
        tok = p.submit(a, b)
        with pytest.raises(ss2.LogicError):
            p.release(a)
        with pytest.raises(ss2.LogicError):
            p.map_image(a)
        p.finish(tok)
        p.release(a)
        with pytest.raises(ss2.InvalidArgument):
            p.compute(a, b)
        c = p.allocate_image(o.format)
        assert c.slot != a.slot


def test_strided_host_planes():
    o, d = helpers.plain_256_pair()
    pad = 37
    views = []
    for img in (o, d):
        planes = []
        for p in range(3):
            off = p * 256 * 256
            plane = img.data[off:off + 256 * 256].reshape(256, 256)
            padded = np.zeros((256, 256 + pad), dtype=np.uint8)
            padded[:, :256] = plane
            planes.append(padded)
        views.append(ss2.HostImage(256, 256, img.format, planes + [None],
                                   (256 + pad, 256 + pad, 256 + pad, 0)))
    with ss2.Ssimulacra2Pipeline(256, 256) as p:
        assert np.array_equal(p.compute(*views).norms, p.compute(o, d).norms)


def test_graphs_on_and_off_agree():
    o, d = helpers.plain_256_pair()
    with ss2.Ssimulacra2Pipeline(256, 256) as p:
        a = p.compute(o, d)
        p.set_graphs(False)
        b = p.compute(o, d)
        p.set_graphs(True)
        c = p.compute(o, d)
    assert np.array_equal(a.norms, b.norms) and np.array_equal(a.norms, c.norms)


def test_identity_at_4k():
    o, _, _ = synthetic.yuv_pair(3840, 2160, seed=9)
    with ss2.Ssimulacra2Pipeline(3840, 2160) as p:
        r = p.compute(o, o)
    assert r.score() == 100.0 and np.all(r.norms == 0.0)


def _random_case(seed):
    """A seeded format, size, chroma siting, filter and background."""
    rng = np.random.default_rng(9000 + seed)
    F, T, P = ss2.ImageFormat, ss2.TransferCharacteristics, ss2.PixelType
    kinds = [
        lambda: F(type=P.Byte),
        lambda: F(type=P.Byte, range=ss2.PixelRange.Limited, transfer=T.Bt709),
        lambda: F(type=P.Word, depth=int(rng.choice([10, 12, 16]))),
        lambda: F(type=P.Float, transfer=T.Linear),
        lambda: F(type=P.Half),
        lambda: F(type=P.Byte, family=ss2.ColorFamily.Grey, matrix=ss2.MatrixCoefficients.Bt709),
        lambda: F(type=P.Byte, alpha=ss2.AlphaType.Straight),
    ]
    for sw, sh in ((1, 1), (1, 0), (0, 0), (0, 1)):
        kinds.append(lambda sw=sw, sh=sh: F(
            type=P.Word if rng.random() < 0.6 else P.Byte,
            depth=int(rng.choice([10, 12])) if rng.random() < 0.6 else 0,
            family=ss2.ColorFamily.Yuv, range=ss2.PixelRange.Limited,
            matrix=ss2.MatrixCoefficients.Bt709,
            transfer=[T.Bt709, T.Bt470M, T.Bt470Bg, T.Srgb][int(rng.integers(0, 4))],
            primaries=ss2.ColorPrimaries.Bt709 if rng.random() < 0.7 else ss2.ColorPrimaries.Bt2020,
            chroma_location=int(rng.integers(0, 6)), subsample_w=sw, subsample_h=sh))
    fmt = kinds[int(rng.integers(0, len(kinds)))]()
    if fmt.type == P.Byte and fmt.depth:
        fmt.depth = 0
    w = int(rng.integers(8, 400)) << fmt.subsample_w
    h = int(rng.integers(8, 260)) << fmt.subsample_h
    sub = fmt.subsample_w or fmt.subsample_h
    chroma_filter = int(rng.integers(0, 3)) if sub else 0
    background = float(rng.choice([0.1, 0.5, 0.9]))
    return fmt, w, h, chroma_filter, background


@pytest.mark.parametrize("seed", range(24))
def test_randomized_formats_and_sizes(seed):
    """Seeded sweep over formats, sizes (odd included where the format
    allows), chroma sitings and filters, transfers and backgrounds: the
    device result matches the oracle, whichever decode path each image
    takes."""
    fmt, w, h, chroma_filter, background = _random_case(seed)
    ov = _values(fmt, w, h, 100 + seed)
    rng = np.random.default_rng(200 + seed)
    dv = [None if v is None else np.clip(v + rng.normal(0, 0.02, v.shape),
                                         -0.5 if i in (1, 2) and fmt.family == 2 else 0, 1)
          for i, v in enumerate(ov)]
    o, d = helpers.pack_planes(fmt, w, h, ov), helpers.pack_planes(fmt, w, h, dv)
    path = ss2.decode_path(fmt, chroma_filter)
    with ss2.Ssimulacra2Pipeline(w, h, chroma_filter=chroma_filter) as p:
        check_parity(p.compute(o, d, background), o, d, background, chroma_filter,
                     label=f"seed {seed} {w}x{h} path {path}")
