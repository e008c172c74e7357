"""Shared test fixtures: the reference suite's images, oracle conversion and
norm comparison.

The image builders restate the reference test support
(tests/support.h of GreatValueCreamSoda/vqm): MakeGradient (:93-103,
259-289), MakeRampImage (:291-316) and PackPlanes (:185-249).
"""

from __future__ import annotations

import math

import numpy as np

from oracle import binding as ob
from tests import synthetic
from vqm_b200 import ss2

SIDE = 32

# Per-feature tolerance against the FP32 oracle (the VQM proxy): relative to
# the value with a small absolute floor; pruned features must be exactly 0.
FEATURE_RTOL = 1e-4
FEATURE_ATOL = 1e-9
SCORE_TOL = 1e-2


def pinned_format(alpha=ss2.AlphaType.None_, type=ss2.PixelType.Float) -> ss2.ImageFormat:
    """PinnedFormat (tests/support.h:105-117)."""
    return ss2.ImageFormat(type=type, family=ss2.ColorFamily.Rgb, alpha=alpha,
                           matrix=ss2.MatrixCoefficients.Rgb,
                           transfer=ss2.TransferCharacteristics.Srgb,
                           primaries=ss2.ColorPrimaries.Bt709)


def gradient(variant: int) -> ss2.Image:
    """MakeGradient(variant): 0 gradient, 1 checkerboard +16 red, 2 3-bit
    truncation; 32x32 8-bit sRGB."""
    x = np.arange(SIDE)[None, :].repeat(SIDE, 0)
    y = np.arange(SIDE)[:, None].repeat(SIDE, 1)
    r = (x * 255) // (SIDE - 1)
    g = (y * 255) // (SIDE - 1)
    b = ((x * 7 + y * 11) * 13) & 255
    if variant == 1:
        r = np.where(((x + y) & 1) == 0, np.minimum(r + 16, 255), r)
    if variant == 2:
        r, g, b = r & 0xF8, g & 0xF8, b & 0xF8
    fmt = pinned_format(type=ss2.PixelType.Byte)
    data = np.concatenate([r.ravel(), g.ravel(), b.ravel()]).astype(np.uint8)
    assert data.nbytes == ss2.required_bytes(fmt, SIDE, SIDE)
    return ss2.Image(SIDE, SIDE, fmt, data)


def _half_bits(values: np.ndarray) -> np.ndarray:
    return values.astype(np.float16).view(np.uint16)


def pack_planes(fmt: ss2.ImageFormat, w: int, h: int, values) -> ss2.Image:
    """PackPlanes: normalised values -> the format's samples (lround of the
    inverse of the decode's scale/offset, clamped for integer types)."""
    data = np.zeros(ss2.required_bytes(fmt, w, h), dtype=np.uint8)
    layout = ss2.plane_layout(fmt, w, h)
    depth = fmt.depth or {0: 8, 1: 16, 2: 16, 3: 32}[fmt.type]
    integer = fmt.type in (ss2.PixelType.Byte, ss2.PixelType.Word)
    for p, geo in enumerate(layout):
        if geo is None:
            continue
        off, pw, ph, sb = geo
        v = np.asarray(values[p], dtype=np.float64).reshape(-1)[: pw * ph]
        chroma = p in (1, 2) and fmt.family == ss2.ColorFamily.Yuv
        scale, offset = plane_scale_offset(fmt, chroma, p == 3)
        raw = (v - offset) / scale
        if integer:
            raw = np.clip(raw, 0, (1 << depth) - 1)
            code = np.floor(np.abs(raw) + 0.5) * np.sign(raw)  # lround
            dt = np.uint8 if fmt.type == ss2.PixelType.Byte else np.dtype("<u2")
            bytes_ = code.astype(dt).view(np.uint8)
        elif fmt.type == ss2.PixelType.Half:
            bytes_ = _half_bits(raw.astype(np.float32)).view(np.uint8)
        else:
            bytes_ = raw.astype("<f4").view(np.uint8)
        data[off:off + bytes_.size] = bytes_
    return ss2.Image(w, h, fmt, data)


def plane_scale_offset(fmt: ss2.ImageFormat, chroma: bool, alpha: bool):
    """PlaneScaleOffset (src/input.cc:714-757), as float32 values."""
    if fmt.type in (ss2.PixelType.Half, ss2.PixelType.Float):
        return 1.0, 0.0
    depth = fmt.depth or {0: 8, 1: 16}[fmt.type]
    full = alpha or fmt.range == ss2.PixelRange.Full
    ycgco = fmt.matrix == ss2.MatrixCoefficients.YCgCo
    rng = (1 << depth) - 1 if full else ((224 if chroma and not ycgco else 219) << (depth - 8))
    off = 0.0 if alpha else (float(1 << (depth - 1)) if chroma else (0.0 if full else float(16 << (depth - 8))))
    return float(np.float32(1.0 / rng)), float(np.float32(-off / rng))


def ramp_image(w: int, h: int, with_alpha: bool, type=ss2.PixelType.Float) -> ss2.Image:
    """MakeRampImage (tests/support.h:291-316)."""
    x = np.arange(w)[None, :].repeat(h, 0).astype(np.float32)
    y = np.arange(h)[:, None].repeat(w, 1).astype(np.float32)
    xi, yi = x.astype(np.int64), y.astype(np.int64)
    v0 = x / np.float32(w - 1)
    v1 = y / np.float32(h - 1)
    v2 = ((xi * 7 + yi * 11) % 256).astype(np.float32) / np.float32(255.0)
    values = [v0, v1, v2, None]
    if with_alpha:
        values[3] = ((xi + 3 * yi) % 7).astype(np.float32) / np.float32(6.0)
    fmt = pinned_format(ss2.AlphaType.Straight if with_alpha else ss2.AlphaType.None_, type)
    return pack_planes(fmt, w, h, values)


def plain_256_pair():
    """The seeded 256x256 8-bit sRGB pair (texture; noise sigma 4; 8x8 block
    quantisation step 16)."""
    return synthetic.pair_plain_256(0)


def to_oracle(img: ss2.Image) -> ob.Image:
    f = img.format
    of = ob.Format(*[getattr(f, n) for n, _ in f._fields_])
    return ob.Image(img.width, img.height, of, img.data)


def oracle_compute(o: ss2.Image, d: ss2.Image, background=0.5, chroma_filter=0, precision=32,
                   blur=0):
    return ob.compute(to_oracle(o), to_oracle(d), background, chroma_filter, precision, blur)


def feature_mismatch(actual: np.ndarray, expected: np.ndarray, rtol=FEATURE_RTOL,
                     atol=FEATURE_ATOL):
    """(index, actual, expected) of every feature outside tolerance, and of
    every feature whose expected value is exactly 0 (pruned) but not 0."""
    a = np.asarray(actual, dtype=np.float64).reshape(-1)
    e = np.asarray(expected, dtype=np.float64).reshape(-1)
    bad = []
    for i, (x, y) in enumerate(zip(a, e)):
        if y == 0.0:
            if x != 0.0 and abs(x) > atol:
                bad.append((i, x, y))
        elif not (abs(x - y) <= rtol * abs(y) + atol) or not math.isfinite(x):
            bad.append((i, x, y))
    return bad


def pruned_mask(scales: int) -> np.ndarray:
    """[scales, 18] True where the (channel, scale) pair is pruned."""
    m = np.zeros((scales, 18), dtype=bool)
    for s in range(scales):
        for c in range(3):
            if ob.channel_pruned(c, s, scales):
                m[s, c * 2:c * 2 + 2] = True
                m[s, 6 + c * 4:6 + c * 4 + 4] = True
    return m
