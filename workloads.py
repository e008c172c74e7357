"""Seeded synthetic image pairs with the shapes, formats and distortions of
the benchmark workloads. No corpus ships with the reference for this path
(its bench pairs are ffmpeg testsrc2 renders that are not in the repository),
so these stand in for it.

Textures: per channel, a sum of 8 plane waves (random orientation and phase,
period uniform in [4, 64] px) plus a linear gradient, min-max scaled to
0..255. Distortions: Gaussian noise, Gaussian blur, or 8x8 block
quantisation. The block quantisation keeps every pixel's offset from its
8x8 block mean and rounds the block mean itself to a multiple of the step
(a DC-only quantiser), so it produces blocking without flattening texture.

10-bit 4:2:0 inputs are BT.709 Y'CbCr in limited range (Y 64..940,
C 64..960): the RGB texture's normalised code values go through the BT.709
matrix, chroma is the mean of each 2x2 block. 4:2:0 needs even sizes (the
reference rejects odd ones, src/input.cc:176-179), so odd sizes drawn for
those pairs are rounded up to even; odd geometries are exercised with 8-bit
RGB pairs instead.

This module is numpy only: it loads no native code, so the CPU reference
arm of the benchmark and the CUDA arm draw the same pixels without the CPU
arm touching the CUDA library. Images come back as `Planar` records (size,
format kind, packed bytes in the reference's plane layout); the tests and
the benchmark wrap them in the image type of whichever scorer they call.
"""

from __future__ import annotations

import math
from typing import NamedTuple

import numpy as np

try:  # scipy is in the image; only the blur distortion needs it
    from scipy.ndimage import gaussian_filter
except Exception:  # pragma: no cover
    gaussian_filter = None


# vqm::ImageFormat (include/vqm_image.h:325-337) as its 12 byte fields: type,
# family, alpha, range, matrix, transfer, primaries, chroma_location,
# subsample_w, subsample_h, depth, reserved.
FORMAT_FIELDS = {
    # 8-bit sRGB planar RGB, full range, BT.709 primaries.
    "srgb8": (0, 1, 0, 1, 0, 13, 1, 0, 0, 0, 0, 0),
    # 10-bit 4:2:0 Y'CbCr, BT.709 matrix, transfer and primaries, limited
    # range, Word samples, left chroma siting.
    "yuv420p10": (1, 2, 0, 0, 1, 1, 1, 0, 1, 1, 10, 0),
}


class Planar(NamedTuple):
    """One packed image: planes back to back, each starting on a 4-byte
    boundary (src/input.cc:114-145)."""

    width: int
    height: int
    kind: str          # a key of FORMAT_FIELDS
    data: np.ndarray   # uint8


def plane_offsets(kind: str, w: int, h: int):
    """[(offset, width, height, sample bytes)] of the Y/R, U/G, V/B planes and
    the total byte count (the reference's RequiredBytes)."""
    sb, (cw, ch) = (1, (w, h)) if kind == "srgb8" else (2, (w >> 1, h >> 1))
    planes, cursor = [], 0
    for p in range(3):
        pw, ph = (w, h) if p == 0 else (cw, ch)
        planes.append((cursor, pw, ph, sb))
        cursor = (cursor + pw * ph * sb + 3) // 4 * 4
    return planes, cursor


def _waves(w: int, h: int, rng: np.random.Generator) -> np.ndarray:
    x = np.arange(w, dtype=np.float64)
    y = np.arange(h, dtype=np.float64)
    out = np.zeros((h, w), dtype=np.float32)
    for _ in range(8):
        theta = rng.uniform(0, math.pi)
        period = rng.uniform(4, 64)
        phase = rng.uniform(0, 2 * math.pi)
        amp = rng.uniform(0.3, 1.0)
        k = 2 * math.pi / period
        a = k * math.cos(theta) * x            # along x
        b = k * math.sin(theta) * y + phase    # along y
        # sin(a + b) = sin a cos b + cos a sin b, as two outer products.
        sa, ca = (amp * np.sin(a)).astype(np.float32), (amp * np.cos(a)).astype(np.float32)
        out += np.outer(np.cos(b).astype(np.float32), sa)
        out += np.outer(np.sin(b).astype(np.float32), ca)
    gx, gy = rng.uniform(-1, 1, size=2)
    g = rng.uniform(1, 4)
    out += (g * gx * x / max(w - 1, 1)).astype(np.float32)[None, :]
    out += (g * gy * y / max(h - 1, 1)).astype(np.float32)[:, None]
    return out


def texture(w: int, h: int, rng: np.random.Generator, offset=(0, 0)) -> np.ndarray:
    """[3, h, w] float64 in 0..255. `offset` shifts the texture (video)."""
    ox, oy = offset
    planes = []
    for _ in range(3):
        big = _waves(w + ox, h + oy, rng)[oy:, ox:]
        lo, hi = float(big.min()), float(big.max())
        planes.append((big - lo) * np.float32(255.0 / max(hi - lo, 1e-9)))
    return np.stack(planes)


def add_rectangles(img: np.ndarray, rng: np.random.Generator, count: int = 32) -> np.ndarray:
    _, h, w = img.shape
    img = img.copy()
    for _ in range(count):
        rw = int(rng.integers(max(2, w // 40), max(3, w // 6)))
        rh = int(rng.integers(max(2, h // 40), max(3, h // 6)))
        x0 = int(rng.integers(0, max(1, w - rw)))
        y0 = int(rng.integers(0, max(1, h - rh)))
        img[:, y0:y0 + rh, x0:x0 + rw] = rng.uniform(0, 255, size=3)[:, None, None]
    return img


def block_quantise(img: np.ndarray, step: float, block: int = 8) -> np.ndarray:
    """Round each 8x8 block mean to a multiple of `step`, keep the residual."""
    c, h, w = img.shape
    hp, wp = (h + block - 1) // block * block, (w + block - 1) // block * block
    pad = np.pad(img, ((0, 0), (0, hp - h), (0, wp - w)), mode="edge")
    blocks = pad.reshape(c, hp // block, block, wp // block, block)
    mean = blocks.mean(axis=(2, 4), keepdims=True)
    q = blocks - mean + step * np.round(mean / step)
    return q.reshape(c, hp, wp)[:, :h, :w]


def blur(img: np.ndarray, sigma: float) -> np.ndarray:
    if gaussian_filter is None:
        raise RuntimeError("scipy is needed for the blur distortion")
    return np.stack([gaussian_filter(p, sigma, mode="nearest") for p in img])


def to_u8(img: np.ndarray) -> np.ndarray:
    return np.clip(np.rint(img), 0, 255).astype(np.uint8)


def rgb8_image(planes_u8: np.ndarray) -> Planar:
    _, h, w = planes_u8.shape
    layout, total = plane_offsets("srgb8", w, h)
    data = np.zeros(total, dtype=np.uint8)
    for p in range(3):
        off = layout[p][0]
        data[off:off + w * h] = planes_u8[p].reshape(-1)
    return Planar(w, h, "srgb8", data)


def yuv420_10bit_image(rgb: np.ndarray) -> Planar:
    """RGB code values (0..255 floats) -> BT.709 limited 10-bit 4:2:0."""
    _, h, w = rgb.shape
    if w % 2 or h % 2:
        raise ValueError("4:2:0 needs even dimensions")
    r, g, b = (np.clip(rgb, 0, 255) / 255.0)
    kr, kb = 0.2126, 0.0722
    kg = 1 - kr - kb
    y = kr * r + kg * g + kb * b
    cb = (b - y) / (2 - 2 * kb)
    cr = (r - y) / (2 - 2 * kr)

    def sub(p):
        return p.reshape(h // 2, 2, w // 2, 2).mean(axis=(1, 3))

    yc = np.clip(np.rint(64 + 876 * y), 64, 940)
    cbc = np.clip(np.rint(512 + 896 * sub(cb)), 64, 960)
    crc = np.clip(np.rint(512 + 896 * sub(cr)), 64, 960)
    layout, total = plane_offsets("yuv420p10", w, h)
    data = np.zeros(total, dtype=np.uint8)
    for p, arr in enumerate((yc, cbc, crc)):
        off, pw, ph, _ = layout[p]
        data[off:off + pw * ph * 2] = arr.astype("<u2").reshape(-1).view(np.uint8)
    return Planar(w, h, "yuv420p10", data)


# --- workloads --------------------------------------------------------------


def pair_plain_256(seed: int = 0):
    """One 256x256 8-bit sRGB pair: noise sigma 4, then 8x8 quantisation
    step 16, clipped to 8 bits."""
    rng = np.random.default_rng(seed)
    ref = texture(256, 256, rng)
    dist = ref + rng.normal(0, 4, size=ref.shape)
    dist = block_quantise(dist, 16)
    return rgb8_image(to_u8(ref)), rgb8_image(to_u8(dist))


def distort(ref: np.ndarray, rng: np.random.Generator) -> tuple[np.ndarray, str]:
    kind = int(rng.integers(0, 3))
    if kind == 0:
        s = rng.uniform(1, 8)
        return ref + rng.normal(0, s, size=ref.shape).astype(np.float32), f"noise{s:.2f}"
    if kind == 1:
        s = rng.uniform(0.5, 3)
        return blur(ref, s), f"blur{s:.2f}"
    s = rng.uniform(4, 32)
    return block_quantise(ref, s), f"quant{s:.2f}"


def rgb_pair(w: int, h: int, seed: int):
    """8-bit sRGB pair: texture + 32 rectangles, one random distortion."""
    rng = np.random.default_rng(seed)
    ref = add_rectangles(texture(w, h, rng), rng)
    dist, kind = distort(ref, rng)
    return rgb8_image(to_u8(ref)), rgb8_image(to_u8(dist)), kind


def yuv_pair(w: int, h: int, seed: int):
    """10-bit 4:2:0 pair of the same content model (sizes rounded to even)."""
    w += w % 2
    h += h % 2
    rng = np.random.default_rng(seed)
    ref = add_rectangles(texture(w, h, rng), rng)
    dist, kind = distort(ref, rng)
    return yuv420_10bit_image(ref), yuv420_10bit_image(np.clip(dist, 0, 255)), kind


def plain_1080p(count: int = 64, seed0: int = 1000, width: int = 1920, height: int = 1080):
    return [rgb_pair(width, height, seed0 + i)[:2] for i in range(count)]


def uneven_jobs(count: int = 128, seed0: int = 2000, odd_rgb: int = 8):
    """The uneven batch's draw as (kind, width, height, seed) jobs: `count`
    10-bit 4:2:0 pairs of sizes W in [320, 3840], H in [180, 2160] (rounded
    up to even when generated), then `odd_rgb` 8-bit RGB pairs keeping odd
    sizes. `make_pair` turns a job into its pair, so the jobs can be
    generated in parallel."""
    rng = np.random.default_rng(seed0)
    jobs = [("yuv", int(rng.integers(320, 3841)), int(rng.integers(180, 2161)), seed0 + 1 + i)
            for i in range(count)]
    jobs += [("rgb", int(rng.integers(320, 3841)) | 1, int(rng.integers(180, 2161)) | 1,
              seed0 + 10_000 + i) for i in range(odd_rgb)]
    return jobs


def make_pair(job):
    """(kind, width, height, seed) -> (original, distorted) Planar pair."""
    kind, w, h, seed = job
    make = yuv_pair if kind == "yuv" else rgb_pair
    return make(w, h, seed)[:2]


def uneven_batch(count: int = 128, seed0: int = 2000, odd_rgb: int = 8):
    """The uneven batch's pairs in draw order (see `uneven_jobs`)."""
    return [make_pair(j) for j in uneven_jobs(count, seed0, odd_rgb)]


def video_offsets(count: int, seed: int):
    """Per-frame (x, y) offsets of the translating reference: 1-3 px right
    and 0-1 px down per frame."""
    rng = np.random.default_rng(seed)
    total_shift = 3 * count + 4
    x = y = 0
    out = []
    for _ in range(count):
        x += int(rng.integers(1, 4))
        y += int(rng.integers(0, 2))
        out.append((min(x, total_shift - 1), min(y, total_shift - 1)))
    return out


def video_base(count: int, width: int, height: int, seed: int) -> np.ndarray:
    """The texture the reference stream is cut from (large enough for every
    frame's offset)."""
    total_shift = 3 * count + 4
    base_rng = np.random.default_rng(seed + 1)
    return add_rectangles(texture(width + total_shift, height + total_shift, base_rng), base_rng)


def video_frame(f: int, count: int, width: int, height: int, seed: int, base=None,
                offsets=None):
    """Frame pair f of the clip: the reference is the base texture at the
    frame's offset; the distorted frame is 8x8 quantised with a step drifting
    8 -> 48 over the clip plus noise sigma 2 (8-bit units, seeded per frame).
    Both as 10-bit 4:2:0 images. Frames are independent of each other, so a
    clip can be generated in parallel."""
    base = video_base(count, width, height, seed) if base is None else base
    x, y = (offsets or video_offsets(count, seed))[f]
    ref = base[:, y:y + height, x:x + width]
    step = 8 + (48 - 8) * f / max(count - 1, 1)
    rng = np.random.default_rng(seed + 10 + f)
    dist = block_quantise(ref, step) + rng.normal(0, 2, size=ref.shape).astype(np.float32)
    return yuv420_10bit_image(ref), yuv420_10bit_image(np.clip(dist, 0, 255))


def video_frames(count: int = 240, width: int = 3840, height: int = 2160, seed: int = 4000):
    """The clip's frame pairs in order (see video_frame)."""
    base = video_base(count, width, height, seed)
    offsets = video_offsets(count, seed)
    for f in range(count):
        yield video_frame(f, count, width, height, seed, base, offsets)
