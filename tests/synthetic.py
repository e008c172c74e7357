"""The benchmark workloads' seeded pairs (`workloads.py`, numpy only) as
images of the CUDA scorer's Python binding, for the tests."""

from __future__ import annotations

import workloads
from workloads import texture  # noqa: F401  (re-exported for the tests)
from vqm_b200 import ss2


def image(p: workloads.Planar) -> ss2.Image:
    """A Planar record as an ss2.Image (same packed bytes)."""
    fmt = ss2.ImageFormat.from_buffer_copy(bytes(workloads.FORMAT_FIELDS[p.kind]))
    return ss2.Image(p.width, p.height, fmt, p.data)


def rgb_pair(w: int, h: int, seed: int):
    o, d, kind = workloads.rgb_pair(w, h, seed)
    return image(o), image(d), kind


def yuv_pair(w: int, h: int, seed: int):
    o, d, kind = workloads.yuv_pair(w, h, seed)
    return image(o), image(d), kind


def pair_plain_256(seed: int = 0):
    o, d = workloads.pair_plain_256(seed)
    return image(o), image(d)


def make_pair(job):
    o, d = workloads.make_pair(job)
    return image(o), image(d)


def yuv420_10bit_image(rgb):
    return image(workloads.yuv420_10bit_image(rgb))


def rgb8_image(planes_u8):
    return image(workloads.rgb8_image(planes_u8))
