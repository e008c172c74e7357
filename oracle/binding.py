"""ctypes binding of the CPU oracle -- TEST INFRASTRUCTURE ONLY.

Loaded by the tests, by ``__graft_entry__.smoke()`` and by the CPU-baseline
leg of ``bench.py``, always as the checker. The CUDA scorer never imports it.

``liboracle_ss2.so`` restates VQM's SSIMULACRA 2.1 arithmetic (see
``ss2_oracle.h``); ``_ref/libvqm_ref.so`` is the reference's own score.cc and
input.cc compiled from the reference checkout, used to pin the restatement.
"""

from __future__ import annotations

import ctypes
import os
import subprocess
from dataclasses import dataclass

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "liboracle_ss2.so")
REF_PATH = os.path.join(HERE, "_ref", "libvqm_ref.so")
# The reference checkout whose host sources `make ref` compiles into
# _ref/libvqm_ref.so; None when the environment does not name one (the GPU
# box only uses the prebuilt library).
REFERENCE_CHECKOUT = os.environ.get("VQM_REFERENCE") or None


class Format(ctypes.Structure):
    """vqm::ImageFormat (include/vqm_image.h:325-337) as 12 bytes."""

    _fields_ = [
        ("type", ctypes.c_uint8),
        ("family", ctypes.c_uint8),
        ("alpha", ctypes.c_uint8),
        ("range", ctypes.c_uint8),
        ("matrix", ctypes.c_uint8),
        ("transfer", ctypes.c_uint8),
        ("primaries", ctypes.c_uint8),
        ("chroma_location", ctypes.c_uint8),
        ("subsample_w", ctypes.c_uint8),
        ("subsample_h", ctypes.c_uint8),
        ("depth", ctypes.c_uint8),
        ("reserved", ctypes.c_uint8),
    ]

    def as_bytes(self) -> bytes:
        return bytes(self)


class _Image(ctypes.Structure):
    _fields_ = [
        ("width", ctypes.c_uint32),
        ("height", ctypes.c_uint32),
        ("format", Format),
        ("data", ctypes.c_void_p),
        ("bytes", ctypes.c_size_t),
    ]


def build(reference: bool = True, checkout: str | None = None) -> None:
    """Compile the oracle and, when a reference checkout is given (argument
    or VQM_REFERENCE), the reference pins."""
    subprocess.run(["make", "-s", "-C", HERE], check=True)
    checkout = checkout or REFERENCE_CHECKOUT
    if reference and checkout and os.path.isdir(checkout):
        subprocess.run(["make", "-s", "-C", HERE, "ref", f"VQM_REFERENCE={checkout}"], check=True)


_lib = None
_ref = None


def lib() -> ctypes.CDLL:
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            build(reference=False)
        _lib = ctypes.CDLL(LIB_PATH)
        _lib.ss2o_last_error.restype = ctypes.c_char_p
    return _lib


def ref() -> ctypes.CDLL | None:
    """The reference's own score.cc/input.cc, or None when it was not built."""
    global _ref
    if _ref is None:
        if not os.path.exists(REF_PATH) and REFERENCE_CHECKOUT:
            build(reference=True)
        if not os.path.exists(REF_PATH):
            return None
        _ref = ctypes.CDLL(REF_PATH)
        _ref.vqmref_last_error.restype = ctypes.c_char_p
    return _ref


@dataclass
class Image:
    """A packed image in vqm::Image's layout: width, height, format, bytes."""

    width: int
    height: int
    format: Format
    data: np.ndarray  # uint8, RequiredBytes long

    def c(self) -> _Image:
        buf = np.ascontiguousarray(self.data, dtype=np.uint8)
        self.data = buf
        return _Image(self.width, self.height, self.format,
                      buf.ctypes.data_as(ctypes.c_void_p), buf.nbytes)


class OracleError(ValueError):
    pass


def _check(status: int) -> None:
    if status != 0:
        raise OracleError(lib().ss2o_last_error().decode())


def compute(original: Image, distorted: Image, background: float = 0.5,
            chroma_filter: int = 0, precision: int = 32, blur: int = 0):
    """Returns (norms[scales, 18], score) of one pair. blur: 0 VQM's sampled
    Gaussian, 1 the recursive Gaussian."""
    norms = np.zeros(108, dtype=np.float64)
    scales = ctypes.c_uint32()
    score = ctypes.c_double()
    a, b = original.c(), distorted.c()
    _check(lib().ss2o_compute(ctypes.byref(a), ctypes.byref(b),
                              ctypes.c_float(background), chroma_filter,
                              precision, blur,
                              norms.ctypes.data_as(ctypes.c_void_p),
                              ctypes.byref(scales), ctypes.byref(score)))
    return norms[: 18 * scales.value].reshape(scales.value, 18), score.value


def compute_many(pairs, background: float = 0.5, chroma_filter: int = 0,
                 precision: int = 32, threads: int | None = None, blur: int = 0):
    """Scores a list of (original, distorted) on host threads; returns
    (norms[n, 108], scales[n], scores[n])."""
    n = len(pairs)
    threads = threads or os.cpu_count() or 1
    origs = (_Image * n)(*[p[0].c() for p in pairs])
    dists = (_Image * n)(*[p[1].c() for p in pairs])
    norms = np.zeros((n, 108), dtype=np.float64)
    scales = np.zeros(n, dtype=np.uint32)
    scores = np.zeros(n, dtype=np.float64)
    _check(lib().ss2o_compute_many(
        n, origs, dists, ctypes.c_float(background), chroma_filter, precision,
        blur, threads, norms.ctypes.data_as(ctypes.c_void_p),
        scales.ctypes.data_as(ctypes.c_void_p),
        scores.ctypes.data_as(ctypes.c_void_p)))
    return norms, scales, scores


def plan_scales(width: int, height: int):
    sizes = (ctypes.c_uint32 * 12)()
    n = lib().ss2o_plan_scales(width, height, sizes)
    if n < 0:
        raise OracleError(lib().ss2o_last_error().decode())
    return [(sizes[2 * i], sizes[2 * i + 1]) for i in range(n)]


def gaussian() -> np.ndarray:
    taps = np.zeros(13, dtype=np.float32)
    lib().ss2o_gaussian(taps.ctypes.data_as(ctypes.c_void_p))
    return taps


def recursive_gaussian():
    """(radius, freqs[3], beta[3], taps[13] in double) of the recursive
    Gaussian, sigma 1.5."""
    radius = ctypes.c_int()
    freqs, beta, taps = np.zeros(3), np.zeros(3), np.zeros(13)
    lib().ss2o_recursive_gaussian(ctypes.byref(radius), freqs.ctypes.data_as(ctypes.c_void_p),
                                  beta.ctypes.data_as(ctypes.c_void_p),
                                  taps.ctypes.data_as(ctypes.c_void_p))
    return radius.value, freqs, beta, taps


def blur_plane(plane: np.ndarray, blur: int = 0, precision: int = 64) -> np.ndarray:
    """One plane blurred, zero padded (precision 64: double, the recursive
    mode by its recursion; 32: float, the 13-tap passes)."""
    src = np.ascontiguousarray(plane, dtype=np.float64)
    out = np.zeros_like(src)
    h, w = src.shape
    _check(lib().ss2o_blur_plane(blur, precision, src.ctypes.data_as(ctypes.c_void_p), w, h,
                                 out.ctypes.data_as(ctypes.c_void_p)))
    return out


def channel_pruned(channel: int, scale: int, scales: int) -> bool:
    return bool(lib().ss2o_channel_pruned(channel, scale, scales))


def score(norms: np.ndarray, scales: int) -> float:
    flat = np.asarray(norms, dtype=np.float64).reshape(-1)
    buf = np.zeros(max(108, flat.size), dtype=np.float64)
    buf[: flat.size] = flat
    out = ctypes.c_double()
    _check(lib().ss2o_score(buf.ctypes.data_as(ctypes.c_void_p), scales,
                            ctypes.byref(out)))
    return out.value


def required_bytes(fmt: Format, width: int, height: int) -> int:
    out = ctypes.c_size_t()
    _check(lib().ss2o_required_bytes(ctypes.byref(fmt), width, height,
                                     ctypes.byref(out)))
    return out.value


def source_desc(fmt: Format, chroma_filter: int = 0) -> np.ndarray:
    words = np.zeros(44, dtype=np.uint32)
    _check(lib().ss2o_source_desc(ctypes.byref(fmt), chroma_filter,
                                  words.ctypes.data_as(ctypes.c_void_p)))
    return words


def pyramid(image: Image, background: float = 0.5, chroma_filter: int = 0):
    """The FP32 XYB pyramid: list of arrays [3, H_l, W_l] (pruned = NaN)."""
    count = ctypes.c_size_t()
    img = image.c()
    _check(lib().ss2o_pyramid(ctypes.byref(img), ctypes.c_float(background),
                              chroma_filter, None, 0, ctypes.byref(count)))
    out = np.zeros(count.value, dtype=np.float32)
    _check(lib().ss2o_pyramid(ctypes.byref(img), ctypes.c_float(background),
                              chroma_filter,
                              out.ctypes.data_as(ctypes.c_void_p), out.size,
                              ctypes.byref(count)))
    levels, at = [], 0
    for (w, h) in plan_scales(image.width, image.height):
        n = 3 * w * h
        levels.append(out[at:at + n].reshape(3, h, w))
        at += n
    return levels


def level_sums(original: Image, distorted: Image, background: float = 0.5,
               chroma_filter: int = 0) -> np.ndarray:
    sums = np.zeros(108, dtype=np.float32)
    scales = ctypes.c_uint32()
    a, b = original.c(), distorted.c()
    _check(lib().ss2o_level_sums(ctypes.byref(a), ctypes.byref(b),
                                 ctypes.c_float(background), chroma_filter,
                                 sums.ctypes.data_as(ctypes.c_void_p),
                                 ctypes.byref(scales)))
    return sums[: 18 * scales.value].reshape(scales.value, 18)
