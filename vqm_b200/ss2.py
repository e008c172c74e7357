"""SSIMULACRA 2.1 on B200: Python mirror of VQM's metric API over the C ABI.

The classes follow the reference's C++ interface (include/ssimulacra2.h,
include/vqm_pool.h) name for name: ``Ssimulacra2Pipeline`` with
``compute`` / ``submit`` / ``finish`` / ``upload`` / ``release`` /
``allocate_image`` / ``map_image`` / ``get_memory_usage``,
``Ssimulacra2Result.score()``, and ``Ssimulacra2Pool.compute_many`` /
``score_many``. The reference's exception types map to ``InvalidArgument``
(std::invalid_argument, a ValueError), ``LogicError`` (std::logic_error),
``CudaError`` (std::runtime_error) and ``OverflowError``.

Every call goes through libvqm_ss2.so (include/vqm_cu_ss2.h). There is no
CPU fallback: without the compiled extension, importing this module fails.
"""

from __future__ import annotations

import collections
import ctypes
import os
from dataclasses import dataclass, field
from typing import Iterable, Sequence

import numpy as np

_LIB_PATH = os.path.join(os.path.dirname(os.path.abspath(__file__)), "libvqm_ss2.so")

if not os.path.exists(_LIB_PATH):
    raise ImportError(
        f"vqm_b200: the CUDA extension {_LIB_PATH} is not built; run "
        "`python -m vqm_b200.build` (needs nvcc). There is no CPU fallback.")

_lib = ctypes.CDLL(_LIB_PATH)

# ---------------------------------------------------------------------------
# Enums (include/vqm_image.h:243-316, zimg numeric values)
# ---------------------------------------------------------------------------


class PixelType:
    Byte, Word, Half, Float = 0, 1, 2, 3


class PixelRange:
    Limited, Full = 0, 1


class ColorFamily:
    Grey, Rgb, Yuv = 0, 1, 2


class AlphaType:
    None_, Straight, Premultiplied = 0, 1, 2


class ChromaLocation:
    Left, Center, TopLeft, Top, BottomLeft, Bottom = 0, 1, 2, 3, 4, 5


class MatrixCoefficients:
    Rgb, Bt709, Unspecified = 0, 1, 2
    Fcc, Bt470Bg, St170M, St240M, YCgCo = 4, 5, 6, 7, 8
    Bt2020Ncl, Bt2020Cl, St2085YDzDx = 9, 10, 11
    ChromaticityDerivedNcl, ChromaticityDerivedCl, Bt2100ICtCp = 12, 13, 14
    St2128IptC2, YCgCoRe, YCgCoRo = 15, 16, 17


class TransferCharacteristics:
    Bt709, Unspecified, Bt470M, Bt470Bg, Bt601, St240M, Linear = 1, 2, 4, 5, 6, 7, 8
    Log100, Log316, Iec61966_2_4, Bt1361, Srgb = 9, 10, 11, 12, 13
    Bt2020_10, Bt2020_12, St2084, St428, AribB67 = 14, 15, 16, 17, 18


class ColorPrimaries:
    Bt709, Unspecified, Bt470M, Bt470Bg, St170M, St240M, Film = 1, 2, 4, 5, 6, 7, 8
    Bt2020, St428, St431_2, St432_1, Ebu3213E = 9, 10, 11, 12, 22


class ChromaFilter:
    Bilinear, Bicubic, Lanczos = 0, 1, 2


class Ssimulacra2Blur:
    """The blur (no counterpart in VQM's config). SAMPLED: VQM's 13-tap
    sampled Gaussian, sigma 1.5 (pipeline.cc:274-291), VQM's scores.
    RECURSIVE (opt-in): the third-order recursive Gaussian, sigma 1.5, of
    Cloudinary's ssimulacra2, which VQM replaced on purpose
    (docs/divergence.md:22); its scores follow that filter, not VQM."""
    SAMPLED, RECURSIVE = 0, 1


# ---------------------------------------------------------------------------
# C structs (include/vqm_cu_ss2.h)
# ---------------------------------------------------------------------------


class MemoryPolicy:
    """vqm::MemoryPolicy (vqm_memory_types.h:12-14)."""
    AUTOMATIC, DIRECT, STAGED = 0, 1, 2


class ImageFormat(ctypes.Structure):
    """vqm::ImageFormat; the defaults are the reference's (8-bit needs type)."""

    _fields_ = [(n, ctypes.c_uint8) for n in (
        "type", "family", "alpha", "range", "matrix", "transfer", "primaries",
        "chroma_location", "subsample_w", "subsample_h", "depth", "reserved")]

    def __init__(self, type=PixelType.Float, family=ColorFamily.Rgb,
                 alpha=AlphaType.None_, range=PixelRange.Full,
                 matrix=MatrixCoefficients.Rgb,
                 transfer=TransferCharacteristics.Srgb,
                 primaries=ColorPrimaries.Bt709,
                 chroma_location=ChromaLocation.Left, subsample_w=0,
                 subsample_h=0, depth=0):
        super().__init__(type, family, alpha, range, matrix, transfer,
                         primaries, chroma_location, subsample_w, subsample_h,
                         depth, 0)

    def copy(self, **changes) -> "ImageFormat":
        values = {n: getattr(self, n) for n, _ in self._fields_ if n != "reserved"}
        values.update(changes)
        return ImageFormat(**values)


def srgb8_format() -> ImageFormat:
    """The format the reference's CLI decoders pin for 8-bit sRGB input."""
    return ImageFormat(type=PixelType.Byte)


def yuv420_10bit_bt709_format() -> ImageFormat:
    """10-bit 4:2:0 BT.709 limited range, Word samples, left chroma siting."""
    return ImageFormat(type=PixelType.Word, family=ColorFamily.Yuv,
                       range=PixelRange.Limited, matrix=MatrixCoefficients.Bt709,
                       transfer=TransferCharacteristics.Bt709,
                       primaries=ColorPrimaries.Bt709, subsample_w=1,
                       subsample_h=1, depth=10)


class _CImage(ctypes.Structure):
    _fields_ = [
        ("width", ctypes.c_uint32),
        ("height", ctypes.c_uint32),
        ("format", ImageFormat),
        ("memory", ctypes.c_int32),
        ("planes", ctypes.c_void_p * 4),
        ("strides", ctypes.c_size_t * 4),
    ]


class _Config(ctypes.Structure):
    _fields_ = [
        ("width", ctypes.c_uint32),
        ("height", ctypes.c_uint32),
        ("gpu_resident_images", ctypes.c_uint32),
        ("half_planes", ctypes.c_uint32),
        ("chroma_filter", ctypes.c_uint32),
        ("streaming_inputs", ctypes.c_uint32),
        ("input_bytes", ctypes.c_uint64),
        ("device", ctypes.c_int32),
        ("blur", ctypes.c_uint32),
        ("memory_policy", ctypes.c_uint32),
    ]


class _BatchConfig(ctypes.Structure):
    _fields_ = [
        ("max_pixels", ctypes.c_uint64),
        ("max_pairs", ctypes.c_uint32),
        ("chroma_filter", ctypes.c_uint32),
        ("device", ctypes.c_int32),
        ("tile_w", ctypes.c_uint32),
        ("tile_h", ctypes.c_uint32),
        ("variant", ctypes.c_uint32),
        ("half_planes", ctypes.c_uint32),
        ("blur", ctypes.c_uint32),
    ]


class _ServerConfig(ctypes.Structure):
    _fields_ = [
        ("memory_budget", ctypes.c_uint64),
        ("workers", ctypes.c_uint32),
        ("max_batch_pairs", ctypes.c_uint32),
        ("chroma_filter", ctypes.c_uint32),
        ("device", ctypes.c_int32),
        ("variant", ctypes.c_uint32),
        ("blur", ctypes.c_uint32),
    ]


class ServerStats(ctypes.Structure):
    _fields_ = [(n, ctypes.c_uint64) for n in (
        "submitted", "completed", "failed", "batches", "largest_batch", "bytes_in_flight",
        "peak_bytes", "queued", "budget_bytes", "device_bytes", "peak_device_bytes", "trims")]


class MemoryUsage(ctypes.Structure):
    _fields_ = [(n, ctypes.c_uint64) for n in (
        "pyramid_bytes", "resident_bytes", "input_bytes", "scratch_bytes",
        "total_bytes", "host_bytes")] + [("uses_staging", ctypes.c_uint32),
                                        ("reserved", ctypes.c_uint32)]


_P = ctypes.c_void_p
_U64P = ctypes.POINTER(ctypes.c_uint64)
_SIGS = {
    "vqm_cu_last_error": ([], ctypes.c_char_p),
    "vqm_cu_version": ([], ctypes.c_uint32),
    "vqm_cu_required_bytes": ([_P, ctypes.c_uint32, ctypes.c_uint32, _P], ctypes.c_int),
    "vqm_cu_validate_format": ([_P, ctypes.c_uint32, ctypes.c_uint32, ctypes.c_char_p], ctypes.c_int),
    "vqm_cu_ss2_plan_scales": ([ctypes.c_uint32, ctypes.c_uint32, _P, _P], ctypes.c_int),
    "vqm_cu_ss2_channel_pruned": ([ctypes.c_uint32] * 3 + [_P], ctypes.c_int),
    "vqm_cu_ss2_blur_taps": ([ctypes.c_uint32, _P], ctypes.c_int),
    "vqm_cu_ss2_auto_blur_variant": ([_P, ctypes.c_uint32, ctypes.c_uint32, _P], ctypes.c_int),
    "vqm_cu_ss2_check_cbrt": ([ctypes.c_uint32, ctypes.c_uint32, _P, _P], ctypes.c_int),
    "vqm_cu_ss2_check_division": ([ctypes.c_uint32, ctypes.c_uint32, _P, _P], ctypes.c_int),
    "vqm_cu_ss2_score": ([_P, ctypes.c_uint32, _P], ctypes.c_int),
    "vqm_cu_ss2_source_constants": ([_P, ctypes.c_uint32, _P], ctypes.c_int),
    "vqm_cu_ss2_create": ([_P, _P], ctypes.c_int),
    "vqm_cu_ss2_destroy": ([_P], ctypes.c_int),
    "vqm_cu_ss2_set_stream": ([_P, _P], ctypes.c_int),
    "vqm_cu_ss2_get_stream": ([_P, _P], ctypes.c_int),
    "vqm_cu_ss2_set_graphs": ([_P, ctypes.c_int], ctypes.c_int),
    "vqm_cu_ss2_reference_reuses": ([_P, _P], ctypes.c_int),
    "vqm_cu_ss2_in_flight": ([_P, _P], ctypes.c_int),
    "vqm_cu_device_count": ([_P], ctypes.c_int),
    "vqm_cu_device_info": ([ctypes.c_uint32, ctypes.c_char_p, ctypes.c_size_t, _P, _P],
                           ctypes.c_int),
    "vqm_cu_set_default_device": ([_P], ctypes.c_int),
    "vqm_cu_ss2_submit": ([_P, _P, _P, ctypes.c_float, _P], ctypes.c_int),
    "vqm_cu_ss2_submit_resident": ([_P, ctypes.c_uint64, ctypes.c_uint64, ctypes.c_float, _P], ctypes.c_int),
    "vqm_cu_ss2_submit_resident_image": ([_P, ctypes.c_uint64, _P, ctypes.c_float, _P], ctypes.c_int),
    "vqm_cu_ss2_submit_buffers": ([_P, ctypes.c_uint64, ctypes.c_uint64, ctypes.c_float, _P], ctypes.c_int),
    "vqm_cu_ss2_submit_sync": ([_P, _P, _P, _P, ctypes.c_uint32, _P, ctypes.c_uint32, ctypes.c_float, _P], ctypes.c_int),
    "vqm_cu_ss2_finish": ([_P, ctypes.c_uint64, _P, _P], ctypes.c_int),
    "vqm_cu_ss2_compute": ([_P, _P, _P, ctypes.c_float, _P, _P, _P], ctypes.c_int),
    "vqm_cu_ss2_upload": ([_P, _P, _P], ctypes.c_int),
    "vqm_cu_ss2_release": ([_P, ctypes.c_uint64], ctypes.c_int),
    "vqm_cu_ss2_allocate_image": ([_P, _P, _P, _P], ctypes.c_int),
    "vqm_cu_ss2_map_image": ([_P, ctypes.c_uint64, _P], ctypes.c_int),
    "vqm_cu_ss2_release_image": ([_P, ctypes.c_uint64], ctypes.c_int),
    "vqm_cu_ss2_memory_usage": ([_P, _P], ctypes.c_int),
    "vqm_cu_ss2_debug_plane": ([_P, ctypes.c_uint32, ctypes.c_uint32, ctypes.c_uint32, _P], ctypes.c_int),
    "vqm_cu_ss2_compute_noalloc": ([_P, _P, ctypes.c_float, ctypes.c_uint32, _P, _P], ctypes.c_int),
    "vqm_cu_ss2_batch_create": ([_P, _P], ctypes.c_int),
    "vqm_cu_ss2_batch_destroy": ([_P], ctypes.c_int),
    "vqm_cu_ss2_batch_set_stream": ([_P, _P], ctypes.c_int),
    "vqm_cu_ss2_batch_submit": ([_P, ctypes.c_uint32, _P, _P, ctypes.c_float, _P], ctypes.c_int),
    "vqm_cu_ss2_batch_submit_borrowed": ([_P, ctypes.c_uint32, _P, _P, ctypes.c_float, _P], ctypes.c_int),
    "vqm_cu_ss2_batch_finish": ([_P, ctypes.c_uint64, _P, _P, _P], ctypes.c_int),
    "vqm_cu_ss2_batch_set_timing": ([_P, ctypes.c_int], ctypes.c_int),
    "vqm_cu_ss2_blur_variants": ([_P, _P], ctypes.c_int),
    "vqm_cu_ss2_decode_path": ([_P, ctypes.c_uint32, _P], ctypes.c_int),
    "vqm_cu_ss2_batch_stage_ms": ([_P, _P], ctypes.c_int),
    "vqm_cu_ss2_batch_device_bytes": ([_P, _P], ctypes.c_int),
    "vqm_cu_ss2_batch_device_bytes_after": ([_P, ctypes.c_uint32, _P, _P, _P], ctypes.c_int),
    "vqm_cu_ss2_batch_trim": ([_P], ctypes.c_int),
    "vqm_cu_ss2_batch_compute": ([_P, ctypes.c_uint32, _P, _P, ctypes.c_float, _P, _P, _P], ctypes.c_int),
    "vqm_cu_ss2_server_create": ([_P, _P], ctypes.c_int),
    "vqm_cu_ss2_server_destroy": ([_P], ctypes.c_int),
    "vqm_cu_ss2_server_submit": ([_P, _P, _P, ctypes.c_float, _P], ctypes.c_int),
    "vqm_cu_ss2_server_wait": ([_P, ctypes.c_uint64, ctypes.c_int32, _P, _P, _P, _P], ctypes.c_int),
    "vqm_cu_ss2_server_get_stats": ([_P, _P], ctypes.c_int),
}
for _name, (_args, _res) in _SIGS.items():
    _fn = getattr(_lib, _name)
    _fn.argtypes = _args
    _fn.restype = _res

EXPORTED_SYMBOLS = tuple(_SIGS)


def library_path() -> str:
    return _LIB_PATH


# ---------------------------------------------------------------------------
# Errors
# ---------------------------------------------------------------------------


class InvalidArgument(ValueError):
    """std::invalid_argument."""


class LogicError(RuntimeError):
    """std::logic_error."""


class CudaError(RuntimeError):
    """std::runtime_error: no device, allocation or CUDA failure."""


class Timeout(TimeoutError):
    """A server wait ran out; the request is still pending."""


_ERRORS = {1: InvalidArgument, 2: LogicError, 3: CudaError, 4: OverflowError, 5: Timeout}


def _check(status: int) -> None:
    if status != 0:
        msg = _lib.vqm_cu_last_error().decode()
        raise _ERRORS.get(status, CudaError)(msg)


# ---------------------------------------------------------------------------
# Images
# ---------------------------------------------------------------------------


def required_bytes(fmt: ImageFormat, width: int, height: int) -> int:
    """RequiredBytes (include/vqm_image.h:360-363)."""
    out = ctypes.c_size_t()
    _check(_lib.vqm_cu_required_bytes(ctypes.byref(fmt), width, height, ctypes.byref(out)))
    return out.value


def validate_format(fmt: ImageFormat, width: int, height: int, name: str = "image") -> None:
    _check(_lib.vqm_cu_validate_format(ctypes.byref(fmt), width, height, name.encode()))


def plane_layout(fmt: ImageFormat, width: int, height: int):
    """[(offset, width, height, sample_bytes) or None] for planes 0..3
    (src/input.cc:114-145)."""
    sb = {0: 1, 1: 2, 2: 2, 3: 4}[fmt.type]
    cw, ch = width >> fmt.subsample_w, height >> fmt.subsample_h
    out, cursor = [], 0
    for p in range(4):
        chroma = p in (1, 2)
        present = p == 0 or (chroma and fmt.family != 0) or (p == 3 and fmt.alpha != 0)
        if not present:
            out.append(None)
            continue
        w, h = (cw, ch) if chroma else (width, height)
        out.append((cursor, w, h, sb))
        cursor = (cursor + w * h * sb + 3) // 4 * 4
    return out


@dataclass
class Image:
    """vqm::Image: packed planes (Y/R, U/G, V/B, alpha) in one byte buffer."""

    width: int
    height: int
    format: ImageFormat
    data: np.ndarray

    @property
    def size(self):
        return (self.width, self.height)

    def _c(self) -> _CImage:
        self.data = np.ascontiguousarray(self.data, dtype=np.uint8)
        expected = required_bytes(self.format, self.width, self.height)
        if self.data.nbytes != expected:
            raise InvalidArgument(
                f"image: data size does not match the image format (expected {expected} bytes)")
        c = _CImage(self.width, self.height, self.format, 0)
        base = self.data.ctypes.data
        for p, geo in enumerate(plane_layout(self.format, self.width, self.height)):
            if geo is not None:
                c.planes[p] = base + geo[0]
        return c


def _c_bytes(image) -> bytes:
    """The vqm_cu_image bytes of any image kind."""
    f = getattr(image, "_c_bytes", None)
    return f() if f is not None else bytes(image._c())


@dataclass
class DeviceImage:
    """A caller-owned device buffer (the CUDA counterpart of VulkanBufferView):
    plane device addresses and byte strides (0 = packed rows)."""

    width: int
    height: int
    format: ImageFormat
    planes: Sequence[int]
    strides: Sequence[int] = (0, 0, 0, 0)
    owner: object = None  # keeps the memory alive (e.g. a torch tensor)

    @staticmethod
    def packed(width: int, height: int, fmt: ImageFormat, base_ptr: int, owner=None):
        planes = [0, 0, 0, 0]
        for p, geo in enumerate(plane_layout(fmt, width, height)):
            if geo is not None:
                planes[p] = base_ptr + geo[0]
        return DeviceImage(width, height, fmt, planes, (0, 0, 0, 0), owner)

    def _c_bytes(self) -> bytes:
        # The struct's bytes are kept with the fields they came from, so a
        # buffer scored call after call is converted once (the conversion
        # was a sizeable part of a one-pair call's host time).
        key = (self.width, self.height, bytes(self.format), tuple(self.planes),
               tuple(self.strides))
        cached = self.__dict__.get("_c_cache")
        if cached is None or cached[0] != key:
            c = _CImage(self.width, self.height, self.format, 1)
            for p in range(4):
                c.planes[p] = int(self.planes[p]) if self.planes[p] else None
                c.strides[p] = int(self.strides[p])
            cached = (key, bytes(c))
            self.__dict__["_c_cache"] = cached
        return cached[1]

    def _c(self) -> _CImage:
        return _CImage.from_buffer_copy(self._c_bytes())


@dataclass
class HostImage:
    """vqm::ImageView: separately allocated, optionally padded host planes."""

    width: int
    height: int
    format: ImageFormat
    planes: Sequence[np.ndarray | None]
    strides: Sequence[int] = (0, 0, 0, 0)

    def _c(self) -> _CImage:
        c = _CImage(self.width, self.height, self.format, 0)
        for p in range(4):
            arr = self.planes[p] if p < len(self.planes) else None
            if arr is not None:
                c.planes[p] = arr.ctypes.data
                c.strides[p] = int(self.strides[p])
        return c


# ---------------------------------------------------------------------------
# Results
# ---------------------------------------------------------------------------


@dataclass
class Ssimulacra2Scale:
    """18 norms of one scale (include/ssimulacra2.h:18-25)."""

    avg_ssim: np.ndarray      # [channel * 2 + norm]
    avg_edgediff: np.ndarray  # [channel * 4 + n]: ringing 0, 1; blurring 2, 3


@dataclass
class Ssimulacra2Result:
    norms: np.ndarray  # [scales, 18]
    device_score: float | None = None
    scales: list = field(init=False)

    def __post_init__(self):
        self.scales = [Ssimulacra2Scale(r[:6].copy(), r[6:].copy()) for r in self.norms]

    def score(self) -> float:
        """Ssimulacra2Result::Score (score.cc:118-163), FP64 on the host."""
        return score(self.norms)


def score(norms: np.ndarray) -> float:
    norms = np.asarray(norms, dtype=np.float64)
    scales = norms.shape[0] if norms.ndim == 2 else norms.size // 18
    buf = np.zeros(max(108, norms.size), dtype=np.float64)
    buf[: norms.size] = norms.reshape(-1)
    out = ctypes.c_double()
    _check(_lib.vqm_cu_ss2_score(buf.ctypes.data, scales, ctypes.byref(out)))
    return out.value


def source_constants(fmt: ImageFormat, chroma_filter: int = 0) -> np.ndarray:
    """The 44 SourceDesc words this library derives for `fmt`."""
    words = np.zeros(44, dtype=np.uint32)
    _check(_lib.vqm_cu_ss2_source_constants(ctypes.byref(fmt), chroma_filter, words.ctypes.data))
    return words


def plan_scales(width: int, height: int):
    sizes = (ctypes.c_uint32 * 12)()
    n = ctypes.c_uint32()
    _check(_lib.vqm_cu_ss2_plan_scales(width, height, sizes, ctypes.byref(n)))
    return [(sizes[2 * i], sizes[2 * i + 1]) for i in range(n.value)]


def channel_pruned(channel: int, scale: int, scales: int) -> bool:
    """Ssimulacra2ChannelPruned (src/metrics/ssimulacra2/score.cc:103-114):
    whether (channel, scale) of a `scales`-level plan is never computed."""
    out = ctypes.c_int()
    _check(_lib.vqm_cu_ss2_channel_pruned(channel, scale, scales, ctypes.byref(out)))
    return bool(out.value)


def auto_blur_variant(sizes, sms: int = 148) -> int:
    """The blur variant (index into blur_variants()) a batch created without
    one takes for pairs of these (width, height) sizes on a device of `sms`
    SMs. Host only."""
    flat = np.asarray(list(sizes), dtype=np.uint32).reshape(-1)
    out = ctypes.c_uint32()
    _check(_lib.vqm_cu_ss2_auto_blur_variant(flat.ctypes.data, flat.size // 2, sms,
                                             ctypes.byref(out)))
    return out.value


def blur_taps(blur: int = 0) -> np.ndarray:
    """The 13 float taps (offsets -6..6) the kernels apply along each axis
    for a blur mode (Ssimulacra2Blur)."""
    taps = np.zeros(13, dtype=np.float32)
    _check(_lib.vqm_cu_ss2_blur_taps(int(blur), taps.ctypes.data))
    return taps


def check_cbrt(first_bits: int, last_bits: int):
    """Runs the prepare kernels' cube root and the shared correctly rounded
    one on every float with a bit pattern in [first_bits, last_bits] on the
    current device: (how many differ, the smallest differing pattern or
    0xffffffff)."""
    n, first = ctypes.c_uint64(), ctypes.c_uint32()
    _check(_lib.vqm_cu_ss2_check_cbrt(first_bits, last_bits, ctypes.byref(n),
                                      ctypes.byref(first)))
    return n.value, first.value


def check_division(first_bits: int, last_bits: int):
    """Runs the blur maps' division and the shared one (ss2dm::divf) for
    every divisor with a bit pattern in [first_bits, last_bits], at sixteen
    quotient values each, on the current device: (how many divisions differ,
    the smallest divisor pattern among them or 0xffffffff)."""
    n, first = ctypes.c_uint64(), ctypes.c_uint32()
    _check(_lib.vqm_cu_ss2_check_division(first_bits, last_bits, ctypes.byref(n),
                                          ctypes.byref(first)))
    return n.value, first.value


def kept_pixels(width: int, height: int) -> int:
    """Pixels of one image's kept (level, channel) pyramid planes: what the
    prepare stage stores and the blur stage reads, per image."""
    plan = plan_scales(width, height)
    return sum(w * h for s, (w, h) in enumerate(plan) for c in range(3)
               if not channel_pruned(c, s, len(plan)))


# ---------------------------------------------------------------------------
# Pipeline
# ---------------------------------------------------------------------------


def _handle_of(h) -> int:
    return int(getattr(h, "slot", h))


@dataclass(frozen=True)
class UploadedImage:
    slot: int
    size: tuple


@dataclass(frozen=True)
class ImageBuffer:
    slot: int
    size: tuple
    bytes: int


@dataclass(frozen=True)
class DeviceInfo:
    """vqm::DeviceInfo (include/vqm_device.h): a 16-byte UUID, the name and
    the kind (DeviceType: 1 integrated, 2 discrete GPU)."""
    uuid: bytes
    name: str
    type: int

    def uuid_text(self) -> str:
        h = self.uuid.hex()
        return f"{h[:8]}-{h[8:12]}-{h[12:16]}-{h[16:20]}-{h[20:]}"


def list_devices() -> list:
    """ListDevices: the CUDA devices in ordinal order."""
    n = ctypes.c_uint32()
    _check(_lib.vqm_cu_device_count(ctypes.byref(n)))
    out = []
    for i in range(n.value):
        name = ctypes.create_string_buffer(256)
        uuid = (ctypes.c_uint8 * 16)()
        kind = ctypes.c_uint32()
        _check(_lib.vqm_cu_device_info(i, name, 256, uuid, ctypes.byref(kind)))
        out.append(DeviceInfo(bytes(uuid), name.value.decode(errors="replace"), kind.value))
    return out


def set_default_device(uuid: bytes) -> None:
    """SetDefaultDevice: the device a config's device = -1 uses from now on."""
    buf = (ctypes.c_uint8 * 16).from_buffer_copy(bytes(uuid))
    _check(_lib.vqm_cu_set_default_device(buf))


def compute_worst_background(pipeline, original, distorted) -> "Ssimulacra2Result":
    """ComputeWorstBackground (include/vqm_alpha.h:12-28): a pair with no
    alpha on either side is scored once at the default background; otherwise
    over a dark (0.1) and a bright (0.9) background, returning the result
    with the lower score. `pipeline` is a Ssimulacra2Pipeline; the images are
    any kind its compute takes."""
    if (original.format.alpha == AlphaType.None_
            and distorted.format.alpha == AlphaType.None_):
        return pipeline.compute(original, distorted)
    dark = pipeline.compute(original, distorted, 0.1)
    bright = pipeline.compute(original, distorted, 0.9)
    return bright if bright.score() < dark.score() else dark


class Ssimulacra2Pipeline:
    """Ssimulacra2Pipeline (include/ssimulacra2.h:83-215) on a CUDA device."""

    def __init__(self, width: int, height: int, gpu_resident_images: int = 2,
                 half_planes: bool = False, chroma_filter: int = 0,
                 input_bytes: int = 0, streaming_inputs: bool = True,
                 device: int = -1, blur: int = 0, memory_policy: int = 0):
        """`blur`: Ssimulacra2Blur.SAMPLED (VQM's) or RECURSIVE (opt-in).
        `memory_policy`: MemoryPolicy.AUTOMATIC/DIRECT read the allocate_image
        pool in place from pinned host memory, STAGED copies its spans to the
        device at submit."""
        cfg = _Config(width, height, gpu_resident_images, int(half_planes),
                      chroma_filter, int(streaming_inputs), input_bytes, device, int(blur),
                      int(memory_policy))
        self._p = ctypes.c_void_p()
        _check(_lib.vqm_cu_ss2_create(ctypes.byref(cfg), ctypes.byref(self._p)))
        self.size = (width, height)

    def close(self):
        if getattr(self, "_p", None) and self._p.value:
            _check(_lib.vqm_cu_ss2_destroy(self._p))
            self._p = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    @property
    def handle(self) -> int:
        return self._p.value

    def set_stream(self, stream: int | None):
        _check(_lib.vqm_cu_ss2_set_stream(self._p, stream or None))

    def set_graphs(self, enabled: bool):
        _check(_lib.vqm_cu_ss2_set_graphs(self._p, int(enabled)))

    def reference_reuses(self) -> int:
        """Submissions that reused the cached pyramid of a resident original
        (vulkan.cc:238-243, 714-736)."""
        n = ctypes.c_uint64()
        _check(_lib.vqm_cu_ss2_reference_reuses(self._p, ctypes.byref(n)))
        return n.value

    def submit(self, original, distorted, background: float = 0.5) -> int:
        tok = ctypes.c_uint64()
        if isinstance(original, UploadedImage) and isinstance(distorted, UploadedImage):
            _check(_lib.vqm_cu_ss2_submit_resident(self._p, original.slot, distorted.slot,
                                                   background, ctypes.byref(tok)))
        elif isinstance(original, UploadedImage):
            d = self._idle_first(distorted._c)
            _check(_lib.vqm_cu_ss2_submit_resident_image(self._p, original.slot, ctypes.byref(d),
                                                         background, ctypes.byref(tok)))
        elif isinstance(original, ImageBuffer) and isinstance(distorted, ImageBuffer):
            _check(_lib.vqm_cu_ss2_submit_buffers(self._p, original.slot, distorted.slot,
                                                  background, ctypes.byref(tok)))
        else:
            o, d = self._idle_first(lambda: (original._c(), distorted._c()))
            _check(_lib.vqm_cu_ss2_submit(self._p, ctypes.byref(o), ctypes.byref(d),
                                          background, ctypes.byref(tok)))
        return tok.value

    def finish(self, token: int) -> Ssimulacra2Result:
        norms = np.zeros(108, dtype=np.float64)
        n = ctypes.c_uint32()
        _check(_lib.vqm_cu_ss2_finish(self._p, token, norms.ctypes.data, ctypes.byref(n)))
        return Ssimulacra2Result(norms[: 18 * n.value].reshape(n.value, 18).copy())

    def compute(self, original, distorted, background: float = 0.5) -> Ssimulacra2Result:
        return self.finish(self.submit(original, distorted, background))

    def _idle_first(self, checks):
        """Runs the host-side image checks; when one fails while a submission
        is in flight, reports the submission first, as VQM does
        (vulkan_runtime.h:275-285)."""
        try:
            return checks()
        except InvalidArgument:
            busy = ctypes.c_uint32()
            if _lib.vqm_cu_ss2_in_flight(self._p, ctypes.byref(busy)) == 0 and busy.value:
                raise LogicError("cuda: a submission is already in flight; Finish it first")
            raise

    def upload(self, image) -> UploadedImage:
        c = self._idle_first(image._c)
        h = ctypes.c_uint64()
        _check(_lib.vqm_cu_ss2_upload(self._p, ctypes.byref(c), ctypes.byref(h)))
        return UploadedImage(h.value, (image.width, image.height))

    def release(self, handle) -> None:
        if isinstance(handle, ImageBuffer):
            _check(_lib.vqm_cu_ss2_release_image(self._p, handle.slot))
        else:
            _check(_lib.vqm_cu_ss2_release(self._p, _handle_of(handle)))

    def allocate_image(self, fmt: ImageFormat) -> ImageBuffer:
        h = ctypes.c_uint64()
        b = ctypes.c_size_t()
        _check(_lib.vqm_cu_ss2_allocate_image(self._p, ctypes.byref(fmt), ctypes.byref(h),
                                              ctypes.byref(b)))
        return ImageBuffer(h.value, self.size, b.value)

    def map_image(self, buffer: ImageBuffer) -> int:
        """Host address of the buffer's bytes in the pinned pool: write them
        (ctypes.memmove, or cudaMemcpy with cudaMemcpyDefault) before the
        submission; the kernels read them in place."""
        ptr = ctypes.c_void_p()
        _check(_lib.vqm_cu_ss2_map_image(self._p, buffer.slot, ctypes.byref(ptr)))
        return ptr.value

    def debug_plane(self, image: int, level: int, channel: int) -> np.ndarray:
        """The XYB plane the last finished pair wrote (diagnostic)."""
        w, h = plan_scales(*self.size)[level]
        out = np.empty((h, w), dtype=np.float32)
        _check(_lib.vqm_cu_ss2_debug_plane(self._p, image, level, channel, out.ctypes.data))
        return out

    def get_memory_usage(self) -> MemoryUsage:
        u = MemoryUsage()
        _check(_lib.vqm_cu_ss2_memory_usage(self._p, ctypes.byref(u)))
        return u


# ---------------------------------------------------------------------------
# Batched scoring
# ---------------------------------------------------------------------------


VARIANT_WORDS = 5

DECODE_PATHS = ("generic", "table", "table_in_range", "yuv")


def decode_path(fmt: "ImageFormat", chroma_filter: int = 0) -> str:
    """Which device decode images of `fmt` take (the results are the same
    whichever runs): "generic", "table" (8-bit grey/RGB through a table),
    "table_in_range" (the same, non-negative linear samples) or "yuv"
    (integer YUV, power-law transfer, at most 2x chroma subsampling; an
    image of such a format with an odd width or height runs the generic
    decode)."""
    path = ctypes.c_uint32()
    _check(_lib.vqm_cu_ss2_decode_path(ctypes.byref(fmt), chroma_filter, ctypes.byref(path)))
    return DECODE_PATHS[path.value]


def blur_variants():
    """[(tile_w, tile_h, threads, strip, persistent)] of the blur kernels
    compiled in; strip = tiles one CTA computes down a column."""
    n = ctypes.c_uint32()
    _check(_lib.vqm_cu_ss2_blur_variants(ctypes.byref(n), None))
    k = VARIANT_WORDS
    shapes = (ctypes.c_uint32 * (k * n.value))()
    _check(_lib.vqm_cu_ss2_blur_variants(ctypes.byref(n), shapes))
    return [tuple(shapes[k * i:k * i + k]) for i in range(n.value)]


class Ssimulacra2Batch:
    """Many pairs of any sizes, scored by one launch per stage."""

    def __init__(self, max_pairs: int = 0, max_pixels: int = 0, chroma_filter: int = 0,
                 device: int = -1, tile: tuple[int, int] | None = None,
                 variant: int | None = None, half_planes: bool = False, blur: int = 0):
        """`variant` picks a compiled blur kernel (see blur_variants());
        `tile` picks the one-tile-per-CTA kernel of that output tile;
        neither: each submit picks a 32x32 strip length from its tile count
        (strips regroup the compensated partial sums, so results agree to
        rounding, ~1e-7 relative, whichever runs). `half_planes` stores the
        pyramid as binary16 (ssimulacra2.h:41-46). `blur`: the filter
        (Ssimulacra2Blur)."""
        tw, th = tile if tile else (0, 0)
        v = 0 if variant is None else variant + 1
        cfg = _BatchConfig(max_pixels, max_pairs, chroma_filter, device, tw, th, v,
                           int(half_planes), int(blur))
        self._b = ctypes.c_void_p()
        _check(_lib.vqm_cu_ss2_batch_create(ctypes.byref(cfg), ctypes.byref(self._b)))

    def close(self):
        if getattr(self, "_b", None) and self._b.value:
            _check(_lib.vqm_cu_ss2_batch_destroy(self._b))
            self._b = ctypes.c_void_p()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def handle(self) -> int:
        return self._b.value

    def set_stream(self, stream: int | None):
        _check(_lib.vqm_cu_ss2_batch_set_stream(self._b, stream or None))

    def set_timing(self, enabled: bool):
        """Record CUDA events around each stage of every batch."""
        _check(_lib.vqm_cu_ss2_batch_set_timing(self._b, int(enabled)))

    def stage_ms(self):
        """(prepare, blur, finalize) device milliseconds of the last batch."""
        ms = (ctypes.c_float * 3)()
        _check(_lib.vqm_cu_ss2_batch_stage_ms(self._b, ms))
        return tuple(ms)

    def device_bytes(self) -> int:
        """Device memory the batch holds now (reused from submit to submit)."""
        out = ctypes.c_uint64()
        _check(_lib.vqm_cu_ss2_batch_device_bytes(self._b, ctypes.byref(out)))
        return out.value

    def device_bytes_after(self, pairs) -> int:
        """Device memory the batch will hold once `pairs` are submitted
        (validated as submit would; nothing is allocated)."""
        n, origs, dists = self._arrays(pairs)
        out = ctypes.c_uint64()
        _check(_lib.vqm_cu_ss2_batch_device_bytes_after(self._b, n, origs, dists,
                                                         ctypes.byref(out)))
        return out.value

    def trim(self):
        """Frees the device memory of an idle batch."""
        _check(_lib.vqm_cu_ss2_batch_trim(self._b))

    @staticmethod
    def _arrays(pairs):
        n = len(pairs)
        origs = (_CImage * n).from_buffer_copy(b"".join(_c_bytes(p[0]) for p in pairs))
        dists = (_CImage * n).from_buffer_copy(b"".join(_c_bytes(p[1]) for p in pairs))
        return n, origs, dists

    def submit(self, pairs, background: float = 0.5, borrow: bool = False) -> int:
        """Queues the pairs. With `borrow`, host images are copied
        asynchronously and must stay unchanged until finish returns."""
        n, origs, dists = self._arrays(pairs)
        self._pending = n
        tok = ctypes.c_uint64()
        fn = _lib.vqm_cu_ss2_batch_submit_borrowed if borrow else _lib.vqm_cu_ss2_batch_submit
        _check(fn(self._b, n, origs, dists, background, ctypes.byref(tok)))
        self._borrowed = pairs if borrow else None
        return tok.value

    def finish(self, token: int):
        n = self._pending
        norms = np.zeros((n, 108), dtype=np.float64)
        scales = np.zeros(n, dtype=np.uint32)
        scores = np.zeros(n, dtype=np.float64)
        status = _lib.vqm_cu_ss2_batch_finish(self._b, token, norms.ctypes.data,
                                              scales.ctypes.data, scores.ctypes.data)
        self._borrowed = None
        _check(status)
        return [Ssimulacra2Result(norms[i, : 18 * scales[i]].reshape(scales[i], 18).copy(),
                                  float(scores[i])) for i in range(n)]

    def compute_many(self, pairs, background: float = 0.5):
        return self.finish(self.submit(pairs, background))

    def score_many(self, pairs, background: float = 0.5):
        return [r.score() for r in self.compute_many(pairs, background)]


class Ssimulacra2Pool:
    """Ssimulacra2Pool (include/vqm_pool.h:51-87): results in input order.

    The reference round-robins pairs over ``workers`` one-in-flight
    pipelines of one geometry. Here each worker is a batch scorer on its own
    stream that takes ``chunk`` pairs (of any sizes) per submission, one
    launch per stage; chunks go to the workers in turn, each worker with at
    most one chunk in flight, so one chunk's host-to-device copies overlap
    the previous chunk's kernels. If a submission or a finish fails, the
    chunks already submitted are drained before that first error propagates
    (pool.cc:64-72); if a drain itself fails, the workers are released and
    every later call raises LogicError (pool.cc:94-109, "pool cannot be
    reused after a failed drain").

    ``compute_many`` is ``results(submit_many(...))``. A caller streaming
    lists through the pool can ``submit_many`` the next list before taking
    the ``results`` of the previous one: its chunks then go to the workers as
    the previous list's chunks finish, so the copies never wait for the end
    of a list. The pairs of a list stay referenced until its results are
    taken."""

    def __init__(self, workers: int = 1, chunk: int = 64, chroma_filter: int = 0,
                 device: int = -1, half_planes: bool = False, blur: int = 0):
        if workers < 1:
            raise InvalidArgument("pool needs at least one worker")
        self._chunk = max(1, chunk)
        self._batches = [Ssimulacra2Batch(max_pairs=self._chunk, chroma_filter=chroma_filter,
                                          device=device, half_planes=half_planes, blur=blur)
                         for _ in range(workers)]
        self._queue = collections.deque()     # (ticket, first, pairs, background) not submitted
        self._inflight = collections.deque()  # (worker, token, ticket, first, pairs) in order
        self._busy = [False] * workers
        self._next = 0                        # next worker in turn
        self._lists = {}                      # ticket -> [results, chunks left]
        self._tickets = 0
        self._poisoned = False

    def workers(self) -> int:
        return len(self._batches)

    def close(self):
        for b in self._batches:
            b.close()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def _pump(self):
        """Submits queued chunks while the next worker in turn is free."""
        while self._queue and not self._busy[self._next]:
            ticket, first, pairs, background = self._queue[0]
            w = self._next
            # The pairs stay referenced until drained, so the copies may run
            # behind the call: chunks' uploads queue back to back.
            token = self._batches[w].submit(pairs, background, borrow=True)
            self._queue.popleft()
            self._busy[w] = True
            self._inflight.append((w, token, ticket, first, pairs))
            self._next = (w + 1) % len(self._batches)

    def _finish_oldest(self):
        w, token, ticket, first, _ = self._inflight.popleft()
        self._busy[w] = False
        results = self._batches[w].finish(token)
        entry = self._lists[ticket]
        entry[0][first:first + len(results)] = results
        entry[1] -= 1

    def _drain(self) -> bool:
        """Finishes every chunk in flight; False if any finish failed."""
        ok = True
        while self._inflight:
            w, token, _, _, _ = self._inflight.popleft()
            self._busy[w] = False
            try:
                self._batches[w].finish(token)
            except Exception:
                ok = False
        return ok

    def _usable(self):
        if self._poisoned:
            raise LogicError("pool cannot be reused after a failed drain")

    def submit_many(self, pairs: Iterable, background: float = 0.5) -> int:
        """Queues a list of pairs; returns the ticket for ``results``."""
        self._usable()
        pairs = list(pairs)
        ticket = self._tickets
        self._tickets += 1
        chunks = range(0, len(pairs), self._chunk)
        self._lists[ticket] = [[None] * len(pairs), len(chunks)]
        for first in chunks:
            self._queue.append((ticket, first, pairs[first:first + self._chunk], background))
        try:
            self._pump()
        except BaseException:
            self._abort()
            raise
        return ticket

    def results(self, ticket: int) -> list:
        """The list's results in input order (waits for its chunks)."""
        self._usable()
        if ticket not in self._lists:
            raise InvalidArgument("pool: no list with that ticket")
        try:
            while self._lists[ticket][1] > 0:
                if not self._inflight:
                    self._pump()
                self._finish_oldest()
                self._pump()
        except BaseException:
            self._abort()
            raise
        return self._lists.pop(ticket)[0]

    def _abort(self):
        """After a failure: drains what is in flight and drops every list;
        a failed drain releases the workers and poisons the pool."""
        drained = self._drain()
        self._queue.clear()
        self._busy = [False] * len(self._batches)
        self._lists.clear()
        if not drained:
            self.close()
            self._batches = []
            self._poisoned = True

    def compute_many(self, pairs: Iterable, background: float = 0.5):
        return self.results(self.submit_many(pairs, background))

    def score_many(self, pairs: Iterable, background: float = 0.5):
        return [r.score() for r in self.compute_many(pairs, background)]


class Ssimulacra2Server:
    """Continuous batching of single-pair requests (vqm_cu_ss2_server_*).

    ``submit`` queues a pair and returns at once with a ticket; a dispatcher
    thread forms batches from the queue in arrival order whenever one of
    ``workers`` batch scorers is free, admitting a batch only while the
    device memory all workers hold together (counted as allocated) stays
    within ``memory_budget`` (lowered to the device's free memory less
    256 MiB if that is smaller), freeing idle workers' memory when the next
    request needs it; a completion thread finishes batches in order.
    ``wait`` returns the pair's result and its latency from submit to
    completion. The images of a request are kept referenced here until its
    wait returns. A request's result is bit-identical to scoring the pair
    alone with the same blur kernel (``variant``, as Ssimulacra2Batch's plus
    one; 0 lets each batch pick a strip length from its size, and results
    then agree to rounding, ~1e-7 relative)."""

    def __init__(self, memory_budget: int = 0, workers: int = 2, max_batch_pairs: int = 64,
                 chroma_filter: int = 0, device: int = -1, variant: int = 0,
                 blur: int = 0):
        cfg = _ServerConfig(memory_budget, workers, max_batch_pairs, chroma_filter, device,
                            variant, int(blur))
        self._s = ctypes.c_void_p()
        _check(_lib.vqm_cu_ss2_server_create(ctypes.byref(cfg), ctypes.byref(self._s)))
        self._keep = {}

    def close(self):
        if self._s:
            _check(_lib.vqm_cu_ss2_server_destroy(self._s))
            self._s = ctypes.c_void_p()
            self._keep.clear()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def submit(self, original, distorted, background: float = 0.5) -> int:
        o, d = original._c(), distorted._c()
        ticket = ctypes.c_uint64()
        _check(_lib.vqm_cu_ss2_server_submit(self._s, ctypes.byref(o), ctypes.byref(d),
                                             background, ctypes.byref(ticket)))
        self._keep[ticket.value] = (original, distorted)
        return ticket.value

    def wait(self, ticket: int, timeout_ms: int = -1):
        """(Ssimulacra2Result, latency in ms) of a submitted pair."""
        norms = np.zeros(108, dtype=np.float64)
        scales = ctypes.c_uint32()
        score = ctypes.c_double()
        latency = ctypes.c_double()
        status = _lib.vqm_cu_ss2_server_wait(self._s, ticket, timeout_ms, norms.ctypes.data,
                                             ctypes.byref(scales), ctypes.byref(score),
                                             ctypes.byref(latency))
        if status != 5:
            self._keep.pop(ticket, None)
        _check(status)
        n = scales.value
        return Ssimulacra2Result(norms[: 18 * n].reshape(n, 18).copy(), score.value), latency.value

    def stats(self) -> ServerStats:
        st = ServerStats()
        _check(_lib.vqm_cu_ss2_server_get_stats(self._s, ctypes.byref(st)))
        return st
