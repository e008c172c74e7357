"""PNG and JPEG still images as one-frame sequences for the CLI.

VQM's CLI reads PNG (8- and 16-bit), baseline and progressive JPEG, and
YUV4MPEG2 (tools/image_io/io.h:15-24). Its still-image formats
(io.cc:217-229, 312-319): PNG palettes are expanded to RGB and a tRNS chunk
to an alpha plane; one or two channels are a grey image (matrix BT.709), three
or four are RGB (matrix RGB); two or four channels carry straight alpha;
16-bit PNG samples are Word samples of depth 16; every still is full range,
sRGB transfer, BT.709 primaries; ICC profiles and gAMA/cHRM/sBIT chunks are
ignored. A still has no frame rate.

The files are decoded by OpenCV (libpng and libjpeg underneath, with no
colour conversion and no EXIF rotation); the samples are laid out as the
scorer's packed planes. Y4M files go to `y4m.Reader`.
"""

from __future__ import annotations

from typing import Iterator

import numpy as np

from . import ss2, y4m

PNG_MAGIC = b"\x89PNG\r\n\x1a\n"
JPEG_MAGIC = b"\xff\xd8\xff"


def _png_color_type(path: str) -> int | None:
    with open(path, "rb") as f:
        head = f.read(26)
    if head[:8] != PNG_MAGIC or len(head) < 26 or head[12:16] != b"IHDR":
        return None
    return head[25]


def _png_transparent_key(path: str):
    """(bit depth, colour type, key samples) of a grey or RGB PNG's tRNS
    chunk, or None. OpenCV keeps the colour key out of its output, while
    libpng (png_set_tRNS_to_alpha) turns it into an alpha plane for VQM."""
    with open(path, "rb") as f:
        data = f.read()
    if data[:8] != PNG_MAGIC:
        return None
    depth, ctype = data[24], data[25]
    at = 8
    while at + 8 <= len(data):
        n = int.from_bytes(data[at:at + 4], "big")
        kind = data[at + 4:at + 8]
        if kind in (b"IDAT", b"IEND"):
            return None
        if kind == b"tRNS" and ctype in (0, 2):
            body = data[at + 8:at + 8 + n]
            key = [int.from_bytes(body[i:i + 2], "big") for i in range(0, len(body) - 1, 2)]
            return depth, ctype, key
        at += 12 + n
    return None


def load(path: str) -> ss2.Image:
    """A PNG or JPEG file as a packed ss2.Image in VQM's still format."""
    try:
        import cv2
    except ImportError as e:  # the decoder, not the scorer, is missing
        raise y4m.Y4mError(f"{path}: PNG/JPEG input needs OpenCV (cv2): {e}") from e
    with open(path, "rb") as f:
        magic = f.read(8)
    if magic[:8] != PNG_MAGIC and magic[:3] != JPEG_MAGIC:
        raise y4m.Y4mError(f"{path}: not a PNG, JPEG or Y4M file")
    pixels = cv2.imread(path, cv2.IMREAD_UNCHANGED)
    if pixels is None:
        raise y4m.Y4mError(f"{path}: the image could not be decoded")
    if pixels.ndim == 2:
        planes = [pixels]
    else:
        c = pixels.shape[2]
        planes = [pixels[..., 2], pixels[..., 1], pixels[..., 0]] if c >= 3 else [pixels[..., 0]]
        if c == 4:
            planes.append(pixels[..., 3])
        # OpenCV widens grey + alpha (PNG colour type 4, or grey with a tRNS
        # chunk) to four channels; libpng gives VQM one grey plane and alpha.
        if c == 4 and _png_color_type(path) in (0, 4):
            planes = [pixels[..., 0], pixels[..., 3]]
    if pixels.dtype not in (np.uint8, np.uint16):
        raise y4m.Y4mError(f"{path}: unsupported sample type {pixels.dtype}")
    key = _png_transparent_key(path) if len(planes) in (1, 3) else None
    if key is not None:
        depth, ctype, values = key
        need = 1 if ctype == 0 else 3
        if len(values) >= need and len(planes) == need:
            # Samples below 8 bits come out of the decoder scaled to 8 bits.
            scale = 255 // ((1 << depth) - 1) if depth < 8 else 1
            hit = np.ones(planes[0].shape, bool)
            for plane, v in zip(planes, values[:need]):
                hit &= plane == v * scale
            top = 65535 if pixels.dtype == np.uint16 else 255
            planes.append(np.where(hit, 0, top).astype(pixels.dtype))
    wide = pixels.dtype == np.uint16
    grey = len(planes) <= 2
    alpha = len(planes) in (2, 4)
    fmt = ss2.ImageFormat(
        type=ss2.PixelType.Word if wide else ss2.PixelType.Byte,
        family=ss2.ColorFamily.Grey if grey else ss2.ColorFamily.Rgb,
        alpha=ss2.AlphaType.Straight if alpha else ss2.AlphaType.None_,
        range=ss2.PixelRange.Full,
        matrix=ss2.MatrixCoefficients.Bt709 if grey else ss2.MatrixCoefficients.Rgb,
        transfer=ss2.TransferCharacteristics.Srgb, primaries=ss2.ColorPrimaries.Bt709,
        depth=16 if wide else 0)
    h, w = planes[0].shape
    data = np.zeros(ss2.required_bytes(fmt, w, h), np.uint8)
    slots = [0, 3] if grey else [0, 1, 2, 3]
    for plane, slot in zip(planes, slots):
        off, pw, ph, sb = ss2.plane_layout(fmt, w, h)[slot]
        data[off:off + pw * ph * sb] = np.ascontiguousarray(plane).view(np.uint8).ravel()
    return ss2.Image(w, h, fmt, data)


class StillReader:
    """One still image with the interface of `y4m.Reader`: `header`,
    `format` (the caller may override colour fields), `remaining`, `skip`
    and iteration."""

    def __init__(self, path: str):
        self._image = load(path)
        self.header = y4m.Header(self._image.width, self._image.height, self._image.format,
                                 None, True, "")
        self.format = self._image.format
        self._left = 1

    def remaining(self) -> int:
        return self._left

    def skip(self, n: int) -> int:
        k = min(n, self._left)
        self._left -= k
        return k

    def __iter__(self) -> Iterator[ss2.Image]:
        while self._left:
            self._left -= 1
            yield ss2.Image(self._image.width, self._image.height, self.format,
                            self._image.data)

    def close(self):
        pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()


def open_sequence(path: str):
    """A Y4M file as `y4m.Reader`, a PNG or JPEG file as `StillReader`."""
    with open(path, "rb") as f:
        magic = f.read(len(y4m.MAGIC))
    if magic == y4m.MAGIC:
        return y4m.Reader(path)
    return StillReader(path)
