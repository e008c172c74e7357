"""YUV4MPEG2 (Y4M) sequences as scorer images.

Restates the reader of VQM's tools/image_io/io.cc (ParseChromaTag,
ReadY4mHeader, ReadY4mFrame, :405-600) for the SSIMULACRA 2 sequence path:
progressive streams, chroma tags mono/420/420jpeg/420mpeg2/420paldv/422/444/
411/444alpha with optional pN depths (9, 10, 12, 14, 16), a missing C tag
meaning 420jpeg, and the format's colour defaults (limited range, BT.470BG
matrix, BT.709 transfer and primaries; y4m carries no colour metadata).
High-bit-depth samples are little-endian 16-bit words.
"""

from __future__ import annotations

import math
from dataclasses import dataclass
from typing import BinaryIO, Iterator

import numpy as np

from . import ss2

MAGIC = b"YUV4MPEG2 "
MAX_HEADER = 1 << 16

# name -> (family, subsample_w, subsample_h, chroma location, alpha)
_TAGS = {
    "mono": (ss2.ColorFamily.Grey, 0, 0, ss2.ChromaLocation.Left, False),
    "420": (ss2.ColorFamily.Yuv, 1, 1, ss2.ChromaLocation.Left, False),
    "420mpeg2": (ss2.ColorFamily.Yuv, 1, 1, ss2.ChromaLocation.Left, False),
    "420jpeg": (ss2.ColorFamily.Yuv, 1, 1, ss2.ChromaLocation.Center, False),
    "420paldv": (ss2.ColorFamily.Yuv, 1, 1, ss2.ChromaLocation.TopLeft, False),
    "422": (ss2.ColorFamily.Yuv, 1, 0, ss2.ChromaLocation.Left, False),
    "444": (ss2.ColorFamily.Yuv, 0, 0, ss2.ChromaLocation.Left, False),
    "411": (ss2.ColorFamily.Yuv, 2, 0, ss2.ChromaLocation.Left, False),
    "444alpha": (ss2.ColorFamily.Yuv, 0, 0, ss2.ChromaLocation.Left, True),
}
_DEPTHS = (9, 10, 12, 14, 16)


class Y4mError(ValueError):
    """A stream that is not a readable progressive Y4M sequence."""


@dataclass
class Header:
    width: int
    height: int
    format: ss2.ImageFormat
    fps: tuple | None  # reduced (numerator, denominator), None if absent/invalid
    progressive: bool
    tag: str


def parse_chroma_tag(tag: str):
    """'C' value -> (table entry, depth); depth 0 means 8-bit."""
    base, depth = tag, 0
    p = tag.rfind("p")
    if p != -1 and p + 1 < len(tag) and tag[p + 1:].isdigit() and int(tag[p + 1:]) in _DEPTHS:
        base, depth = tag[:p], int(tag[p + 1:])
    if base not in _TAGS:
        raise Y4mError("unsupported y4m chroma tag")
    return _TAGS[base], depth


def _read_line(f: BinaryIO) -> bytes:
    out = bytearray()
    while len(out) < MAX_HEADER:
        c = f.read(1)
        if not c:
            raise Y4mError("truncated y4m header")
        if c == b"\n":
            return bytes(out)
        out += c
    raise Y4mError("y4m header line too long")


def read_header(f: BinaryIO) -> Header:
    if f.read(len(MAGIC)) != MAGIC:
        raise Y4mError("not a YUV4MPEG2 file")
    line = _read_line(f).decode("ascii", "replace")
    width = height = None
    chroma = "420jpeg"  # MJPEGtools' default for an omitted C tag
    fps, progressive = None, True
    for token in line.split(" "):
        if len(token) < 2:
            continue
        key, value = token[0], token[1:]
        if key == "W":
            if not value.isdigit():
                raise Y4mError("invalid y4m width")
            width = int(value)
        elif key == "H":
            if not value.isdigit():
                raise Y4mError("invalid y4m height")
            height = int(value)
        elif key == "C":
            chroma = value
        elif key == "F":
            num, _, den = value.partition(":")
            if num.isdigit() and den.isdigit() and int(num) and int(den):
                g = math.gcd(int(num), int(den))
                fps = (int(num) // g, int(den) // g)
        elif key == "I":
            progressive = value == "p"
    if not width or not height:
        raise Y4mError("y4m header has no frame size")
    (family, sw, sh, location, alpha), depth = parse_chroma_tag(chroma)
    if width % (1 << sw) or height % (1 << sh):
        raise Y4mError("y4m dimensions are not divisible by the chroma subsampling")
    fmt = ss2.ImageFormat(
        type=ss2.PixelType.Byte if depth == 0 else ss2.PixelType.Word,
        family=family, alpha=ss2.AlphaType.Straight if alpha else ss2.AlphaType.None_,
        range=ss2.PixelRange.Limited, matrix=ss2.MatrixCoefficients.Bt470Bg,
        transfer=ss2.TransferCharacteristics.Bt709, primaries=ss2.ColorPrimaries.Bt709,
        chroma_location=location, subsample_w=sw, subsample_h=sh, depth=depth)
    return Header(width, height, fmt, fps, progressive, chroma)


def read_frame(f: BinaryIO, header: Header, fmt: ss2.ImageFormat | None = None):
    """The next frame as an ss2.Image in the packed plane layout, or None at
    the end of the stream. `fmt` (same sample layout) overrides the header's
    colour description."""
    first = f.read(1)
    if not first:
        return None
    line = first + _read_line(f)
    if line != b"FRAME" and not line.startswith(b"FRAME "):
        raise Y4mError("y4m file has no frame")
    fmt = header.format if fmt is None else fmt
    data = np.zeros(ss2.required_bytes(fmt, header.width, header.height), dtype=np.uint8)
    for geo in ss2.plane_layout(fmt, header.width, header.height):
        if geo is None:
            continue
        off, pw, ph, sb = geo
        n = pw * ph * sb
        raw = f.read(n)
        if len(raw) != n:
            raise Y4mError("truncated y4m frame")
        data[off:off + n] = np.frombuffer(raw, dtype=np.uint8)  # little-endian words
    return ss2.Image(header.width, header.height, fmt, data)


def frame_bytes(header: Header) -> int:
    """Sample bytes of one frame (the FRAME line excluded)."""
    return sum(g[1] * g[2] * g[3] for g in ss2.plane_layout(header.format, header.width,
                                                             header.height) if g is not None)


class Reader:
    """Iterates a Y4M file's frames as ss2.Image."""

    def __init__(self, path: str, fmt: ss2.ImageFormat | None = None):
        self._f = open(path, "rb")
        try:
            self.header = read_header(self._f)
        except Exception:
            self._f.close()
            raise
        if not self.header.progressive:
            self._f.close()
            raise Y4mError("interlaced y4m input is not supported")
        self.format = fmt or self.header.format

    def remaining(self) -> int:
        """Frames left from the current position (the position is kept)."""
        here = self._f.tell()
        try:
            return self.skip(1 << 62)
        finally:
            self._f.seek(here)

    def skip(self, n: int) -> int:
        """Skips up to n frames without reading their samples (each FRAME
        line is read, since it may carry parameters); returns the number
        skipped, fewer at the end of the stream."""
        size = frame_bytes(self.header)
        for k in range(n):
            first = self._f.read(1)
            if not first:
                return k
            line = first + _read_line(self._f)
            if line != b"FRAME" and not line.startswith(b"FRAME "):
                raise Y4mError("y4m file has no frame")
            here = self._f.tell()
            self._f.seek(0, 2)
            end = self._f.tell()
            if end - here < size:
                raise Y4mError("truncated y4m frame")
            self._f.seek(here + size)
        return n

    def __iter__(self) -> Iterator[ss2.Image]:
        while True:
            img = read_frame(self._f, self.header, self.format)
            if img is None:
                return
            yield img

    def close(self):
        self._f.close()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()


def write(path: str, frames, tag: str, fps=(25, 1)) -> None:
    """Writes images (the packed layout of `tag`) as a Y4M file."""
    frames = list(frames)
    if not frames:
        raise Y4mError("no frames")
    w, h = frames[0].width, frames[0].height
    with open(path, "wb") as f:
        f.write(MAGIC + f"W{w} H{h} F{fps[0]}:{fps[1]} Ip A1:1 C{tag}\n".encode())
        for img in frames:
            f.write(b"FRAME\n")
            for geo in ss2.plane_layout(img.format, w, h):
                if geo is None:
                    continue
                off, pw, ph, sb = geo
                f.write(img.data[off:off + pw * ph * sb].tobytes())
