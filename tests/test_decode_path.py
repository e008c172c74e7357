"""Which device decode each input format takes (host-side selection; the
GPU tests check that every path gives the oracle's planes bit for bit)."""

import pytest

from vqm_b200 import ss2

F = ss2.ImageFormat
T = ss2.TransferCharacteristics


def _yuv(**kw):
    base = dict(type=ss2.PixelType.Word, depth=10, family=ss2.ColorFamily.Yuv,
                range=ss2.PixelRange.Limited, matrix=ss2.MatrixCoefficients.Bt709,
                transfer=T.Bt709, primaries=ss2.ColorPrimaries.Bt709, subsample_w=1,
                subsample_h=1)
    base.update(kw)
    return F(**base)


@pytest.mark.parametrize("fmt,chroma_filter,path", [
    (F(type=ss2.PixelType.Byte), 0, "table_in_range"),
    (F(type=ss2.PixelType.Byte, family=ss2.ColorFamily.Grey,
       matrix=ss2.MatrixCoefficients.Bt709), 0, "table_in_range"),
    (F(type=ss2.PixelType.Byte, range=ss2.PixelRange.Limited), 0, "table"),
    (F(type=ss2.PixelType.Byte, primaries=ss2.ColorPrimaries.Bt2020), 0, "table"),
    (F(type=ss2.PixelType.Byte, alpha=ss2.AlphaType.Straight), 0, "generic"),
    (F(type=ss2.PixelType.Float), 0, "generic"),
    (_yuv(), 0, "yuv"),
    (_yuv(chroma_location=ss2.ChromaLocation.Center), 0, "yuv"),
    (_yuv(chroma_location=ss2.ChromaLocation.TopLeft), 0, "yuv"),
    (_yuv(chroma_location=ss2.ChromaLocation.Bottom), 0, "yuv"),
    (_yuv(subsample_h=0), 0, "yuv"),
    (_yuv(subsample_w=0, subsample_h=0), 0, "yuv"),
    (_yuv(type=ss2.PixelType.Byte, depth=0), 0, "yuv"),
    (_yuv(transfer=T.Bt470M), 0, "yuv"),
    (_yuv(transfer=T.Bt470Bg), 0, "yuv"),
    (_yuv(primaries=ss2.ColorPrimaries.Bt2020, matrix=ss2.MatrixCoefficients.Bt2020Ncl,
          transfer=T.Bt2020_10), 0, "yuv"),
    (_yuv(), 1, "generic"),                       # bicubic chroma
    (_yuv(transfer=T.Srgb), 0, "generic"),         # not a pure power law
    (_yuv(transfer=T.St2084), 0, "generic"),
    (_yuv(subsample_w=2, subsample_h=0), 0, "generic"),  # 4:1:1
    (_yuv(alpha=ss2.AlphaType.Straight), 0, "generic"),
    (_yuv(type=ss2.PixelType.Float, depth=0), 0, "generic"),
    (_yuv(matrix=ss2.MatrixCoefficients.Bt2020Cl, primaries=ss2.ColorPrimaries.Bt2020), 0,
     "generic"),                                   # constant luminance
])
def test_decode_path(fmt, chroma_filter, path):
    assert ss2.decode_path(fmt, chroma_filter) == path


def test_decode_path_rejects_invalid_format():
    with pytest.raises(ss2.InvalidArgument):
        ss2.decode_path(F(type=ss2.PixelType.Byte, family=ss2.ColorFamily.Grey,
                          subsample_w=1))
