"""PNG/JPEG inputs of the CLI (vqm_b200/stills.py): VQM's still formats
(tools/image_io/io.cc:217-229, 312-319) and the CLI on still pairs
(tests/test_cli.py:139-213 of the reference)."""

import io
import json

import numpy as np
import pytest

from tests import helpers, synthetic
from vqm_b200 import ss2, stills

cv2 = pytest.importorskip("cv2")
PIL = pytest.importorskip("PIL.Image")


def _planes(img: ss2.Image):
    out = []
    for geo in ss2.plane_layout(img.format, img.width, img.height):
        if geo is None:
            out.append(None)
            continue
        off, w, h, sb = geo
        dtype = np.uint16 if sb == 2 else np.uint8
        out.append(img.data[off:off + w * h * sb].view(dtype).reshape(h, w))
    return out


def test_png_formats(tmp_path):
    rng = np.random.default_rng(0)
    rgb = rng.integers(0, 256, (9, 13, 3), dtype=np.uint8)
    rgba = rng.integers(0, 256, (9, 13, 4), dtype=np.uint8)
    grey = rng.integers(0, 256, (9, 13), dtype=np.uint8)
    wide = rng.integers(0, 65536, (9, 13, 3), dtype=np.uint16)
    la = rng.integers(0, 256, (9, 13, 2), dtype=np.uint8)
    PIL.fromarray(rgb, "RGB").save(tmp_path / "rgb.png")
    PIL.fromarray(rgba, "RGBA").save(tmp_path / "rgba.png")
    PIL.fromarray(grey, "L").save(tmp_path / "grey.png")
    PIL.fromarray(la, "LA").save(tmp_path / "la.png")
    cv2.imwrite(str(tmp_path / "wide.png"), wide[..., ::-1])  # OpenCV writes BGR
    index = rng.integers(0, 4, (9, 13), dtype=np.uint8)
    palette = [10, 20, 30, 40, 50, 60, 70, 80, 90, 100, 110, 120]
    pal = PIL.fromarray(index, "P")
    pal.putpalette(palette)
    pal.save(tmp_path / "pal.png", transparency=bytes([255, 0, 128, 255]))

    def fmt(path):
        img = stills.load(str(tmp_path / path))
        assert (img.width, img.height) == (13, 9)
        assert img.data.nbytes == ss2.required_bytes(img.format, 13, 9)
        f = img.format
        assert f.transfer == ss2.TransferCharacteristics.Srgb
        assert f.primaries == ss2.ColorPrimaries.Bt709 and f.range == ss2.PixelRange.Full
        return img, f

    img, f = fmt("rgb.png")
    assert (f.type, f.family, f.alpha, f.matrix, f.depth) == (
        ss2.PixelType.Byte, ss2.ColorFamily.Rgb, ss2.AlphaType.None_, ss2.MatrixCoefficients.Rgb, 0)
    p = _planes(img)
    for c in range(3):
        assert np.array_equal(p[c], rgb[..., c])
    img, f = fmt("rgba.png")
    assert f.alpha == ss2.AlphaType.Straight
    assert np.array_equal(_planes(img)[3], rgba[..., 3])
    img, f = fmt("grey.png")
    assert (f.family, f.matrix, f.alpha) == (ss2.ColorFamily.Grey, ss2.MatrixCoefficients.Bt709,
                                             ss2.AlphaType.None_)
    assert np.array_equal(_planes(img)[0], grey)
    img, f = fmt("la.png")
    assert (f.family, f.alpha) == (ss2.ColorFamily.Grey, ss2.AlphaType.Straight)
    p = _planes(img)
    assert np.array_equal(p[0], la[..., 0]) and np.array_equal(p[3], la[..., 1])
    img, f = fmt("wide.png")
    assert (f.type, f.depth) == (ss2.PixelType.Word, 16)
    p = _planes(img)
    for c in range(3):
        assert np.array_equal(p[c], wide[..., c])
    img, f = fmt("pal.png")
    assert (f.family, f.alpha) == (ss2.ColorFamily.Rgb, ss2.AlphaType.Straight)
    p = _planes(img)
    lut = np.array(palette, np.uint8).reshape(4, 3)
    for c in range(3):
        assert np.array_equal(p[c], lut[index, c])
    assert np.array_equal(p[3], np.array([255, 0, 128, 255], np.uint8)[index])
    # A colour key (tRNS of a grey or RGB image) becomes an alpha plane, as
    # libpng's png_set_tRNS_to_alpha gives it to VQM.
    PIL.fromarray(grey, "L").save(tmp_path / "grey_key.png", transparency=int(grey[0, 0]))
    img, f = fmt("grey_key.png")
    assert (f.family, f.alpha) == (ss2.ColorFamily.Grey, ss2.AlphaType.Straight)
    assert np.array_equal(_planes(img)[3], np.where(grey == grey[0, 0], 0, 255))
    key = tuple(int(v) for v in rgb[2, 3])
    PIL.fromarray(rgb, "RGB").save(tmp_path / "rgb_key.png", transparency=key)
    img, f = fmt("rgb_key.png")
    assert (f.family, f.alpha) == (ss2.ColorFamily.Rgb, ss2.AlphaType.Straight)
    assert np.array_equal(_planes(img)[3], np.where((rgb == key).all(-1), 0, 255))


def test_jpeg_and_readers(tmp_path):
    rng = np.random.default_rng(1)
    colour = rng.integers(0, 256, (16, 24, 3), dtype=np.uint8)
    PIL.fromarray(colour, "RGB").save(tmp_path / "c.jpg", quality=90)
    PIL.fromarray(colour[..., 0], "L").save(tmp_path / "g.jpg", quality=90)
    img = stills.load(str(tmp_path / "c.jpg"))
    assert (img.format.type, img.format.family) == (ss2.PixelType.Byte, ss2.ColorFamily.Rgb)
    decoded = cv2.imread(str(tmp_path / "c.jpg"), cv2.IMREAD_UNCHANGED)
    assert np.array_equal(_planes(img)[0], decoded[..., 2])
    assert stills.load(str(tmp_path / "g.jpg")).format.family == ss2.ColorFamily.Grey
    reader = stills.open_sequence(str(tmp_path / "c.jpg"))
    assert reader.header.fps is None and reader.remaining() == 1
    assert len(list(reader)) == 1 and reader.remaining() == 0
    (tmp_path / "x.bin").write_bytes(b"not an image")
    from vqm_b200 import y4m
    with pytest.raises(y4m.Y4mError, match="not a PNG, JPEG or Y4M"):
        stills.open_sequence(str(tmp_path / "x.bin"))


@pytest.mark.gpu
def test_cli_on_png_pairs(tmp_path):
    """Identical PNGs score 100; a PNG pair scores like the pipeline and the
    oracle; a flat opaque image against the same pixels fully transparent
    keeps the worse background on either side, below 90
    (reference tests/test_cli.py:139-213)."""
    from vqm_b200 import cli
    o, d, _ = synthetic.rgb_pair(96, 64, 4)

    def planes(img):
        n = 96 * 64
        return np.stack([img.data[k * n:(k + 1) * n].reshape(64, 96) for k in range(3)], -1)

    PIL.fromarray(planes(o), "RGB").save(tmp_path / "o.png")
    PIL.fromarray(planes(d), "RGB").save(tmp_path / "d.png")
    out = io.StringIO()
    assert cli.run([str(tmp_path / "o.png"), str(tmp_path / "o.png")], out=out) == 0
    assert out.getvalue().strip() == "100.00000000"
    out = io.StringIO()
    assert cli.run([str(tmp_path / "o.png"), str(tmp_path / "d.png"), "--json"], out=out) == 0
    got = json.loads(out.getvalue())["score"]
    lo, ld = stills.load(str(tmp_path / "o.png")), stills.load(str(tmp_path / "d.png"))
    with ss2.Ssimulacra2Pipeline(96, 64) as p:
        assert got == p.compute(lo, ld).score()
    assert abs(got - helpers.oracle_compute(lo, ld)[1]) <= helpers.SCORE_TOL

    flat = np.full((32, 32, 3), 128, np.uint8)
    PIL.fromarray(flat, "RGB").save(tmp_path / "opaque.png")
    PIL.fromarray(np.concatenate([flat, np.zeros((32, 32, 1), np.uint8)], -1),
                  "RGBA").save(tmp_path / "transparent.png")
    for a, b in (("opaque", "transparent"), ("transparent", "opaque")):
        out = io.StringIO()
        assert cli.run([str(tmp_path / f"{a}.png"), str(tmp_path / f"{b}.png")], out=out) == 0
        assert float(out.getvalue()) < 90.0
