"""The sequence path: the Y4M reader (tools/image_io/io.cc:405-600 of the
reference) and the CLI's per-frame scores, clip mean and raw norms."""

import io
import json
import os

import numpy as np
import pytest

from tests import helpers
from tests import synthetic
from vqm_b200 import ss2, y4m


def _clip(tmp_path, frames=3, w=64, h=48):
    pairs = [synthetic.yuv_pair(w, h, 500 + f)[:2] for f in range(frames)]
    po, pd = tmp_path / "o.y4m", tmp_path / "d.y4m"
    y4m.write(str(po), [o for o, _ in pairs], "420p10")
    y4m.write(str(pd), [d for _, d in pairs], "420p10")
    return pairs, str(po), str(pd)


def test_header_defaults_and_tags():
    h = y4m.read_header(io.BytesIO(b"YUV4MPEG2 W64 H48 F30000:1001 Ip A1:1\n"))
    f = h.format
    assert (h.width, h.height, h.fps, h.progressive, h.tag) == (64, 48, (30000, 1001), True,
                                                               "420jpeg")
    assert f.chroma_location == ss2.ChromaLocation.Center
    assert (f.range, f.matrix, f.transfer, f.primaries) == (
        ss2.PixelRange.Limited, ss2.MatrixCoefficients.Bt470Bg,
        ss2.TransferCharacteristics.Bt709, ss2.ColorPrimaries.Bt709)
    assert (f.type, f.depth, f.subsample_w, f.subsample_h) == (ss2.PixelType.Byte, 0, 1, 1)
    h = y4m.read_header(io.BytesIO(b"YUV4MPEG2 W16 H8 C422p12\n"))
    assert (h.format.type, h.format.depth, h.format.subsample_w, h.format.subsample_h,
            h.format.chroma_location) == (ss2.PixelType.Word, 12, 1, 0, ss2.ChromaLocation.Left)
    assert y4m.read_header(io.BytesIO(b"YUV4MPEG2 W8 H8 C444alpha\n")).format.alpha == \
        ss2.AlphaType.Straight
    assert y4m.read_header(io.BytesIO(b"YUV4MPEG2 W8 H8 Cmono\n")).format.family == \
        ss2.ColorFamily.Grey
    assert y4m.read_header(io.BytesIO(b"YUV4MPEG2 W8 H8 C420paldv\n")).format.chroma_location \
        == ss2.ChromaLocation.TopLeft


@pytest.mark.parametrize("header,message", [
    (b"YUV4MPEG3 W8 H8\n", "not a YUV4MPEG2"),
    (b"YUV4MPEG2 W8\n", "no frame size"),
    (b"YUV4MPEG2 W9 H8 C420\n", "not divisible"),
    (b"YUV4MPEG2 W8 H8 C420p11\n", "unsupported y4m chroma tag"),
    (b"YUV4MPEG2 W8 H8 C400\n", "unsupported y4m chroma tag"),
])
def test_header_errors(header, message):
    with pytest.raises(y4m.Y4mError, match=message):
        y4m.read_header(io.BytesIO(header))


def test_frames_round_trip_and_truncation(tmp_path):
    pairs, po, _ = _clip(tmp_path)
    with y4m.Reader(po) as r:
        got = list(r)
    assert len(got) == len(pairs)
    for img, (o, _) in zip(got, pairs):
        assert np.array_equal(img.data, o.data)
        assert img.format.depth == 10 and img.format.type == ss2.PixelType.Word
    data = open(po, "rb").read()
    (tmp_path / "t.y4m").write_bytes(data[:-5])
    with y4m.Reader(str(tmp_path / "t.y4m")) as r, pytest.raises(y4m.Y4mError, match="truncated"):
        list(r)


def test_reader_skip_and_remaining(tmp_path):
    pairs, po, _ = _clip(tmp_path, frames=5)
    with y4m.Reader(po) as r:
        assert r.remaining() == 5
        assert r.skip(2) == 2
        assert r.remaining() == 3
        img = next(iter(r))
        assert np.array_equal(img.data, pairs[2][0].data)
        assert r.skip(10) == 2
        assert r.remaining() == 0
    data = open(po, "rb").read()
    (tmp_path / "t.y4m").write_bytes(data[:-5])
    with y4m.Reader(str(tmp_path / "t.y4m")) as r, pytest.raises(y4m.Y4mError, match="truncated"):
        r.skip(5)


def test_cli_rejects_mismatched_clips(tmp_path, capsys):
    from vqm_b200 import cli
    _, po, _ = _clip(tmp_path, frames=2)
    short = tmp_path / "s.y4m"
    o, _ = synthetic.yuv_pair(64, 48, 1)[:2]
    y4m.write(str(short), [o], "420p10", fps=(30, 1))
    assert cli.main([po, str(short)]) == 1  # a failure while scoring (cli/main.cc:170-173)
    assert "inputs have unequal frame rates" in capsys.readouterr().err


@pytest.mark.gpu
def test_cli_scores_frames_and_clip_mean(tmp_path):
    from vqm_b200 import cli
    pairs, po, pd = _clip(tmp_path)
    # The reader gives the header's colours: limited BT.470BG, BT.709 transfer.
    fmt = y4m.Reader(po).format
    expected = []
    for o, d in pairs:
        oo, dd = ss2.Image(o.width, o.height, fmt, o.data), ss2.Image(d.width, d.height, fmt, d.data)
        norms, score = helpers.oracle_compute(oo, dd)
        expected.append((norms, score))
    for batch in ("1", "2"):
        out = io.StringIO()
        assert cli.run([po, pd, "--json", "--batch", batch], out=out) == 0
        doc = json.loads(out.getvalue())
        assert (doc["sample_id"], doc["metric"], doc["frames"]) == ("pair", "ssimulacra2",
                                                                   len(pairs))
        assert doc["core_seconds"] > 0 and doc["decode_seconds"] > 0
        assert [f["index"] for f in doc["frame_results"]] == list(range(len(pairs)))
        for f, (_, score) in zip(doc["frame_results"], expected):
            assert abs(f["score"] - score) <= helpers.SCORE_TOL
        assert abs(doc["score"] - np.mean([s for _, s in expected])) <= helpers.SCORE_TOL
        out = io.StringIO()
        assert cli.run([po, pd, "--raw", "--batch", batch], out=out) == 0
        lines = out.getvalue().strip().splitlines()
        assert len(lines) == len(pairs) + 1
        assert abs(float(lines[-1]) - doc["score"]) < 1e-7
        raw0 = [float(v) for v in lines[0].rstrip(",").split(",")]
        assert len(raw0) == expected[0][0].size  # 18 per scale
        # Channel-major raw order: channel 0, scale 0, n 0 = ssim[0], ring[0], blur[2].
        n0 = expected[0][0]
        assert abs(raw0[0] - n0[0, 0]) <= 1e-4 * abs(n0[0, 0]) + 1e-9
    # The opt-in recursive blur scores the same frames against its own oracle.
    out = io.StringIO()
    assert cli.run([po, pd, "--json", "--blur", "recursive"], out=out) == 0
    doc = json.loads(out.getvalue())
    for s, (o, d) in zip([f["score"] for f in doc["frame_results"]], pairs):
        oo, dd = ss2.Image(o.width, o.height, fmt, o.data), ss2.Image(d.width, d.height, fmt, d.data)
        _, score = helpers.oracle_compute(oo, dd, blur=ss2.Ssimulacra2Blur.RECURSIVE)
        assert abs(s - score) <= helpers.SCORE_TOL


@pytest.mark.gpu
def test_cli_two_ranks_score_contiguous_ranges(tmp_path):
    """Under torchrun with two ranks the CLI splits the clip into two frame
    ranges and rank 0 prints the same clip as a single process."""
    import socket
    import subprocess
    import sys
    pairs, po, pd = _clip(tmp_path, frames=5)
    one = io.StringIO()
    from vqm_b200 import cli
    assert cli.run([po, pd, "--raw", "--batch", "2"], out=one) == 0
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    res = subprocess.run(
        [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", "--nproc-per-node", "2",
         "--master-addr", "127.0.0.1", "--master-port", str(port), "-m", "vqm_b200.cli",
         po, pd, "--raw", "--batch", "2"],
        capture_output=True, text=True, timeout=600,
        cwd=os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
    assert res.returncode == 0, res.stderr[-2000:]
    # Five frames' raw norms and the clip score, as one process prints them.
    want = one.getvalue().splitlines()
    assert len(want) == 6
    assert res.stdout.splitlines()[-6:] == want


@pytest.mark.gpu
def test_cli_alpha_keeps_the_worse_background(tmp_path):
    from vqm_b200 import cli
    fmt = y4m.read_header(io.BytesIO(b"YUV4MPEG2 W64 H48 C444alpha\n")).format
    rng = np.random.default_rng(3)
    base = synthetic.texture(64, 48, rng) / 255.0
    alpha = 0.2 + 0.8 * base[2]
    ov = [base[0], (base[1] - 0.5) * 0.6, (base[2] - 0.5) * 0.6, alpha]
    dv = [np.clip(v + rng.normal(0, 0.03, v.shape), -0.5 if i in (1, 2) else 0, 1)
          for i, v in enumerate(ov)]
    o, d = helpers.pack_planes(fmt, 64, 48, ov), helpers.pack_planes(fmt, 64, 48, dv)
    po, pd = str(tmp_path / "o.y4m"), str(tmp_path / "d.y4m")
    y4m.write(po, [o], "444alpha")
    y4m.write(pd, [d], "444alpha")
    with ss2.Ssimulacra2Pipeline(64, 48) as p:
        worse = min(p.compute(o, d, 0.1).score(), p.compute(o, d, 0.9).score())
    out = io.StringIO()
    assert cli.run([po, pd, "--json", "--batch", "1"], out=out) == 0
    assert [f["score"] for f in json.loads(out.getvalue())["frame_results"]] == [worse]
