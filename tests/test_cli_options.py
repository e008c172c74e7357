"""The CLI's command line as VQM's (cli/options.cc:211-395, cli/video.cc:52-80,
cli/report.cc:46-276, cli/main.cc:115-173): option rules, pairs files, exit
status, the JSON object and the verbose table."""

import io
import json

import numpy as np
import pytest

from tests import helpers, synthetic
from vqm_b200 import cli, ss2, y4m


@pytest.mark.parametrize("argv, message", [
    (["a", "b", "--json", "--raw"], "--json and --raw cannot be combined"),
    (["a", "b", "-v", "--raw"], "--verbose and --raw cannot be combined"),
    (["--pairs-file", "p.tsv"], "--pairs-file requires --json"),
    (["--json", "--pairs-file", "p.tsv", "a"], "--pairs-file replaces positional paths"),
    (["a"], "expected exactly two image paths, got 1"),
    (["a", "b", "--frobnicate"], "unknown option '--frobnicate'"),
    (["a", "b", "--metric", "vmaf"], "invalid value for --metric: 'vmaf'"),
    (["a", "b", "--metric", "ssimulacra2,butteraugli"], "ssimulacra2 only"),
    (["a", "b", "--metric", "all"], "ssimulacra2 only"),
    (["a", "b", "--input-matrix", "smpte170m"], "invalid value for --input-matrix: 'smpte170m'"),
    (["a", "b", "--iterations", "0"], "invalid value for --iterations: '0'"),
    (["a", "b", "--device"], "--device needs a value"),
    (["a", "b", "--list-devices"], "--list-devices must be used on its own"),
])
def test_rejected_command_lines(argv, message, capsys):
    with pytest.raises(cli.UsageError, match=message.replace("(", r"\(")):
        cli.parse(argv)
    assert cli.main(argv) == 2
    err = capsys.readouterr().err
    assert message in err and "Usage:" in err


def test_accepted_command_lines():
    o = cli.parse(["x.y4m", "y.y4m", "--metric", "ssimulacra2", "--metric", "ssimulacra2",
                   "--input-matrix", "st170m", "--input-transfer", "arib-b67",
                   "--input-primaries", "st431-2", "--input-range", "full",
                   "--chroma-filter", "lanczos", "--half-planes", "--iterations", "3",
                   "--warmup", "1", "-v", "--json"])
    assert o["metrics"] == ["ssimulacra2"]
    assert (o["matrix"], o["transfer"], o["primaries"], o["range"], o["chroma_filter"]) == (
        ss2.MatrixCoefficients.St170M, ss2.TransferCharacteristics.AribB67,
        ss2.ColorPrimaries.St431_2, ss2.PixelRange.Full, 2)
    assert (o["half_planes"], o["iterations"], o["warmup"], o["original"]) == (True, 3, 1,
                                                                              "x.y4m")
    assert cli.parse(["--list-devices"]) == "list-devices"
    assert cli.parse(["a", "--help"]) == "help"
    out = io.StringIO()
    assert cli.run(["--help"], out=out) == 0 and "--pairs-file" in out.getvalue()


def test_pairs_file_rows(tmp_path):
    p = tmp_path / "p.tsv"
    p.write_text("one\ta.png\tb.png\r\ntwo\tc.y4m\td.y4m\n")
    assert cli.read_pairs(str(p)) == [("one", "a.png", "b.png"), ("two", "c.y4m", "d.y4m")]
    for text, message in (("one\ta.png\n", "expected ID, original, distorted TSV"),
                          ("one\ta\tb\none\tc\td\n", "duplicate sample ID: one"),
                          ("", "empty pair list"),
                          ("one\ta\tb\tc\n", "expected ID, original, distorted TSV")):
        p.write_text(text)
        with pytest.raises(ss2.InvalidArgument, match=message):
            cli.read_pairs(str(p))
    with pytest.raises(RuntimeError, match="cannot open pairs file"):
        cli.read_pairs(str(tmp_path / "missing.tsv"))


def test_frame_ranges_need_compressed_video(capsys):
    assert cli.main(["a.y4m", "b.y4m", "--start-frame", "2"]) == 1
    assert "--start-frame and --frame-count" in capsys.readouterr().err


@pytest.mark.gpu
def test_pairs_file_iterations_and_verbose(tmp_path, capsys):
    """Two pairs of a pairs file (a Y4M clip and a still pair), one JSON
    object each in file order; -v adds scoring_fps and frame_stats; the
    verbose table; iterations and warm-up give the same scores; an
    unavailable device fails before reading the inputs."""
    clip = [synthetic.yuv_pair(64, 48, 900 + f)[:2] for f in range(3)]
    y4m.write(str(tmp_path / "o.y4m"), [o for o, _ in clip], "420p10")
    y4m.write(str(tmp_path / "d.y4m"), [d for _, d in clip], "420p10")
    o, d = synthetic.yuv_pair(64, 48, 950)[:2]
    y4m.write(str(tmp_path / "so.y4m"), [o], "420p10")
    y4m.write(str(tmp_path / "sd.y4m"), [o], "420p10")
    pairs = tmp_path / "pairs.tsv"
    pairs.write_text(f"clip\t{tmp_path / 'o.y4m'}\t{tmp_path / 'd.y4m'}\n"
                     f"same\t{tmp_path / 'so.y4m'}\t{tmp_path / 'sd.y4m'}\n")
    out = io.StringIO()
    assert cli.run(["--json", "-v", "--pairs-file", str(pairs), "--iterations", "3",
                    "--warmup", "1"], out=out) == 0
    docs = [json.loads(line) for line in out.getvalue().splitlines()]
    assert [x["sample_id"] for x in docs] == ["clip", "same"]
    fmt = y4m.Reader(str(tmp_path / "o.y4m")).format
    want = [helpers.oracle_compute(ss2.Image(64, 48, fmt, a.data),
                                   ss2.Image(64, 48, fmt, b.data))[1] for a, b in clip]
    got = [f["score"] for f in docs[0]["frame_results"]]
    assert all(abs(g - w) <= helpers.SCORE_TOL for g, w in zip(got, want))
    st = docs[0]["frame_stats"]
    assert (st["min"], st["max"]) == (min(got), max(got))
    assert st["finite_mean"] == pytest.approx(np.mean(got)) and st["infinite_frames"] == 0
    assert docs[0]["scoring_fps"] > 0
    assert docs[1]["score"] == 100.0 and docs[1]["frame_stats"]["perfect_frames"] == 1
    out = io.StringIO()
    assert cli.run([str(tmp_path / "o.y4m"), str(tmp_path / "d.y4m"), "-v"], out=out) == 0
    lines = out.getvalue().splitlines()
    assert lines[0] == "Frames: 3" and lines[1].startswith("Scoring FPS: ")
    assert lines[3].split()[0] == "ssimulacra2"
    assert float(lines[3].split()[1]) == pytest.approx(docs[0]["score"], rel=1e-7)
    assert cli.main([str(tmp_path / "o.y4m"), str(tmp_path / "d.y4m"), "--device",
                     "999999"]) == 1
    err = capsys.readouterr().err
    assert "--device 999999 is unavailable" in err and "--list-devices" in err
    out = io.StringIO()
    assert cli.run(["--list-devices"], out=out) == 0
    first = out.getvalue().splitlines()[0]
    assert first.startswith("0  ")
    assert len(first.split("  ")[-1]) == 36  # the device UUID, 8-4-4-4-12
