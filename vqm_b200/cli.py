"""SSIMULACRA 2.1 of two Y4M sequences or PNG/JPEG images, on the GPU.

    python -m vqm_b200.cli original.y4m distorted.y4m [--raw|--json] [-v]
    python -m vqm_b200.cli original.png distorted.png
    python -m vqm_b200.cli --json --pairs-file pairs.tsv

VQM's command line for this metric (cli/options.cc:211-395, cli/video.cc,
cli/report.cc, docs/ssimulacra2.md:3-6): the same flags, rules, exit status
(2 for a rejected command line, 1 for a failure while scoring) and output.
Both inputs must be two images or two Y4M sequences of the same frame size,
frame count and frame rate; every frame pair is scored independently and the
clip score is the mean of the frame scores, printed with eight decimals.
A PNG or JPEG file is one frame without a frame rate (`stills.py`, VQM's
still formats). Inputs with alpha are scored over the dark and bright
backgrounds (0.1 and 0.9) and the worse score is kept
(include/vqm_alpha.h:17-28). --raw prints each frame's 108 norms in the
channel-major order of the reference tool's tuning build (report.cc:221-248)
before the score; --json prints one object per pair (sample_id, metric, score,
frames, core_seconds, decode_seconds, frame_results; with -v also scoring_fps
and frame_stats); -v alone prints a table. --metric accepts VQM's metric names;
this build scores ssimulacra2 and rejects the others.

Frames go to the scorer `--batch` pairs at a time (one launch per stage per
batch); 1 scores each pair through a pipeline whose kernels replay as one
CUDA graph.

Under torchrun (WORLD_SIZE > 1) every rank scores a contiguous range of the
frames on its own GPU (LOCAL_RANK), reading only that range, and rank 0
prints the whole clip in frame order; the ranks exchange only per-frame
results (gloo, for the plumbing):

    python -m torch.distributed.run --nproc-per-node 8 -m vqm_b200.cli a.y4m b.y4m
"""

from __future__ import annotations

import datetime
import json
import math
import os
import statistics
import sys
import time

from . import replicas, ss2, stills, y4m

# The names of VQM's --input-* flags (tools/image_io/io.cc:706-762).
_MATRICES = {
    "rgb": ss2.MatrixCoefficients.Rgb, "bt709": ss2.MatrixCoefficients.Bt709,
    "fcc": ss2.MatrixCoefficients.Fcc, "bt470bg": ss2.MatrixCoefficients.Bt470Bg,
    "st170m": ss2.MatrixCoefficients.St170M, "st240m": ss2.MatrixCoefficients.St240M,
    "ycgco": ss2.MatrixCoefficients.YCgCo, "bt2020ncl": ss2.MatrixCoefficients.Bt2020Ncl,
    "bt2020cl": ss2.MatrixCoefficients.Bt2020Cl,
    "chromaticity-derived-ncl": ss2.MatrixCoefficients.ChromaticityDerivedNcl,
    "chromaticity-derived-cl": ss2.MatrixCoefficients.ChromaticityDerivedCl,
    "ictcp": ss2.MatrixCoefficients.Bt2100ICtCp,
}
_TRANSFERS = {
    "bt709": ss2.TransferCharacteristics.Bt709, "bt601": ss2.TransferCharacteristics.Bt601,
    "bt470m": ss2.TransferCharacteristics.Bt470M, "bt470bg": ss2.TransferCharacteristics.Bt470Bg,
    "st240m": ss2.TransferCharacteristics.St240M, "linear": ss2.TransferCharacteristics.Linear,
    "log100": ss2.TransferCharacteristics.Log100, "log316": ss2.TransferCharacteristics.Log316,
    "xvycc": ss2.TransferCharacteristics.Iec61966_2_4,
    "bt1361": ss2.TransferCharacteristics.Bt1361, "srgb": ss2.TransferCharacteristics.Srgb,
    "bt2020-10": ss2.TransferCharacteristics.Bt2020_10,
    "bt2020-12": ss2.TransferCharacteristics.Bt2020_12,
    "st2084": ss2.TransferCharacteristics.St2084, "st428": ss2.TransferCharacteristics.St428,
    "arib-b67": ss2.TransferCharacteristics.AribB67,
}
_PRIMARIES = {
    "bt709": ss2.ColorPrimaries.Bt709, "bt470m": ss2.ColorPrimaries.Bt470M,
    "bt470bg": ss2.ColorPrimaries.Bt470Bg, "st170m": ss2.ColorPrimaries.St170M,
    "st240m": ss2.ColorPrimaries.St240M, "film": ss2.ColorPrimaries.Film,
    "bt2020": ss2.ColorPrimaries.Bt2020, "st428": ss2.ColorPrimaries.St428,
    "st431-2": ss2.ColorPrimaries.St431_2, "st432-1": ss2.ColorPrimaries.St432_1,
    "ebu3213e": ss2.ColorPrimaries.Ebu3213E,
}
_FILTERS = {"bilinear": 0, "bicubic": 1, "lanczos": 2}
_BLURS = {"sampled": ss2.Ssimulacra2Blur.SAMPLED, "recursive": ss2.Ssimulacra2Blur.RECURSIVE}


def raw_norms(result) -> list[float]:
    """The 108 norms channel-major: per channel, per scale, per norm n in
    (0, 1): ssim[c*2+n], ringing[c*4+n], blurring[c*4+2+n] (report.cc:221-232)."""
    out = []
    for c in range(3):
        for scale in result.scales:
            for n in range(2):
                out += [float(scale.avg_ssim[c * 2 + n]), float(scale.avg_edgediff[c * 4 + n]),
                        float(scale.avg_edgediff[c * 4 + 2 + n])]
    return out


def _format(header, opts):
    """The decoder's format with the --input-* overrides applied
    (io.cc:789-794)."""
    f = ss2.ImageFormat.from_buffer_copy(header.format)
    for field in ("range", "matrix", "transfer", "primaries"):
        if opts[field] is not None:
            setattr(f, field, opts[field])
    return f


class _Scorer:
    """Frame pairs -> results, batched, or one pair per call on two pipelines
    in turn (frame i + 1's upload overlaps frame i's kernels)."""

    def __init__(self, width, height, batch, chroma_filter, device, blur=0, half_planes=False):
        self.batch = batch
        if batch > 1:
            self.s = [ss2.Ssimulacra2Batch(max_pairs=batch, chroma_filter=chroma_filter,
                                           device=device, blur=blur, half_planes=half_planes)]
        else:
            self.s = [ss2.Ssimulacra2Pipeline(width, height, chroma_filter=chroma_filter,
                                              device=device, blur=blur,
                                              half_planes=half_planes) for _ in range(2)]

    def score(self, pairs, background):
        if self.batch > 1:
            return self.s[0].compute_many(pairs, background)
        results, pending = [], []
        try:
            for i, (o, d) in enumerate(pairs):
                if len(pending) == 2:
                    p, tok = pending.pop(0)
                    results.append(p.finish(tok))
                p = self.s[i % 2]
                pending.append((p, p.submit(o, d, background)))
            while pending:
                p, tok = pending.pop(0)
                results.append(p.finish(tok))
        finally:
            # After an error, finish what is still in flight before it
            # propagates, so no submission outlives the call (pool.cc:64-72).
            for p, tok in pending:
                try:
                    p.finish(tok)
                except Exception:
                    pass
        return results

    def close(self):
        for s in self.s:
            s.close()




# ---- options (cli/options.cc:211-395) ----------------------------------------

_METRICS = ("ssimulacra2", "butteraugli", "vmaf-v0", "vmaf-v1", "cvvdp", "psnr-hvs")
_RANGES = {"limited": ss2.PixelRange.Limited, "full": ss2.PixelRange.Full}
_COLOR_FLAGS = {"--input-matrix": ("matrix", _MATRICES),
                "--input-transfer": ("transfer", _TRANSFERS),
                "--input-primaries": ("primaries", _PRIMARIES),
                "--input-range": ("range", _RANGES),
                "--chroma-filter": ("chroma_filter", _FILTERS)}

USAGE = """\
Usage: python -m vqm_b200.cli [--metric ssimulacra2] [--raw|--json] [--verbose]
          [--device INDEX] [--half-planes] [--iterations N] [--warmup N]
          [--chroma-filter KERNEL] [--input-matrix M] [--input-transfer T]
          [--input-primaries P] [--input-range R] [--batch N] [--blur MODE]
          original distorted
       python -m vqm_b200.cli --json --pairs-file PAIRS.tsv [options]
       python -m vqm_b200.cli --list-devices

SSIMULACRA 2.1 on CUDA devices. Inputs may be PNG (8/16-bit), JPEG or
progressive YUV4MPEG2; every Y4M frame is scored and the clip score is the mean
of the frame scores. PNG and JPEG use sRGB with BT.709 primaries. Y4M defaults
to the bt470bg matrix, bt709 transfer and primaries, and limited range.
--pairs-file reads tab-separated rows of sample ID, original and distorted path
and prints one JSON object per pair. --iterations repeats whole clips and
reports the one with the median core time; --warmup runs untimed clips first.
--verbose (-v) prints a table of the clip score and frame statistics.
--input-matrix     rgb|bt709|fcc|bt470bg|st170m|st240m|ycgco|bt2020ncl|
                   bt2020cl|chromaticity-derived-ncl|chromaticity-derived-cl|ictcp
--input-transfer   bt709|bt601|bt470m|bt470bg|st240m|linear|log100|log316|xvycc|
                   bt1361|srgb|bt2020-10|bt2020-12|st2084|st428|arib-b67
--input-primaries  bt709|bt470m|bt470bg|st170m|st240m|film|bt2020|st428|st431-2|
                   st432-1|ebu3213e
--input-range      limited|full
--chroma-filter    bilinear|bicubic|lanczos
Beyond VQM's flags: --batch N scores N frame pairs per launch (1: one pair per
call, its kernels replayed as a CUDA graph); --blur sampled|recursive picks
VQM's 13-tap Gaussian or the recursive Gaussian of Cloudinary's ssimulacra2
(opt-in; not VQM's scores).
"""


class UsageError(ValueError):
    """A command line VQM's parser rejects (exit status 2)."""


def parse(argv):
    """The options of one command line, "help", or "list-devices"."""
    o = {"raw": False, "json": False, "verbose": False, "pairs_file": None, "iterations": 1,
         "warmup": 0, "device": None, "half_planes": False, "metrics": [],
         "start_frame": None, "frame_count": None, "matrix": None, "transfer": None,
         "primaries": None, "range": None, "chroma_filter": _FILTERS["bilinear"],
         "batch": 8, "blur": "sampled", "original": None, "distorted": None}
    positional = []
    i = 0

    def value(flag):
        nonlocal i
        if i + 1 >= len(argv):
            raise UsageError(f"{flag} needs a value")
        i += 1
        return argv[i]

    def count(flag, text, zero_ok=True):
        if not text.isdigit() or (not zero_ok and int(text) == 0):
            raise UsageError(f"invalid value for {flag}: '{text}'")
        return int(text)

    while i < len(argv):
        arg = argv[i]
        if arg == "--raw":
            o["raw"] = True
        elif arg == "--json":
            o["json"] = True
        elif arg in ("--verbose", "-v"):
            o["verbose"] = True
        elif arg in ("--start-frame", "--frame-count"):
            o[arg[2:].replace("-", "_")] = count(arg, value(arg), arg == "--start-frame")
        elif arg == "--pairs-file":
            o["pairs_file"] = value(arg)
        elif arg in ("--iterations", "--warmup", "--device", "--batch"):
            n = count(arg, value(arg), arg not in ("--iterations", "--batch"))
            o[arg[2:]] = n
        elif arg == "--list-devices":
            if len(argv) != 1:
                raise UsageError("--list-devices must be used on its own")
            return "list-devices"
        elif arg == "--half-planes":
            o["half_planes"] = True
        elif arg == "--metric":
            for name in value(arg).split(","):
                if name == "all":
                    picked = list(_METRICS)
                elif name in _METRICS:
                    picked = [name]
                else:
                    raise UsageError(f"invalid value for --metric: '{name}' (expected "
                                     "ssimulacra2|butteraugli|vmaf-v0|vmaf-v1|cvvdp|psnr-hvs|all)")
                o["metrics"] += [m for m in picked if m not in o["metrics"]]
        elif arg == "--blur":
            text = value(arg)
            if text not in _BLURS:
                raise UsageError(f"invalid value for --blur: '{text}' (expected sampled|recursive)")
            o["blur"] = text
        elif arg in ("--help", "-h"):
            return "help"
        elif arg in _COLOR_FLAGS:
            field, names = _COLOR_FLAGS[arg]
            text = value(arg)
            if text not in names:
                raise UsageError(f"invalid value for {arg}: '{text}' (expected {'|'.join(names)})")
            o[field] = names[text]
        elif arg.startswith("-") and arg != "-":
            raise UsageError(f"unknown option '{arg}'")
        else:
            positional.append(arg)
        i += 1
    if not o["metrics"]:
        o["metrics"] = ["ssimulacra2"]
    others = [m for m in o["metrics"] if m != "ssimulacra2"]
    if others:
        raise UsageError(f"this build scores ssimulacra2 only (asked for {','.join(others)})")
    if o["json"] and o["raw"]:
        raise UsageError("--json and --raw cannot be combined")
    if o["verbose"] and o["raw"]:
        raise UsageError("--verbose and --raw cannot be combined")
    if o["pairs_file"] is not None:
        if not o["json"]:
            raise UsageError("--pairs-file requires --json")
        if positional:
            raise UsageError("--pairs-file replaces positional paths")
        return o
    if len(positional) != 2:
        raise UsageError(f"expected exactly two image paths, got {len(positional)}")
    o["original"], o["distorted"] = positional
    return o


def read_pairs(path):
    """(sample ID, original, distorted) rows of a pairs file
    (cli/video.cc:52-80)."""
    try:
        with open(path, newline="") as f:
            text = f.read()
    except OSError as e:
        raise RuntimeError(f"cannot open pairs file: {path}") from e
    pairs, ids = [], set()
    lines = text.split("\n")
    if lines[-1] == "":
        lines.pop()  # the end of the last row, or an empty file
    for line in lines:
        line = line[:-1] if line.endswith("\r") else line
        parts = line.split("\t", 2)
        if len(parts) != 3 or not all(parts) or "\t" in parts[2]:
            raise ss2.InvalidArgument("expected ID, original, distorted TSV")
        if parts[0] in ids:
            raise ss2.InvalidArgument(f"duplicate sample ID: {parts[0]}")
        ids.add(parts[0])
        pairs.append(tuple(parts))
    if not pairs:
        raise ss2.InvalidArgument("empty pair list")
    return pairs


def list_devices(out) -> None:
    """One line per CUDA device: index, name, kind and UUID, as VQM's
    --list-devices lists its Vulkan devices (cli/main.cc:71-88)."""
    devices = ss2.list_devices()
    if not devices:
        print("No CUDA devices found.", file=out)
        return
    kinds = {1: "integrated GPU", 2: "discrete GPU"}
    for i, d in enumerate(devices):
        print(f"{i}  {d.name}  ({kinds.get(d.type, 'other')})  {d.uuid_text()}", file=out)


def _device_count() -> int:
    return len(ss2.list_devices())


# ---- scoring (cli/video.cc:419-506) -------------------------------------------

def _scorer(cache, o, width, height, device):
    """The scorer for this frame size, kept across pairs and iterations (VQM
    keeps its metric pipelines per input key, cli/video.cc:300-385): a batch
    scorer takes any size, one-pair pipelines are per size."""
    key = (width, height) if o["batch"] <= 1 else None
    if key not in cache:
        cache[key] = _Scorer(width, height, max(1, o["batch"]), o["chroma_filter"], device,
                             _BLURS[o["blur"]], o["half_planes"])
    return cache[key]


def _score_clip(o, original, distorted, device, world, rank, cache):
    """One clip of a pair: (frames as (score, raw norms), core seconds,
    decode seconds), this rank's frames gathered on rank 0."""
    t = time.perf_counter()
    ro = stills.open_sequence(original)
    try:
        rd = stills.open_sequence(distorted)
    except Exception:
        ro.close()
        raise
    decode = time.perf_counter() - t
    core = 0.0
    frames = []
    try:
        ho, hd = ro.header, rd.header
        if (ho.width, ho.height) != (hd.width, hd.height):
            raise ss2.InvalidArgument("Image size mismatch")
        if isinstance(ro, stills.StillReader) != isinstance(rd, stills.StillReader):
            raise ss2.InvalidArgument("inputs require two images or two Y4M sequences")
        if ho.fps != hd.fps:
            raise ss2.InvalidArgument("inputs have unequal frame rates")
        ro.format, rd.format = _format(ho, o), _format(hd, o)
        alpha = ro.format.alpha != ss2.AlphaType.None_ or rd.format.alpha != ss2.AlphaType.None_
        total, todo, first = None, None, 0
        if world > 1:
            total = ro.remaining()
            if rd.remaining() != total:
                raise ss2.InvalidArgument("inputs have unequal frame counts")
            mine = replicas.contiguous(total, world)[rank]
            ro.skip(mine.start)
            rd.skip(mine.start)
            todo, first = len(mine), mine.start
        scorer = _scorer(cache, o, ho.width, ho.height, device)
        io_, id_ = iter(ro), iter(rd)
        while todo is None or len(frames) < todo:
            t = time.perf_counter()
            chunk = []
            want = o["batch"] if todo is None else min(o["batch"], todo - len(frames))
            for _ in range(max(1, want)):
                a, b = next(io_, None), next(id_, None)
                if (a is None) != (b is None):
                    raise ss2.InvalidArgument("inputs have unequal frame counts")
                if a is None:
                    break
                chunk.append((a, b))
            decode += time.perf_counter() - t
            if not chunk:
                break
            t = time.perf_counter()
            if alpha:
                # The worse of the dark and bright backgrounds
                # (include/vqm_alpha.h:17-28).
                dark = scorer.score(chunk, 0.1)
                bright = scorer.score(chunk, 0.9)
                picked = [x if x.score() <= y.score() else y for x, y in zip(dark, bright)]
            else:
                picked = scorer.score(chunk, 0.5)
            core += time.perf_counter() - t
            frames += [(r.score(), raw_norms(r) if o["raw"] else None) for r in picked]
    finally:
        ro.close()
        rd.close()
    if world > 1:
        import torch.distributed as dist
        frames = replicas.gather_ordered(frames, first, total)
        times = [None] * world
        dist.all_gather_object(times, (core, decode))
        core, decode = max(t[0] for t in times), max(t[1] for t in times)
    return frames, core, decode


def _stats(scores):
    """frame_stats of report.cc:46-68 (perfect: 100)."""
    finite = [s for s in scores if math.isfinite(s)]
    return {"min": min(scores), "max": max(scores),
            "finite_mean": statistics.fmean(finite) if finite else None,
            "finite_stddev": statistics.pstdev(finite) if finite else None,
            "infinite_frames": len(scores) - len(finite),
            "perfect_frames": sum(1 for s in scores if s == 100.0)}


def _print_clip(o, sample_id, frames, core, decode, out):
    """report.cc:249-276 for one metric."""
    scores = [s for s, _ in frames]
    clip = statistics.fmean(scores)
    if not math.isfinite(clip):
        raise RuntimeError("non-finite clip score")
    fps = len(frames) / core if core > 0 else None
    if o["json"]:
        doc = {"sample_id": sample_id, "metric": "ssimulacra2", "score": clip,
               "frames": len(frames), "core_seconds": core, "decode_seconds": decode}
        if o["verbose"]:
            doc["scoring_fps"] = fps
            doc["frame_stats"] = _stats(scores)
        doc["frame_results"] = [{"index": i, "score": s} for i, s in enumerate(scores)]
        print(json.dumps(doc), file=out)
        return
    if o["verbose"]:
        st = _stats(scores)
        g = lambda v: "n/a" if v is None else f"{v:.8g}"  # noqa: E731
        print(f"Frames: {len(frames)}", file=out)
        print(f"Scoring FPS: {'n/a' if fps is None else f'{fps:.2f}'}", file=out)
        print(f"{'Metric':<12} {'Aggregate':>15} {'Frame min':>15} {'Frame max':>15} "
              f"{'Finite stddev':>15} {'Perfect':>8}", file=out)
        print(f"{'ssimulacra2':<12} {g(clip):>15} {g(st['min']):>15} {g(st['max']):>15} "
              f"{g(st['finite_stddev']):>15} {st['perfect_frames']:>8}", file=out)
        return
    if o["raw"]:
        for _, raw in frames:
            print("".join(f"{v:.12f}," for v in raw), file=out)
    print(f"{clip:.8f}", file=out)


def run(argv=None, out=sys.stdout) -> int:
    """The CLI on `argv`; raises UsageError for a rejected command line and
    the scorer's or the readers' errors for a failed one."""
    o = parse(list(sys.argv[1:] if argv is None else argv))
    if o == "help":
        print(USAGE, end="", file=out)
        return 0
    if o == "list-devices":
        list_devices(out)
        return 0
    if o["start_frame"] is not None or o["frame_count"] is not None:
        raise ss2.InvalidArgument("--start-frame and --frame-count apply to compressed video "
                                  "inputs, which this build does not decode")
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    device = -1 if o["device"] is None else o["device"]
    if world > 1:
        import torch
        import torch.distributed as dist
        dist.init_process_group("gloo", timeout=datetime.timedelta(seconds=600))
        # One GPU per rank; ranks beyond the GPU count share them (their
        # work is independent).
        device = int(os.environ.get("LOCAL_RANK", str(rank))) % max(1, torch.cuda.device_count())
    elif o["device"] is not None and o["device"] >= _device_count():
        raise ss2.InvalidArgument(f"--device {o['device']} is unavailable. Run --list-devices "
                                  "to see available indexes.")
    cache = {}
    try:
        pairs = (read_pairs(o["pairs_file"]) if o["pairs_file"] is not None
                 else [("pair", o["original"], o["distorted"])])
        for sample_id, original, distorted in pairs:
            for _ in range(o["warmup"]):
                _score_clip(o, original, distorted, device, world, rank, cache)
            runs = sorted((_score_clip(o, original, distorted, device, world, rank, cache)
                           for _ in range(o["iterations"])), key=lambda r: r[1])
            frames, core, decode = runs[len(runs) // 2]
            if not frames:
                raise ss2.InvalidArgument("input sequence has no frames")
            if rank == 0:
                _print_clip(o, sample_id, frames, core, decode, out)
    finally:
        for scorer in cache.values():
            scorer.close()
        if world > 1:
            import torch.distributed as dist
            dist.destroy_process_group()
    return 0


def main(argv=None) -> int:
    """Exit status as VQM's CLI: 2 and the usage for a rejected command line,
    1 for a failure while scoring (cli/main.cc:115-173)."""
    try:
        return run(argv)
    except UsageError as e:
        print(f"{e}\n{USAGE}", end="", file=sys.stderr)
        return 2
    except (ValueError, RuntimeError, OSError) as e:
        print(f"{e}", file=sys.stderr)
        return 1


if __name__ == "__main__":
    sys.exit(main())
