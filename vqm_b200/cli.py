"""SSIMULACRA 2.1 of two Y4M sequences or PNG/JPEG images, on the GPU.

    python -m vqm_b200.cli original.y4m distorted.y4m [--raw] [--json] [-v]
    python -m vqm_b200.cli original.png distorted.png

The sequence path of VQM's CLI for this metric (cli/video.cc:175-348,
cli/report.cc:197-248, docs/ssimulacra2.md:3-6): both clips must have the
same frame size, frame count and frame rate; every frame pair is scored
independently and the clip score is the mean of the frame scores, printed
with eight decimals as the last line. A PNG or JPEG file is a one-frame
sequence without a frame rate (`stills.py`, VQM's still formats). Inputs with alpha are scored over the
dark and bright backgrounds (0.1 and 0.9) and the worse score is kept
(include/vqm_alpha.h:17-28). --raw prints each frame's 108 norms in the
channel-major order of the reference tool's tuning build (report.cc:234-248)
before its score; --json prints one JSON object instead.

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

import argparse
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


def _format(header, args):
    f = ss2.ImageFormat.from_buffer_copy(header.format)
    if args.input_range:
        f.range = ss2.PixelRange.Full if args.input_range == "full" else ss2.PixelRange.Limited
    if args.input_matrix:
        f.matrix = _MATRICES[args.input_matrix]
    if args.input_transfer:
        f.transfer = _TRANSFERS[args.input_transfer]
    if args.input_primaries:
        f.primaries = _PRIMARIES[args.input_primaries]
    return f


class _Scorer:
    """Frame pairs -> results, batched, or one pair per call on two pipelines
    in turn (frame i + 1's upload overlaps frame i's kernels)."""

    def __init__(self, width, height, batch, chroma_filter, device, blur=0):
        self.batch = batch
        if batch > 1:
            self.s = [ss2.Ssimulacra2Batch(max_pairs=batch, chroma_filter=chroma_filter,
                                           device=device, blur=blur)]
        else:
            self.s = [ss2.Ssimulacra2Pipeline(width, height, chroma_filter=chroma_filter,
                                              device=device, blur=blur) for _ in range(2)]

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


def run(argv=None, out=sys.stdout) -> int:
    ap = argparse.ArgumentParser(prog="python -m vqm_b200.cli", description=__doc__.split("\n")[0])
    ap.add_argument("original")
    ap.add_argument("distorted")
    ap.add_argument("--raw", action="store_true", help="print each frame's 108 norms")
    ap.add_argument("--json", action="store_true")
    ap.add_argument("-v", "--verbose", action="store_true")
    ap.add_argument("--input-range", choices=["limited", "full"])
    ap.add_argument("--input-matrix", choices=sorted(_MATRICES))
    ap.add_argument("--input-transfer", choices=sorted(_TRANSFERS))
    ap.add_argument("--input-primaries", choices=sorted(_PRIMARIES))
    ap.add_argument("--chroma-filter", choices=list(_FILTERS), default="bilinear")
    ap.add_argument("--batch", type=int, default=8, help="frame pairs per launch (1 = graphs)")
    ap.add_argument("--device", type=int, default=-1)
    ap.add_argument("--blur", choices=list(_BLURS), default="sampled",
                    help="sampled: VQM's 13-tap Gaussian; recursive: the recursive Gaussian "
                         "of Cloudinary's ssimulacra2 (opt-in; not VQM's scores)")
    args = ap.parse_args(argv)

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    device = args.device
    if world > 1:
        import torch
        import torch.distributed as dist
        dist.init_process_group("gloo", timeout=datetime.timedelta(seconds=600))
        # One GPU per rank; ranks beyond the GPU count share them (their
        # work is independent).
        device = int(os.environ.get("LOCAL_RANK", str(rank))) % max(1, torch.cuda.device_count())
    ro = stills.open_sequence(args.original)
    try:
        rd = stills.open_sequence(args.distorted)
    except Exception:
        ro.close()
        raise
    try:
        ho, hd = ro.header, rd.header
        if (ho.width, ho.height) != (hd.width, hd.height):
            raise y4m.Y4mError("clips differ in frame size")
        if ho.fps != hd.fps:
            raise y4m.Y4mError("clips differ in frame rate")
        ro.format, rd.format = _format(ho, args), _format(hd, args)
        alpha = ro.format.alpha != ss2.AlphaType.None_ or rd.format.alpha != ss2.AlphaType.None_
        total = None
        todo = None  # frames this rank scores; None: to the end
        if world > 1:
            total = ro.remaining()
            if rd.remaining() != total:
                raise y4m.Y4mError("clips differ in frame count")
            mine = replicas.contiguous(total, world)[rank]
            ro.skip(mine.start)
            rd.skip(mine.start)
            todo = len(mine)
        scorer = _Scorer(ho.width, ho.height, max(1, args.batch), _FILTERS[args.chroma_filter],
                         device, _BLURS[args.blur])
        frames = []  # (score, raw norms)
        t0 = time.perf_counter()
        io, idis = iter(ro), iter(rd)
        while todo is None or len(frames) < todo:
            chunk = []
            want = max(1, args.batch) if todo is None else min(max(1, args.batch),
                                                                todo - len(frames))
            for _ in range(want):
                a, b = next(io, None), next(idis, None)
                if (a is None) != (b is None):
                    raise y4m.Y4mError("clips differ in frame count")
                if a is None:
                    break
                chunk.append((a, b))
            if not chunk:
                break
            if alpha:
                dark = scorer.score(chunk, 0.1)
                bright = scorer.score(chunk, 0.9)
                picked = [x if x.score() <= y.score() else y for x, y in zip(dark, bright)]
            else:
                picked = scorer.score(chunk, 0.5)
            frames += [(r.score(), raw_norms(r) if args.raw else None) for r in picked]
        seconds = time.perf_counter() - t0
        scorer.close()
    finally:
        ro.close()
        rd.close()
    if world > 1:
        import torch.distributed as dist
        frames = replicas.gather_ordered(frames, mine.start, total)
        slowest = [None] * world
        dist.all_gather_object(slowest, seconds)
        seconds = max(slowest)
        dist.destroy_process_group()
        if rank != 0:
            return 0
    if not frames:
        raise y4m.Y4mError("clips have no frames")

    scores = [s for s, _ in frames]
    clip = statistics.fmean(scores)
    if args.json:
        doc = {"metric": "ssimulacra2", "score": clip, "frames": len(frames),
               "frame_scores": scores, "scoring_fps": len(frames) / seconds}
        if args.raw:
            doc["frame_norms"] = [raw for _, raw in frames]
        print(json.dumps(doc), file=out)
        return 0
    if args.verbose:
        finite = [s for s in scores if math.isfinite(s)]
        print(f"Frames: {len(frames)}", file=out)
        print(f"Scoring FPS: {len(frames) / seconds:.2f}", file=out)
        print(f"{'Metric':<12} {'Aggregate':>15} {'Frame min':>15} {'Frame max':>15} "
              f"{'Finite stddev':>15} {'Perfect':>8}", file=out)
        sd = statistics.pstdev(finite) if len(finite) > 1 else 0.0
        print(f"{'SSIMULACRA2':<12} {clip:>15.8g} {min(scores):>15.8g} {max(scores):>15.8g} "
              f"{sd:>15.8g} {sum(1 for s in scores if s == 100.0):>8}", file=out)
    if args.raw:
        for _, raw in frames:
            print(",".join(f"{v:.12f}" for v in raw) + ",", file=out)
    print(f"{clip:.8f}", file=out)
    return 0


def main(argv=None) -> int:
    try:
        return run(argv)
    except (y4m.Y4mError, ss2.InvalidArgument, ss2.LogicError) as e:
        print(f"error: {e}", file=sys.stderr)
        return 2


if __name__ == "__main__":
    sys.exit(main())
