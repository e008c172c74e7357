"""SSIMULACRA 2.1 throughput on B200.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl reference]

Workload: 64 pairs of 1920x1080 8-bit sRGB planar images (seeded synthetic
textures with 32 uniform rectangles; each pair distorted by Gaussian noise,
Gaussian blur or 8x8 block quantisation), resident in device memory. A step
scores all 64 pairs through the batched path (one launch per stage over every
pair). Reported beside it: the plain one-pair-per-call path on the same
pairs, the end-to-end number through the public API from pinned host memory
(H2D of every image and D2H of every result inside the timed region), the
live roofline of the dominant kernel, the clocks seen during the timed
region and a CPU baseline (the oracle on the host cores), whose results are
also compared with the GPU's for the same pairs.

With one GPU the default line also carries bounded runs of the other
workloads, each with its own clocks: `video_4k` (3840x2160 10-bit 4:2:0
frames, resident and streamed), `uneven` (the 136-pair uneven batch),
`serve` (Poisson requests through the serving loop) and `plain256` (one
small pair per call). `--workload` runs any of them alone at full size.

Multi-GPU: one process per GPU (torchrun), each scoring its own 64 pairs;
no data-path collective (the pairs are independent). Timings are CUDA events
on the launching stream, max over ranks.

`--impl reference` times the CPU implementation of the path (the FP32
restatement of VQM's shaders in oracle/; VQM itself needs Vulkan, which this
machine does not have) on all host threads, on the same 64 pairs, and prints
the same JSON line with "impl": "reference". That arm loads nothing but the
oracle: its pixels come from `workloads.py`, which is numpy only.
"""

from __future__ import annotations

import argparse
import json
import os
import statistics
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

import workloads  # noqa: E402  (numpy only: loads no native code)

METRIC = "SSIMULACRA2 pairs/s 1080p+4K, plain vs batched/served; p50/p99 ms; % HBM peak"
WIDTH, HEIGHT, PAIRS = 1920, 1080, 64
SEED0 = 1000
RESULT_BYTES = 112 * 8  # per pair: 108 norms, score, scale count, status


def rank_env():
    return (int(os.environ.get("RANK", 0)), int(os.environ.get("WORLD_SIZE", 1)),
            int(os.environ.get("LOCAL_RANK", 0)))


# ---------------------------------------------------------------------------
# Inputs: seeded synthetic pairs (workloads.py), generated in spawned worker
# processes before any CUDA call, then wrapped for the scorer that uses them.
# ---------------------------------------------------------------------------


def _pool_map(fn, jobs):
    from concurrent.futures import ProcessPoolExecutor
    import multiprocessing as mp
    workers = min(len(jobs), os.cpu_count() or 1, 16)
    if workers <= 1:
        return [fn(j) for j in jobs]
    with ProcessPoolExecutor(workers, mp_context=mp.get_context("spawn")) as ex:
        return list(ex.map(fn, jobs))


def gen_pairs(jobs):
    """(kind, w, h, seed) jobs -> [(original, distorted)] Planar pairs."""
    return _pool_map(workloads.make_pair, jobs)


def plain_jobs(count, seed0):
    return [("rgb", WIDTH, HEIGHT, seed0 + i) for i in range(count)]


def _gen_frames(job):
    first, last, count, w, h, seed = job
    base = workloads.video_base(count, w, h, seed)
    offsets = workloads.video_offsets(count, seed)
    return [(f,) + workloads.video_frame(f, count, w, h, seed, base, offsets)
            for f in range(first, last)]


def gen_frames(count, w=3840, h=2160, seed=4000):
    chunk = max(1, (count + 15) // 16)
    jobs = [(a, min(a + chunk, count), count, w, h, seed) for a in range(0, count, chunk)]
    frames = [None] * count
    for part in _pool_map(_gen_frames, jobs):
        for f, o, d in part:
            frames[f] = (o, d)
    return frames


def ss2_image(p):
    from vqm_b200 import ss2
    fmt = ss2.ImageFormat.from_buffer_copy(bytes(workloads.FORMAT_FIELDS[p.kind]))
    return ss2.Image(p.width, p.height, fmt, p.data)


def ss2_pairs(pairs):
    return [(ss2_image(o), ss2_image(d)) for o, d in pairs]


def oracle_image(p):
    from oracle import binding as ob
    return ob.Image(p.width, p.height, ob.Format(*workloads.FORMAT_FIELDS[p.kind]), p.data)


def to_device(pairs):
    """ss2 image pairs -> DeviceImage pairs on the current device."""
    import torch
    from vqm_b200 import ss2
    dev = []
    for o, d in pairs:
        to = torch.from_numpy(o.data).cuda()
        td = torch.from_numpy(d.data).cuda()
        dev.append((ss2.DeviceImage.packed(o.width, o.height, o.format, to.data_ptr(), to),
                    ss2.DeviceImage.packed(d.width, d.height, d.format, td.data_ptr(), td)))
    return dev


def pinned(pairs):
    """ss2 image pairs -> the same images in pinned host memory."""
    import torch
    from vqm_b200 import ss2
    out = []
    for o, d in pairs:
        imgs = []
        for img in (o, d):
            buf = torch.empty(img.data.nbytes, dtype=torch.uint8, pin_memory=True).numpy()
            buf[:] = img.data
            imgs.append(ss2.Image(img.width, img.height, img.format, buf))
        out.append(tuple(imgs))
    return out


# ---------------------------------------------------------------------------
# Roofline bookkeeping (the library's own plan and pruning rule)
# ---------------------------------------------------------------------------

# FP32 lane operations the blur must perform per kept pyramid pixel (one
# image pair), counting a fused multiply-add or a division as one: the five
# 13-tap passes in VQM's order (65 horizontal + 65 vertical: no symmetric
# folding), the three products and 31 map and norm-sum operations (SSIM' 11,
# edge maps 8, the six sums and their squares 12).
BLUR_OPS_PER_KEPT_PIXEL = 164
FFMA_LANES_PER_SM = 128


def pair_alg_bytes(width, height, fmt):
    """Algorithmic bytes of one pair: both inputs read once, the FP32 XYB
    pyramid of the kept channels written once and read once, both images.
    Returns (prepare, blur, whole pair)."""
    from vqm_b200 import ss2
    kept = ss2.kept_pixels(width, height)
    inp = 2 * ss2.required_bytes(fmt, width, height)
    pyramid = 2 * 4 * kept
    return inp + pyramid, pyramid, inp + 2 * pyramid


def fp32_roofline(blur_ms, pairs, clocks):
    """The blur against the FP32 issue roof that bounds it: algorithmic lane
    operations per launch over its CUDA-event time, against 128 FFMA lanes
    per SM at the sampled SM clock."""
    import torch
    from vqm_b200 import ss2
    sms = torch.cuda.get_device_properties(torch.cuda.current_device()).multi_processor_count
    mhz = clocks.get("sm_mhz") or clocks.get("sm_max_mhz") or 1965.0
    ops = BLUR_OPS_PER_KEPT_PIXEL * ss2.kept_pixels(WIDTH, HEIGHT) * pairs
    achieved = ops / (blur_ms / 1e3) / 1e12
    peak = sms * FFMA_LANES_PER_SM * mhz * 1e6 / 1e12
    return {"bound": "fp32 issue", "kernel": "blur", "ops_per_kept_pixel": BLUR_OPS_PER_KEPT_PIXEL,
            "achieved": achieved, "peak": peak, "unit": "T lane-op/s", "frac": achieved / peak,
            "peak_basis": f"{sms} SMs x {FFMA_LANES_PER_SM} lanes x {mhz:.0f} MHz"}


class ClockSampler:
    """Samples SM clock and throttle reasons of one GPU while running."""

    REASONS = {"hw_slowdown": 0x8, "hw_thermal_slowdown": 0x40,
               "sw_thermal_slowdown": 0x20, "sw_power_cap": 0x4}

    def __init__(self, device_index: int):
        self.samples, self.reasons, self.max_mhz = [], set(), None
        self._stop = threading.Event()
        self._h = None
        try:
            import pynvml
            pynvml.nvmlInit()
            import torch
            uuid = str(torch.cuda.get_device_properties(device_index).uuid)
            if not uuid.startswith("GPU-"):
                uuid = "GPU-" + uuid
            self._nv = pynvml
            self._h = pynvml.nvmlDeviceGetHandleByUUID(uuid.encode())
            self.max_mhz = pynvml.nvmlDeviceGetMaxClockInfo(self._h, pynvml.NVML_CLOCK_SM)
        except Exception:
            self._h = None
        self._t = threading.Thread(target=self._run, daemon=True)

    def _sample(self):
        nv = self._nv
        self.samples.append(nv.nvmlDeviceGetClockInfo(self._h, nv.NVML_CLOCK_SM))
        mask = nv.nvmlDeviceGetCurrentClocksEventReasons(self._h)
        for name, bit in self.REASONS.items():
            if mask & bit:
                self.reasons.add(name)

    def _run(self):
        while not self._stop.is_set():
            try:
                self._sample()
            except Exception:
                return
            self._stop.wait(0.02)

    def __enter__(self):
        if self._h is not None:
            self._t.start()
        return self

    def __exit__(self, *exc):
        self._stop.set()
        if self._h is not None:
            self._t.join()
            try:
                self._sample()
            except Exception:
                pass

    def summary(self):
        if not self.samples:
            return {"sm_mhz": None, "sm_max_mhz": self.max_mhz, "reasons": ["unsampled"]}
        return {"sm_mhz": statistics.median(self.samples), "sm_max_mhz": self.max_mhz,
                "reasons": sorted(self.reasons), "samples": len(self.samples)}


def peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(path):
        with open(path) as f:
            return float(json.load(f)["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def traffic_per_launch(stage, pairs):
    """Per-launch DRAM bytes (read + write) of `stage` at the default
    workload (64 pairs of 1920x1080), from the ncu summaries under
    profiles/ (their "traffic_bytes_per_launch <stage> <bytes>" lines); None
    for any other workload."""
    import glob
    import re
    if (WIDTH, HEIGHT, pairs) != (1920, 1080, 64):
        return None
    pattern = re.compile(r"traffic_bytes_per_launch\s+(\w+)\s+([0-9.eE+]+)")
    for path in sorted(glob.glob(os.path.join(ROOT, "profiles", "*.md"))):
        with open(path) as f:
            for m in pattern.finditer(f.read()):
                if m.group(1) == stage:
                    return float(m.group(2))
    return None


# ---------------------------------------------------------------------------
# CPU leg: the oracle on the host cores, timed, and as the checker of the
# GPU's results for the same pairs
# ---------------------------------------------------------------------------


def cpu_leg(pairs, gpu_results, threads):
    """Times the oracle on `pairs` (Planar) and compares each result with the
    GPU's (`gpu_results`, one Ssimulacra2Result per pair): returns (pairs/s,
    seconds, parity dict). The comparison uses the parity bound: per feature
    |d| <= 1e-4 |oracle| + 1e-9, pruned features exactly 0."""
    from oracle import binding as ob
    op = [(oracle_image(o), oracle_image(d)) for o, d in pairs]
    ob.compute_many(op[:threads], threads=threads)  # warm-up
    t0 = time.perf_counter()
    norms, scales, scores = ob.compute_many(op, threads=threads)
    dt = time.perf_counter() - t0
    worst_rel, worst_score, bad = 0.0, 0.0, 0
    for i, r in enumerate(gpu_results):
        want = norms[i, : 18 * int(scales[i])]
        got = np.asarray(r.norms, dtype=np.float64).reshape(-1)
        nz = want != 0
        rel = np.abs(got[nz] - want[nz]) / np.abs(want[nz])
        worst_rel = max(worst_rel, float(rel.max()) if rel.size else 0.0)
        worst_score = max(worst_score, abs(r.score() - float(scores[i])))
        ok = np.all(np.abs(got[nz] - want[nz]) <= 1e-4 * np.abs(want[nz]) + 1e-9)
        bad += int(not ok or np.any(got[~nz] != 0.0))
    parity = {"pairs_checked": len(gpu_results), "max_rel_feature_err": worst_rel,
              "max_score_err": worst_score, "pairs_outside_bound": bad,
              "checker": "FP32 oracle (oracle/), outside the timed region"}
    return len(op) / dt, dt, parity


def run_reference(args):
    """The CPU implementation of the path on all host threads, over the same
    64 pairs the GPU arm scores (rank 0 only; other ranks exit at once)."""
    rank, world, _ = rank_env()
    if rank != 0:
        return 0
    from oracle import binding as ob
    threads = os.cpu_count() or 1
    pairs = gen_pairs(plain_jobs(args.pairs, SEED0))
    op = [(oracle_image(o), oracle_image(d)) for o, d in pairs]
    for _ in range(args.warmup):
        ob.compute_many(op, threads=threads)
    t0 = time.perf_counter()
    for _ in range(args.steps):
        ob.compute_many(op, threads=threads)
    dt = time.perf_counter() - t0
    value = len(op) * args.steps / dt
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": "pairs/s",
        "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": 1e3 * dt / args.steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": {"workload": f"{args.pairs} pairs {WIDTH}x{HEIGHT} 8-bit sRGB planar",
                   "pairs_per_step_per_gpu": args.pairs, "parallelism": "host threads"},
        "cpu_baseline": {"value": value, "unit": "pairs/s", "cores": threads, "kind": "port",
                         "sample": f"the same {args.pairs} pairs of {WIDTH}x{HEIGHT} per step as "
                                   f"the GPU arm, {args.steps} steps, FP32 restatement of VQM's "
                                   "shaders"},
        "e2e": {"value": value, "unit": "pairs/s", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)
    return 0


# ---------------------------------------------------------------------------
# Further workloads. Each returns a dict; run alone (--workload) it prints it
# as its own JSON line, and with one GPU the default line carries a bounded
# run of each.
# ---------------------------------------------------------------------------


def _alternating_steps(batches, dev, n, collect=None):
    """n steps over two batch scorers in turn (the host builds one step's
    tables while the device runs the other's); returns the last results."""
    pending = [None, None]
    last = None
    for k in range(n):
        b = batches[k % 2]
        if pending[k % 2] is not None:
            last = b.finish(pending[k % 2])
            if collect is not None:
                collect.append(b.stage_ms())
        pending[k % 2] = b.submit(dev)
    for i in (n % 2, (n + 1) % 2):
        if pending[i] is not None:
            last = batches[i].finish(pending[i])
            if collect is not None:
                collect.append(batches[i].stage_ms())
    return last


def uneven(steps, warmup, count=None):
    """The uneven batch: 128 10-bit 4:2:0 pairs of random sizes plus 8
    odd-sized RGB pairs, scored as one batch per step. Returns (line, planar
    pairs, results of one step)."""
    import torch
    from vqm_b200 import autotune, ss2
    jobs = workloads.uneven_jobs()
    if count is not None and count < len(jobs):  # a smaller case of the same draw
        jobs = jobs[:count]
    planar = gen_pairs(jobs)
    pairs = ss2_pairs(planar)
    dev = to_device(pairs)
    stream = torch.cuda.Stream()
    tuned = autotune.tune(dev, stream=stream.cuda_stream, use_cache=False)
    batches = [ss2.Ssimulacra2Batch(max_pairs=len(dev), variant=tuned.variant) for _ in range(2)]
    for b in batches:
        b.set_stream(stream.cuda_stream)
        b.set_timing(True)
    _alternating_steps(batches, dev, warmup)
    torch.cuda.synchronize()
    stage = []
    start, end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with ClockSampler(torch.cuda.current_device()) as clocks:
        start.record(stream)
        results = _alternating_steps(batches, dev, steps, stage)
        end.record(stream)
        torch.cuda.synchronize()
    ms = start.elapsed_time(end)
    for b in batches:
        b.close()
    ab = [pair_alg_bytes(o.width, o.height, o.format) for o, _ in pairs]
    prep_b, blur_b, whole_b = (sum(x[i] for x in ab) for i in range(3))
    avg = np.sum(np.array(stage), axis=0) / steps
    peak, kind = peaks()
    px = sum(o.width * o.height for o, _ in pairs)
    line = {
        "workload": "uneven", "metric": "pairs/s", "value": len(pairs) * steps / (ms / 1e3),
        "pairs": len(pairs), "megapixels_per_step": px / 1e6, "steps": steps,
        "ms_per_step": ms / steps, "blur_variant": tuned.variant,
        "tuning_blur_ms": {str(k): round(v, 4) for k, v in tuned.blur_ms.items()},
        "stage_ms_per_step": dict(zip(("prepare", "blur", "finalize"), avg.tolist())),
        "roofline": {"prepare_gbs": prep_b / (avg[0] / 1e3) / 1e9,
                     "blur_gbs": blur_b / (avg[1] / 1e3) / 1e9,
                     "step_gbs": whole_b / (ms / steps / 1e3) / 1e9, "peak": peak,
                     "peak_source": kind},
        "clocks": clocks.summary(),
        "config": "128 10-bit 4:2:0 BT.709 limited pairs, W 320-3840 x H 180-2160 (even), "
                  "+ 8 odd-sized 8-bit RGB pairs; resident in HBM; one batch per step"}
    return line, planar, results


SERVE_SIZES = [((640, 360), 0.2), ((1280, 720), 0.3), ((1920, 1080), 0.3), ((2560, 1440), 0.1),
               ((3840, 2160), 0.1)]


def serve(rates, duration, workers, distinct):
    """Poisson request streams through the serving loop; one dict per rate."""
    import torch
    from vqm_b200 import ss2
    per = max(1, distinct)
    jobs = [(kind, w, h, 30000 + 97 * i + 7 * j)
            for i, ((w, h), _) in enumerate(SERVE_SIZES) for kind in ("rgb", "yuv")
            for j in range(per)]
    host = pinned(ss2_pairs(gen_pairs(jobs)))
    by = {}
    for (kind, w, h, _), p in zip(jobs, host):
        size_idx = [s for s, _ in SERVE_SIZES].index((w, h))
        by.setdefault((size_idx, kind), []).append(p)
    probs = np.array([p for _, p in SERVE_SIZES])
    lines = []
    for rate in rates:
        rng = np.random.default_rng(int(rate))
        n = max(int(rate * duration), 200)
        gaps = rng.exponential(1.0 / rate, n)
        sizes = rng.choice(len(SERVE_SIZES), n, p=probs)
        kinds = rng.integers(0, 2, n)
        picks = rng.integers(0, per, n)
        reqs = [by[(int(sizes[i]), ("rgb", "yuv")[int(kinds[i])])][int(picks[i])]
                for i in range(n)]
        with ss2.Ssimulacra2Server(memory_budget=40 << 30, workers=workers,
                                   max_batch_pairs=64) as server:
            # Warm-up: every size and format once, then bursts of the
            # largest pairs so every worker's device memory has grown to its
            # largest batch before the timed stream.
            for key in by:
                server.wait(server.submit(*by[key][0]))
            big = [by[(len(SERVE_SIZES) - 1, kind)][0] for kind in ("rgb", "yuv")]
            burst = [server.submit(*big[k % 2]) for k in range(64 * workers)]
            for t in burst:
                server.wait(t)
            tickets = [None] * n
            late = np.zeros(n)
            t0 = time.perf_counter()
            arrival = t0 + np.cumsum(gaps)

            def produce():
                for i in range(n):
                    wait = arrival[i] - time.perf_counter()
                    if wait > 0:
                        time.sleep(wait)
                    late[i] = max(0.0, time.perf_counter() - arrival[i])
                    tickets[i] = server.submit(*reqs[i])

            th = threading.Thread(target=produce)
            with ClockSampler(torch.cuda.current_device()) as clocks:
                th.start()
                lat = np.zeros(n)
                for i in range(n):
                    while tickets[i] is None:
                        time.sleep(0.0002)
                    _, lat[i] = server.wait(tickets[i])
                th.join()
                t1 = time.perf_counter()
            stats = server.stats()
        total = lat + 1e3 * late  # arrival -> result on the host
        px = sum(reqs[i][0].width * reqs[i][0].height for i in range(n))
        lines.append({
            "workload": "serve", "rate_req_s": rate, "seconds": duration, "requests": n,
            "throughput_req_s": n / (t1 - t0), "megapixels_per_s": px / 1e6 / (t1 - t0),
            "latency_ms_p50": float(np.percentile(total, 50)),
            "latency_ms_p90": float(np.percentile(total, 90)),
            "latency_ms_p99": float(np.percentile(total, 99)),
            "latency_ms_max": float(total.max()),
            "latency_ms_mean": float(total.mean()),
            "server_ms_p50_p99": [float(np.percentile(lat, 50)), float(np.percentile(lat, 99))],
            "submit_late_ms_p99": float(1e3 * np.percentile(late, 99)),
            "batches": int(stats.batches), "largest_batch": int(stats.largest_batch),
            "budget_bytes": int(stats.budget_bytes),
            "peak_device_bytes": int(stats.peak_device_bytes),
            "peak_requested_bytes": int(stats.peak_bytes), "trims": int(stats.trims),
            "clocks": clocks.summary(),
            "config": "Poisson arrivals; sizes 640x360/1280x720/1920x1080/2560x1440/"
                      "3840x2160 at 0.2/0.3/0.3/0.1/0.1; 8-bit RGB or 10-bit 4:2:0 50/50; "
                      f"pinned host inputs; 40 GB budget; {workers} workers"})
    return lines


def video(count):
    """`count` consecutive 3840x2160 10-bit 4:2:0 frame pairs through one
    fixed-shape pipeline (CUDA-graph replay per frame): streamed from pinned
    host memory and resident, frames per second."""
    import torch
    from vqm_b200 import ss2
    w, h = 3840, 2160
    frames = ss2_pairs(gen_frames(count, w, h))
    host = pinned(frames)
    dev = to_device(frames)
    pipe = ss2.Ssimulacra2Pipeline(w, h)
    out = {}
    with ClockSampler(torch.cuda.current_device()) as clocks:
        for name, src in (("streaming", host), ("resident", dev)):
            for o, d in src[:3]:
                pipe.compute(o, d)
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            scores = [pipe.compute(o, d).score() for o, d in src]
            torch.cuda.synchronize()
            dt = time.perf_counter() - t0
            out[name] = {"frames_per_s": count / dt, "clip_mean_score": float(np.mean(scores))}
        # Streaming through two pipelines in turn: frame i + 1's upload (on
        # one pipeline's stream) runs while frame i's kernels run on the
        # other's.
        pipes = [pipe, ss2.Ssimulacra2Pipeline(w, h)]
        for o, d in host[:3]:
            pipes[1].compute(o, d)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        pending, scores = [], []
        for i, (o, d) in enumerate(host):
            if len(pending) == 2:
                p, tok = pending.pop(0)
                scores.append(p.finish(tok).score())
            p = pipes[i % 2]
            pending.append((p, p.submit(o, d)))
        for p, tok in pending:
            scores.append(p.finish(tok).score())
        dt = time.perf_counter() - t0
        out["streaming_two_pipelines"] = {"frames_per_s": count / dt,
                                          "clip_mean_score": float(np.mean(scores))}
        # The same frames as batches of 8 (one launch per stage per 8 frames).
        batch = ss2.Ssimulacra2Batch(max_pairs=8)
        batch.compute_many(dev[:8])  # warm-up: allocation and first kernel loads
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        for a in range(0, count - count % 8, 8):
            batch.compute_many(dev[a:a + 8])
        torch.cuda.synchronize()
        out["resident_batched8"] = {"frames_per_s": (count - count % 8) /
                                    (time.perf_counter() - t0)}
    for p in pipes:
        p.close()
    batch.close()
    return {"workload": "video", "frames": count, "size": [w, h], **out,
            "clocks": clocks.summary(),
            "config": "3840x2160 10-bit 4:2:0 BT.709 limited; reference translating "
                      "1-3 px per frame; distorted: 8x8 quantisation step 8->48 plus "
                      "noise sigma 2; one pipeline, CUDA-graph replay per frame"}


def plain256(calls):
    """The single small pair: latency of one call through the pipeline
    (its kernels replay as one CUDA graph), resident and from host memory."""
    import torch
    from vqm_b200 import ss2
    o, d = ss2_pairs([workloads.pair_plain_256(0)])[0]
    dev = to_device([(o, d)])[0]
    host = pinned([(o, d)])[0]
    pipe = ss2.Ssimulacra2Pipeline(256, 256)
    out = {}
    with ClockSampler(torch.cuda.current_device()) as clocks:
        for name, pair in (("resident", dev), ("host", host)):
            for _ in range(20):
                pipe.compute(*pair)
            torch.cuda.synchronize()
            lat = []
            for _ in range(calls):
                t0 = time.perf_counter()
                score = pipe.compute(*pair).score()
                lat.append(1e3 * (time.perf_counter() - t0))
            out[name] = {"latency_ms_p50": float(np.percentile(lat, 50)),
                         "latency_ms_p99": float(np.percentile(lat, 99)),
                         "pairs_per_s": 1e3 / float(np.mean(lat)), "score": score}
    pipe.close()
    return {"workload": "plain256", **out, "calls": calls, "clocks": clocks.summary(),
            "config": "one 256x256 8-bit sRGB pair (seeded texture, noise sigma 4, "
                      "8x8 quantisation step 16), one pipeline call per pair"}


def _cpu_check(planar, results, sample):
    """The CPU leg on a sample of a workload's pairs (rank 0, one GPU)."""
    threads = os.cpu_count() or 1
    idx = sample if isinstance(sample, list) else list(range(min(sample, len(planar))))
    value, secs, parity = cpu_leg([planar[i] for i in idx], [results[i] for i in idx],
                                  threads)
    return value, secs, threads, idx, parity


def run_workload(args):
    import torch
    torch.cuda.set_device(0)
    if args.workload == "uneven":
        line, planar, results = uneven(args.steps, args.warmup, args.uneven_pairs)
        if not args.skip_cpu:
            value, secs, threads, idx, parity = _cpu_check(planar, results,
                                                           _uneven_sample(planar))
            line["cpu_baseline"] = {"value": value, "unit": "pairs/s", "cores": threads,
                                    "kind": "port", "sample": f"pairs {idx} of the batch, "
                                                              f"{secs:.1f} s wall"}
            line["parity"] = parity
        print(json.dumps(line), flush=True)
    elif args.workload == "serve":
        for line in serve([float(r) for r in args.rates.split(",")], args.duration,
                          args.serve_workers, args.serve_distinct):
            print(json.dumps(line), flush=True)
    elif args.workload == "video":
        print(json.dumps(video(args.frames)), flush=True)
    elif args.workload == "plain256":
        line = plain256(max(200, args.steps * 20))
        if not args.skip_cpu:
            from oracle import binding as ob
            o, d = workloads.pair_plain_256(0)
            t0 = time.perf_counter()
            for _ in range(5):
                ob.compute(oracle_image(o), oracle_image(d))
            line["cpu_port_ms"] = 1e3 * (time.perf_counter() - t0) / 5
            line["cpu_port_threads"] = 1
        print(json.dumps(line), flush=True)
    return 0


def _uneven_sample(planar):
    """Four pairs of the uneven batch for the oracle check: the largest and
    smallest 4:2:0 pairs, the first odd-sized RGB pair and one more 4:2:0
    pair (bounded so the CPU check stays a few seconds)."""
    yuv = [i for i, (o, _) in enumerate(planar) if o.kind == "yuv420p10"]
    rgb = [i for i, (o, _) in enumerate(planar) if o.kind == "srgb8"]
    area = lambda i: planar[i][0].width * planar[i][0].height  # noqa: E731
    pick = []
    if yuv:
        pick += [max(yuv, key=area), min(yuv, key=area), yuv[len(yuv) // 2]]
    if rgb:
        pick.append(rgb[0])
    return sorted(set(pick))


# ---------------------------------------------------------------------------
# Default: the 1080p batched bench line
# ---------------------------------------------------------------------------


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=50)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="vqm_b200", choices=["vqm_b200", "reference"])
    ap.add_argument("--pairs", type=int, default=PAIRS)
    ap.add_argument("--cpu-sample", type=int, default=32)
    ap.add_argument("--skip-cpu", action="store_true")
    ap.add_argument("--skip-extras", action="store_true",
                    help="leave out the bounded video/uneven/serve/plain256 runs")
    ap.add_argument("--batched-only", action="store_true",
                    help="time the batched path only (for profiler runs)")
    ap.add_argument("--variant", type=int, default=None,
                    help="blur kernel variant; default: chosen by the autotuner")
    ap.add_argument("--streams", type=int, default=1, choices=[1, 2],
                    help="streams for the two alternating batch scorers")
    ap.add_argument("--workload", default="plain1080",
                    choices=["plain1080", "uneven", "serve", "video", "plain256"])
    ap.add_argument("--rates", default="200,500,1000,2000", help="serve: requests/s")
    ap.add_argument("--duration", type=float, default=10.0, help="serve: seconds per rate")
    ap.add_argument("--serve-workers", type=int, default=3)
    ap.add_argument("--serve-distinct", type=int, default=3,
                    help="serve: distinct pairs per (size, format)")
    ap.add_argument("--frames", type=int, default=240, help="video: frame pairs")
    ap.add_argument("--uneven-pairs", type=int, default=136,
                    help="uneven: pairs of the draw to use (136 = all)")
    args = ap.parse_args(argv)
    if args.warmup < 3:
        args.warmup = 3
    if args.impl == "reference":
        return run_reference(args)
    if args.workload != "plain1080":
        return run_workload(args)

    rank, world, local = rank_env()
    planar = gen_pairs(plain_jobs(args.pairs, SEED0 + 100_000 * rank))
    extras_wanted = world == 1 and not args.skip_extras and not args.batched_only

    import torch
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                device_id=torch.device("cuda", local))

    from vqm_b200 import autotune, ss2

    def barrier():
        if dist is not None:
            dist.barrier()
        torch.cuda.synchronize()

    def max_over_ranks(x):
        if dist is None:
            return x
        t = torch.tensor([x], dtype=torch.float64, device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        return float(t.item())

    pairs = ss2_pairs(planar)
    dev = to_device(pairs)  # inputs resident in HBM
    stream = torch.cuda.Stream()
    # The blur kernel variant from the project's autotuner, timed on this
    # workload (untimed here; a fresh box has no cache).
    if args.variant is None:
        tuned = autotune.tune(dev, stream=stream.cuda_stream, use_cache=False)
    else:
        tuned = autotune.TuneResult(args.variant, tuple(ss2.blur_variants()[args.variant]))
    # Two batch scorers on one stream, used alternately: while the GPU runs
    # one step, the host prepares the next step's tables on the other.
    batches = [ss2.Ssimulacra2Batch(max_pairs=args.pairs, variant=tuned.variant)
               for _ in range(2)]
    # With --streams 2 the two scorers run on their own streams, so one
    # step's prepare can overlap the previous step's blur on the device.
    streams = [stream, torch.cuda.Stream() if args.streams == 2 else stream]
    for b, s in zip(batches, streams):
        b.set_stream(s.cuda_stream)
        b.set_timing(True)

    _alternating_steps(batches, dev, args.warmup)
    barrier()
    stage_runs = []
    start, end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with ClockSampler(local) as clocks:
        start.record(streams[0])
        streams[1].wait_event(start)
        results = _alternating_steps(batches, dev, args.steps, stage_runs)
        end1 = torch.cuda.Event()
        end1.record(streams[1])
        streams[0].wait_event(end1)
        end.record(streams[0])
        torch.cuda.synchronize()
    stage = np.sum(np.array(stage_runs), axis=0)
    elapsed_ms = max_over_ranks(start.elapsed_time(end))
    barrier()
    scores = [r.score() for r in results]
    value = world * args.pairs * args.steps / (elapsed_ms / 1e3)
    for b in batches:
        b.close()

    # Roofline of the dominant stage, from its live CUDA-event time.
    fmt = pairs[0][0].format
    prep_b, blur_b, pair_b = pair_alg_bytes(WIDTH, HEIGHT, fmt)
    avg = stage / args.steps  # ms per launch
    names = ("prepare", "blur", "finalize")
    dom = int(np.argmax(avg))
    per_launch = {0: prep_b, 1: blur_b, 2: 0}[dom] * args.pairs
    peak, peak_kind = peaks()
    achieved = per_launch / (avg[dom] / 1e3) / 1e9
    traffic = traffic_per_launch(names[dom], args.pairs)

    if args.batched_only:
        if rank == 0:
            print(json.dumps({"metric": METRIC, "value": value, "unit": "pairs/s",
                              "stage_ms_per_step": dict(zip(names, map(float, avg))),
                              "pairs": args.pairs, "steps": args.steps}), flush=True)
        if dist is not None:
            dist.destroy_process_group()
        return 0

    # Plain path: one pair per call, same resident pairs.
    pipe = ss2.Ssimulacra2Pipeline(WIDTH, HEIGHT)
    pipe.set_stream(stream.cuda_stream)
    for o, d in dev[:3]:
        pipe.compute(o, d)
    barrier()
    ps, pe = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    lat = []
    ps.record(stream)
    for o, d in dev:
        t0 = time.perf_counter()
        pipe.compute(o, d)
        lat.append(1e3 * (time.perf_counter() - t0))
    pe.record(stream)
    torch.cuda.synchronize()
    plain_ms = max_over_ranks(ps.elapsed_time(pe))
    plain_value = world * len(dev) / (plain_ms / 1e3)
    pipe.close()

    # End to end through the public API from pinned host memory, over the
    # same step count as the batched number. Eight workers of 4-pair chunks:
    # each chunk's host-to-device copies overlap the kernels of the chunks
    # before it. Each step's list is submitted before the previous step's
    # results are taken, so its uploads start as the previous step's chunks
    # finish; every step still copies its inputs in and reads its results
    # back.
    host = pinned(pairs)
    h2d = sum(o.data.nbytes + d.data.nbytes for o, d in host)
    pool = ss2.Ssimulacra2Pool(workers=8, chunk=4, device=local)
    for _ in range(2):
        pool.compute_many(host)
    barrier()
    t0 = time.perf_counter()
    ticket = pool.submit_many(host)
    for step in range(args.steps):
        nxt = pool.submit_many(host) if step + 1 < args.steps else None
        e2e_scores = [r.score() for r in pool.results(ticket)]
        ticket = nxt
    torch.cuda.synchronize()
    e2e_ms = max_over_ranks(1e3 * (time.perf_counter() - t0))
    pool.close()
    e2e_value = world * args.pairs * args.steps / (e2e_ms / 1e3)
    assert len(e2e_scores) == args.pairs

    extras = {}
    if extras_wanted:
        extras["plain256"] = plain256(400)
        extras["video_4k"] = video(48)
        uneven_line, uneven_planar, uneven_results = uneven(args.steps, args.warmup)
        extras["uneven"] = uneven_line
        extras["serve"] = serve([1000.0], 3.0, 3, 1)[0]

    line = None
    if rank == 0:
        cpu = parity = None
        if world == 1 and not args.skip_cpu:
            value_c, secs, threads, idx, parity = _cpu_check(planar, results, args.cpu_sample)
            cpu = {"value": value_c, "unit": "pairs/s", "cores": threads, "kind": "port",
                   "sample": f"{len(idx)} of the {WIDTH}x{HEIGHT} pairs, "
                             f"{secs:.1f} s wall on {threads} threads"}
            if "uneven" in extras:
                _, _, _, idx_u, parity_u = _cpu_check(uneven_planar, uneven_results,
                                                      _uneven_sample(uneven_planar))
                extras["uneven"]["parity"] = dict(parity_u, pairs=idx_u)
        line = {
            "metric": METRIC, "value": value, "unit": "pairs/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": elapsed_ms / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {"workload": f"{args.pairs} pairs {WIDTH}x{HEIGHT} 8-bit sRGB planar, "
                                   "resident in HBM, batched path (one launch per stage)",
                       "pairs_per_step_per_gpu": args.pairs, "parallelism": f"replicas{world}",
                       "l2": "inputs larger than L2 (796 MB of images per step)",
                       "blur_variant": tuned.variant, "blur_tile": list(tuned.shape),
                       "tuning_blur_ms": {str(k): round(v, 4) for k, v in tuned.blur_ms.items()}},
            "e2e": {"value": e2e_value, "unit": "pairs/s", "h2d_bytes_per_step": h2d,
                    "d2h_bytes_per_step": RESULT_BYTES * args.pairs, "steps": args.steps,
                    "path": "Ssimulacra2Pool(workers=8, chunk=4) on pinned host images, each "
                            "step's list submitted before the previous step's results are taken"},
            "plain": {"value": plain_value, "unit": "pairs/s",
                      "path": "Ssimulacra2Pipeline.compute, one pair per call, resident",
                      "latency_ms_p50": float(np.percentile(lat, 50)),
                      "latency_ms_p99": float(np.percentile(lat, 99))},
            "batched_over_plain": value / plain_value,
            "stage_ms_per_step": {n: float(a) for n, a in zip(names, avg)},
            "roofline": {"bound": "hbm", "kernel": names[dom], "achieved": achieved,
                         "peak": peak, "peak_source": peak_kind, "unit": "GB/s",
                         "frac": achieved / peak, "traffic": traffic,
                         "alg_bytes_per_launch": per_launch},
            "fp32_roofline": fp32_roofline(avg[1], args.pairs, clocks.summary()),
            "step_roofline": {"alg_bytes_per_pair": pair_b,
                              "achieved_gbs": pair_b * value / world / 1e9,
                              "frac": pair_b * value / world / 1e9 / peak},
            "gpu_launches": 2 * args.steps,  # prepare + blur (finalize is the blur's epilogue)
            "clocks": clocks.summary(),
            "cpu_baseline": cpu,
            "parity": parity,
            "score_sample": scores[:3],
            **extras,
        }
        print(json.dumps(line), flush=True)
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
