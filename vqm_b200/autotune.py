"""Picks the blur kernel variant (output tile shape and CTA size) for a
workload by timing every compiled variant on it.

    from vqm_b200 import autotune, ss2
    best = autotune.tune(pairs)            # times each variant, caches
    batch = ss2.Ssimulacra2Batch(variant=best.variant)

The timing is the blur stage's device time from the batch scorer's CUDA
events (vqm_cu_ss2_batch_stage_ms), median of `repeats` runs after one
warm-up. Results are cached per device name, size class (the pixel count
of the largest pair rounded to a power of two) and compiled variant list in a
JSON file, by default
~/.cache/vqm_b200/blur_variants.json or $VQM_B200_TUNE_CACHE.
"""

from __future__ import annotations

import json
import os
import statistics
from dataclasses import dataclass, field

from . import ss2


@dataclass
class TuneResult:
    variant: int
    shape: tuple
    blur_ms: dict = field(default_factory=dict)  # variant -> median blur ms
    cached: bool = False


def _cache_path() -> str:
    return os.environ.get("VQM_B200_TUNE_CACHE",
                          os.path.join(os.path.expanduser("~"), ".cache", "vqm_b200",
                                       "blur_variants.json"))


def _size_class(pairs) -> int:
    px = max(o.width * o.height for o, _ in pairs)
    return 1 << max(0, (px - 1).bit_length())


def _device_name() -> str:
    try:
        import torch
        return torch.cuda.get_device_name()
    except Exception:
        return "cuda"


def _load() -> dict:
    try:
        with open(_cache_path()) as f:
            return json.load(f)
    except Exception:
        return {}


def _store(data: dict) -> None:
    path = _cache_path()
    try:
        os.makedirs(os.path.dirname(path), exist_ok=True)
        with open(path, "w") as f:
            json.dump(data, f, indent=1)
    except OSError:
        pass  # a read-only home only costs a re-tune


def tune(pairs, repeats: int = 3, use_cache: bool = True, stream: int | None = None,
         variants=None) -> TuneResult:
    """Times every blur variant on `pairs` and returns the fastest."""
    shapes = ss2.blur_variants()
    # The compiled variant list is part of the key: a library with other
    # variants (or another order) never reuses an index tuned for this one.
    signature = ";".join(",".join(str(v) for v in shape) for shape in shapes)
    key = f"{_device_name()}|{_size_class(pairs)}|{signature}"
    if use_cache and variants is None:
        hit = _load().get(key)
        if hit is not None and hit["variant"] < len(shapes):
            return TuneResult(hit["variant"], tuple(shapes[hit["variant"]]),
                              {int(k): v for k, v in hit.get("blur_ms", {}).items()}, True)
    times = {}
    for v in (variants if variants is not None else range(len(shapes))):
        b = ss2.Ssimulacra2Batch(variant=v)
        if stream is not None:
            b.set_stream(stream)
        b.set_timing(True)
        b.compute_many(pairs)
        runs = []
        for _ in range(repeats):
            b.compute_many(pairs)
            runs.append(b.stage_ms()[1])
        times[v] = statistics.median(runs)
        b.close()
    best = min(times, key=times.get)
    if use_cache and variants is None:
        data = _load()
        data[key] = {"variant": best, "shape": list(shapes[best]),
                     "blur_ms": {str(k): t for k, t in times.items()}}
        _store(data)
    return TuneResult(best, tuple(shapes[best]), times, False)
