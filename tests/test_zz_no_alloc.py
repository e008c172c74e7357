"""The scoring entry point that allocates nothing (vqm_cu_ss2_compute_noalloc).

It exists for callers that cannot let a library allocate device memory:
their own allocator owns the GPU's memory, or a cudaMalloc/cudaFree would
stall their real-time streams. It keeps all scratch in one fixed 32 MiB
device array instead. These tests call it through the C ABI with device
images and a device result buffer, several times in a row on different
sizes (the array keeps the last call's contents, so a call must not see the
previous call's), and check each result against the allocating pipeline on
the same pair, within the per-feature tolerance the other parity tests use.
They run last so that a failure here leaves every other test already run.
"""

import ctypes

import numpy as np
import pytest

from tests import helpers
from tests import synthetic
from vqm_b200 import ss2

pytestmark = pytest.mark.gpu


def _device_image(img, torch):
    t = torch.from_numpy(img.data).cuda()
    return ss2.DeviceImage.packed(img.width, img.height, img.format, t.data_ptr(), t), t


def _call(o, d, result_ptr, stream=None, background=0.5):
    co, cd = o._c(), d._c()
    status = ss2._lib.vqm_cu_ss2_compute_noalloc(
        ctypes.byref(co), ctypes.byref(cd), ctypes.c_float(background), 0,
        ctypes.c_void_p(stream), ctypes.c_void_p(result_ptr))
    return status, ss2._lib.vqm_cu_last_error().decode()


def _noalloc(o, d, torch, background=0.5):
    do, keep_o = _device_image(o, torch)
    dd, keep_d = _device_image(d, torch)
    result = torch.full((112,), float("nan"), dtype=torch.float64, device="cuda")
    stream = torch.cuda.current_stream()
    status, msg = _call(do, dd, result.data_ptr(), stream.cuda_stream, background)
    assert status == 0, msg
    stream.synchronize()
    out = result.cpu().numpy()
    del keep_o, keep_d
    return out


def _check_against_pipeline(got, o, d):
    with ss2.Ssimulacra2Pipeline(o.width, o.height) as p:
        want = p.compute(o, d)
    scales = want.norms.shape[0]
    assert int(got[109]) == scales and got[110] == 0.0
    norms = got[:18 * scales].reshape(scales, 18)
    assert np.all(got[18 * scales:108] == 0.0)
    assert not helpers.feature_mismatch(norms, want.norms)
    assert abs(ss2.score(norms) - want.score()) <= helpers.SCORE_TOL
    # The score computed on the device from its own norms equals the host's.
    assert abs(got[108] - ss2.score(norms)) <= 1e-9


def test_noalloc_matches_pipeline_call_after_call():
    """1080p 4:2:0, then a small RGB pair, then the 1080p pair again: the
    two 1080p results are identical bit for bit, and each result matches
    the allocating pipeline."""
    import torch
    big = synthetic.yuv_pair(1920, 1080, 22)[:2]
    small = synthetic.rgb_pair(640, 360, 21)[:2]
    first = _noalloc(*big, torch)
    between = _noalloc(*small, torch)
    again = _noalloc(*big, torch)
    # 108 norms, the score, the scale count and the status word (the last
    # of the 112 doubles is not written).
    assert np.array_equal(first[:111], again[:111])
    _check_against_pipeline(first, *big)
    _check_against_pipeline(between, *small)


def test_noalloc_size_limit_follows_row_width():
    """2048x1200 fits the 32 MiB; 1200x2048 (same area, narrower rows padded
    more) is refused with the bytes it needs, and so is 2560x1440."""
    import torch
    wide = synthetic.rgb_pair(2048, 1200, 25)[:2]
    _check_against_pipeline(_noalloc(*wide, torch), *wide)
    result = torch.zeros(112, dtype=torch.float64, device="cuda")
    for w, h in ((1200, 2048), (2560, 1440)):
        o, d, _ = synthetic.rgb_pair(w, h, 23)
        do, ko = _device_image(o, torch)
        dd, kd = _device_image(d, torch)
        status, msg = _call(do, dd, result.data_ptr())
        assert status == 1, (w, h)
        assert f"{w}x{h} pair needs" in msg and "32 MiB" in msg


def test_noalloc_rejects_host_memory_before_any_kernel():
    import torch
    small_o, small_d, _ = synthetic.rgb_pair(64, 64, 24)
    result = torch.zeros(112, dtype=torch.float64, device="cuda")
    ho, hd = small_o._c(), small_d._c()
    status = ss2._lib.vqm_cu_ss2_compute_noalloc(ctypes.byref(ho), ctypes.byref(hd),
                                                 ctypes.c_float(0.5), 0, None,
                                                 ctypes.c_void_p(result.data_ptr()))
    assert status == 1
    assert "device images only" in ss2._lib.vqm_cu_last_error().decode()
    # Device images, but a pinned host buffer for the result: refused by the
    # pointer check, not written by a kernel.
    do, ko = _device_image(small_o, torch)
    dd, kd = _device_image(small_d, torch)
    pinned = torch.zeros(112, dtype=torch.float64, pin_memory=True)
    status, msg = _call(do, dd, pinned.data_ptr())
    assert status == 1 and "result: must be device memory" in msg
    # The same pair then scores normally.
    _check_against_pipeline(_noalloc(small_o, small_d, torch), small_o, small_d)
