"""The scoring entry point that allocates nothing (vqm_cu_ss2_compute_noalloc).

It exists for callers that cannot let a library allocate device memory:
their own allocator owns the GPU's memory, or a cudaMalloc/cudaFree would
stall their real-time streams. It keeps all scratch in one fixed 32 MiB
device array instead. This test calls it through the C ABI with device
images and a device result buffer, twice in a row (the array keeps the last
call's contents, so the second call must not see the first's), and checks
each result against the allocating pipeline on the same pair, within the
per-feature tolerance the other parity tests use. It runs last so that a
failure here leaves every other test already run.
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


def _noalloc(o, d, torch, background=0.5):
    do, keep_o = _device_image(o, torch)
    dd, keep_d = _device_image(d, torch)
    result = torch.full((112,), float("nan"), dtype=torch.float64, device="cuda")
    stream = torch.cuda.current_stream()
    co, cd = do._c(), dd._c()
    status = ss2._lib.vqm_cu_ss2_compute_noalloc(
        ctypes.byref(co), ctypes.byref(cd), ctypes.c_float(background), 0,
        ctypes.c_void_p(stream.cuda_stream), ctypes.c_void_p(result.data_ptr()))
    assert status == 0, ss2._lib.vqm_cu_last_error().decode()
    stream.synchronize()
    out = result.cpu().numpy()
    del keep_o, keep_d
    return out


def test_noalloc_matches_pipeline_twice_in_a_row():
    import torch
    pairs = [synthetic.rgb_pair(640, 360, 21)[:2], synthetic.yuv_pair(1920, 1080, 22)[:2]]
    for o, d in pairs:
        with ss2.Ssimulacra2Pipeline(o.width, o.height) as p:
            want = p.compute(o, d)
        scales = want.norms.shape[0]
        got = _noalloc(o, d, torch)
        assert int(got[109]) == scales and got[110] == 0.0
        norms = got[:18 * scales].reshape(scales, 18)
        assert np.all(got[18 * scales:108] == 0.0)
        assert not helpers.feature_mismatch(norms, want.norms)
        assert abs(ss2.score(norms) - want.score()) <= helpers.SCORE_TOL
        assert abs(got[108] - want.score()) <= 1e-9


def test_noalloc_rejects_oversized_and_host_images():
    import torch
    o, d, _ = synthetic.rgb_pair(2560, 1440, 23)
    do, ko = _device_image(o, torch)
    dd, kd = _device_image(d, torch)
    result = torch.zeros(112, dtype=torch.float64, device="cuda")
    co, cd = do._c(), dd._c()
    status = ss2._lib.vqm_cu_ss2_compute_noalloc(ctypes.byref(co), ctypes.byref(cd),
                                                 ctypes.c_float(0.5), 0, None,
                                                 ctypes.c_void_p(result.data_ptr()))
    assert status == 1
    assert "32 MiB" in ss2._lib.vqm_cu_last_error().decode()
    small_o, small_d, _ = synthetic.rgb_pair(64, 64, 24)
    ho, hd = small_o._c(), small_d._c()
    status = ss2._lib.vqm_cu_ss2_compute_noalloc(ctypes.byref(ho), ctypes.byref(hd),
                                                 ctypes.c_float(0.5), 0, None,
                                                 ctypes.c_void_p(result.data_ptr()))
    assert status == 1
    assert "device images only" in ss2._lib.vqm_cu_last_error().decode()
