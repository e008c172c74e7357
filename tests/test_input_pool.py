"""Handles and the caller-owned input pool of one pipeline, as VQM's tests
state them (tests/metrics/ssimulacra2/pipeline_test.cc:515-720): handles
belong to the pipeline that made them, the pool's buffers have the exact
size of their format and 64-byte aligned starts, a released span is reused
first-fit, a pipeline holds at most 4095 live buffers, and a stale handle
never matches a later buffer however many allocations come between.

Moves (the C++ half of VQM's ownership test) are covered by the C++ facade,
whose pipeline owns its handle through a unique_ptr.
"""

import ctypes

import numpy as np
import pytest

from tests import helpers
from vqm_b200 import ss2

pytestmark = pytest.mark.gpu

BYTE_RGB = helpers.pinned_format(type=ss2.PixelType.Byte)


def test_handles_belong_to_their_pipeline():
    """pipeline_test.cc:515-546: a handle of one pipeline is rejected by
    another, a foreign release is ignored, tokens are distinct and a foreign
    token cannot be finished."""
    o, d = helpers.gradient(0), helpers.gradient(1)
    with ss2.Ssimulacra2Pipeline(o.width, o.height) as first, \
            ss2.Ssimulacra2Pipeline(o.width, o.height) as second:
        a, b = first.upload(o), second.upload(d)
        assert a.slot != b.slot
        with pytest.raises(ss2.InvalidArgument):
            second.compute(a, b)
        second.release(a)  # ignored: not this pipeline's handle
        identity = second.compute(b, b).score()
        token_a = first.submit(a, a)
        token_b = second.submit(b, b)
        assert token_a != token_b
        with pytest.raises(ss2.InvalidArgument):
            second.finish(token_a)
        assert second.finish(token_b).score() == identity == 100.0
        original_identity = first.finish(token_a).score()
        assert first.compute(a, a).score() == original_identity == 100.0
        with pytest.raises(ss2.InvalidArgument):
            first.compute(b, b)
        first.release(a)


def test_input_pool_exact_size_and_ownership():
    """pipeline_test.cc:567-611."""
    w, h = 33, 17
    nbytes = ss2.required_bytes(BYTE_RGB, w, h)
    assert nbytes == 1692
    with ss2.Ssimulacra2Pipeline(w, h, input_bytes=nbytes) as first, \
            ss2.Ssimulacra2Pipeline(w, h, input_bytes=nbytes) as second:
        a = first.allocate_image(BYTE_RGB)
        b = second.allocate_image(BYTE_RGB)
        assert a.bytes == nbytes and b.bytes == nbytes
        assert a.slot != b.slot
        u = first.get_memory_usage()  # the pool is pinned host memory
        assert u.host_bytes == nbytes and u.input_bytes >= nbytes
        assert u.total_bytes - u.host_bytes >= u.pyramid_bytes > 0
        assert first.map_image(a)
        with pytest.raises(ss2.InvalidArgument):
            second.map_image(a)
        with pytest.raises(ss2.InvalidArgument):
            second.submit(a, b)
        second.release(a)  # ignored
        assert second.map_image(b)
        with pytest.raises(ss2.InvalidArgument):
            first.allocate_image(BYTE_RGB)  # the pool holds one image
        assert first.map_image(a)
        first.release(a)
        second.release(b)


def test_input_handle_beyond_old_generation_limit():
    """pipeline_test.cc:613-645: 2^20 allocations and releases later, the
    first (released) handle still matches no buffer."""
    with ss2.Ssimulacra2Pipeline(8, 8, gpu_resident_images=0, streaming_inputs=False,
                                 input_bytes=ss2.required_bytes(BYTE_RGB, 8, 8)) as p:
        stale = p.allocate_image(BYTE_RGB)
        p.release(stale)
        fmt = ctypes.byref(BYTE_RGB)
        handle, size = ctypes.c_uint64(), ctypes.c_size_t()
        allocate, release = ss2._lib.vqm_cu_ss2_allocate_image, ss2._lib.vqm_cu_ss2_release_image
        n = 1 << 20
        for i in range(n):
            assert allocate(p._p, fmt, ctypes.byref(handle), ctypes.byref(size)) == 0
            if i + 1 != n:
                assert release(p._p, handle.value) == 0
        current = ss2.ImageBuffer(handle.value, (8, 8), size.value)
        assert current.slot != stale.slot
        assert p.map_image(current)
        with pytest.raises(ss2.InvalidArgument):
            p.map_image(stale)
        p.release(current)


def test_input_pool_aligns_starts_and_reuses_gaps():
    """pipeline_test.cc:647-682: the second buffer starts at the first's size
    rounded up to 64 bytes; a released span is reused at the same address,
    and the neighbour's bytes are left alone."""
    w, h = 33, 17
    nbytes = ss2.required_bytes(BYTE_RGB, w, h)
    second_offset = (nbytes + 63) // 64 * 64
    with ss2.Ssimulacra2Pipeline(w, h, input_bytes=second_offset + nbytes) as p:
        first = p.allocate_image(BYTE_RGB)
        second = p.allocate_image(BYTE_RGB)
        first_at, second_at = p.map_image(first), p.map_image(second)
        assert second_at - first_at == second_offset
        ctypes.memset(second_at, 0x5A, nbytes)  # VQM: std::memset(second_memory, 0x5a, bytes)
        with pytest.raises(ss2.InvalidArgument):
            p.allocate_image(BYTE_RGB)
        p.release(first)
        replacement = p.allocate_image(BYTE_RGB)
        assert p.map_image(replacement) == first_at
        assert ctypes.string_at(p.map_image(second), nbytes) == b"\x5a" * nbytes
        p.release(replacement)
        p.release(second)


def test_input_handle_capacity():
    """pipeline_test.cc:684-720: 4095 live buffers at most; a released
    handle does not name its replacement."""
    grey = BYTE_RGB.copy(family=ss2.ColorFamily.Grey, matrix=ss2.MatrixCoefficients.Unspecified)
    nbytes = ss2.required_bytes(grey, 8, 8)
    assert nbytes == 64
    with ss2.Ssimulacra2Pipeline(8, 8, gpu_resident_images=0, streaming_inputs=False,
                                 input_bytes=nbytes * 4096) as p:
        buffers = [p.allocate_image(grey) for _ in range(4095)]
        with pytest.raises(ss2.InvalidArgument):
            p.allocate_image(grey)
        old = buffers[1024]
        p.release(old)
        replacement = p.allocate_image(grey)
        assert replacement.slot != old.slot
        with pytest.raises(ss2.InvalidArgument):
            p.map_image(old)
        assert p.map_image(replacement)


def test_devices_and_default_device():
    """vqm_device.h: ListDevices gives each CUDA device's name, UUID and kind;
    SetDefaultDevice makes a config's device -1 that device; an unknown UUID
    is rejected."""
    devices = ss2.list_devices()
    assert devices and all(len(d.uuid) == 16 and d.name for d in devices)
    assert devices[0].type in (1, 2)
    ss2.set_default_device(devices[0].uuid)
    with ss2.Ssimulacra2Pipeline(32, 32) as p:
        assert p.compute(helpers.gradient(0), helpers.gradient(0)).score() == 100.0
    with pytest.raises(ss2.InvalidArgument, match="device UUID"):
        ss2.set_default_device(bytes(16) if devices[0].uuid != bytes(16) else b"\xff" * 16)


@pytest.mark.parametrize("policy", [ss2.MemoryPolicy.AUTOMATIC, ss2.MemoryPolicy.DIRECT,
                                    ss2.MemoryPolicy.STAGED])
def test_memory_policies_score_alike(policy):
    """Every memory policy scores the pool's buffers like the packed images
    (the same planes either way: read in place, or from the device copy
    STAGED makes at submit); STAGED reports its staging and device mirror."""
    o, d = helpers.plain_256_pair()
    nbytes = o.data.nbytes
    with ss2.Ssimulacra2Pipeline(256, 256, input_bytes=2 * ((nbytes + 63) // 64 * 64),
                                 memory_policy=policy) as p:
        want = p.compute(o, d)
        a, b = p.allocate_image(o.format), p.allocate_image(d.format)
        for buf, img in ((a, o), (b, d)):
            ctypes.memmove(p.map_image(buf), img.data.ctypes.data, nbytes)
        assert np.array_equal(p.compute(a, b).norms, want.norms)
        ctypes.memmove(p.map_image(a), d.data.ctypes.data, nbytes)  # rewritten between calls
        assert p.compute(a, b).score() == 100.0
        u = p.get_memory_usage()
        assert u.uses_staging == (policy == ss2.MemoryPolicy.STAGED)
        assert u.input_bytes >= u.host_bytes * (2 if policy == ss2.MemoryPolicy.STAGED else 1)
    with pytest.raises(ss2.InvalidArgument, match="memory policy"):
        ss2.Ssimulacra2Pipeline(32, 32, memory_policy=3)
