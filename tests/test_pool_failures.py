"""Ssimulacra2Pool's failure path (src/pool.cc:44-109 of the reference):
drain on failure and rethrow the first error; poison the pool when a drain
fails. Failures are made on the host: the Python pool runs over fake batch
scorers that fail where a test says so, and the C++ facade's pool over fakes
of the C ABI calls linked in with ld --wrap (tests/cpp/pool_failure_check.cc).
Neither needs a device. A GPU test then puts an invalid image in the middle
of a real list."""

import os
import shutil
import subprocess

import numpy as np
import pytest

from vqm_b200 import ss2

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


class FakeBatch:
    """Stands in for Ssimulacra2Batch: results are one scale of zeros; a
    pair whose `bad` attribute is set fails the submission, and the finishes
    whose ordinals are in `fail_finish` fail after consuming their token."""

    log = None

    def __init__(self, max_pairs=0, chroma_filter=0, device=-1, half_planes=False, blur=0):
        self.token, self.pending, self.closed = 0, None, False

    def submit(self, pairs, background=0.5, borrow=False):
        if self.pending is not None:
            raise ss2.LogicError("cuda: a batch is in flight; Finish it first")
        if any(getattr(p[0], "bad", False) for p in pairs):
            raise ss2.InvalidArgument("image: invalid in the middle of the list")
        self.token += 1
        self.pending = (self.token, len(pairs))
        FakeBatch.log["submits"] += 1
        return self.token

    def finish(self, token):
        if self.pending is None or self.pending[0] != token:
            raise ss2.InvalidArgument("cuda: no submission with that token")
        n = self.pending[1]
        self.pending = None
        k = FakeBatch.log["finishes"]
        FakeBatch.log["finishes"] += 1
        if k in FakeBatch.log["fail_finish"]:
            raise ss2.CudaError("cuda: the device reported an error")
        return [ss2.Ssimulacra2Result(np.zeros((1, 18))) for _ in range(n)]

    def close(self):
        self.closed = True


class Pair:
    def __init__(self, bad=False):
        self.bad = bad


@pytest.fixture
def pool(monkeypatch):
    FakeBatch.log = {"submits": 0, "finishes": 0, "fail_finish": set()}
    monkeypatch.setattr(ss2, "Ssimulacra2Batch", FakeBatch)
    return ss2.Ssimulacra2Pool(workers=3, chunk=2)


def pairs(n, bad_at=None):
    return [(Pair(i == bad_at), Pair()) for i in range(n)]


def reset():
    FakeBatch.log.update(submits=0, finishes=0, fail_finish=set())


def test_clean_list(pool):
    assert len(pool.compute_many(pairs(10))) == 10
    assert FakeBatch.log["submits"] == FakeBatch.log["finishes"] == 5


def test_failed_submission_drains_and_keeps_the_pool(pool):
    # Pair 6 is in the fourth chunk (chunks of 2, three workers): the first
    # three chunks were submitted and are finished before the error leaves.
    with pytest.raises(ss2.InvalidArgument, match="middle of the list"):
        pool.compute_many(pairs(10, bad_at=6))
    assert FakeBatch.log["submits"] == 3 and FakeBatch.log["finishes"] == 3
    assert all(b.pending is None for b in pool._batches)
    reset()
    assert len(pool.compute_many(pairs(10))) == 10 and pool.workers() == 3


def test_failed_finish_drains_and_keeps_the_pool(pool):
    FakeBatch.log["fail_finish"] = {1}
    with pytest.raises(ss2.CudaError, match="device reported"):
        pool.compute_many(pairs(10))
    assert FakeBatch.log["finishes"] == FakeBatch.log["submits"]
    assert all(b.pending is None for b in pool._batches)
    reset()
    assert len(pool.compute_many(pairs(10))) == 10


def test_failed_drain_poisons_the_pool(pool):
    batches = list(pool._batches)
    FakeBatch.log["fail_finish"] = {1}  # the drain's second finish fails too
    with pytest.raises(ss2.InvalidArgument):  # the interrupting error, not the drain's
        pool.compute_many(pairs(10, bad_at=6))
    assert all(b.closed for b in batches) and pool.workers() == 0
    for call in (lambda: pool.compute_many(pairs(2)), lambda: pool.submit_many(pairs(2))):
        with pytest.raises(ss2.LogicError, match="pool cannot be reused after a failed drain"):
            call()


def test_streamed_lists_drain_on_failure(pool):
    # The first list fills the three workers, so the second list's chunks
    # wait in the queue; its bad chunk is submitted, and fails, while the
    # first list's results are being taken.
    first = pool.submit_many(pairs(6))
    second = pool.submit_many(pairs(6, bad_at=0))
    with pytest.raises(ss2.InvalidArgument, match="middle of the list"):
        pool.results(first)
    # Every chunk in flight was finished; the lists are dropped.
    assert FakeBatch.log["finishes"] == FakeBatch.log["submits"]
    assert all(b.pending is None for b in pool._batches)
    with pytest.raises(ss2.InvalidArgument, match="no list with that ticket"):
        pool.results(second)
    assert len(pool.compute_many(pairs(4))) == 4


def test_cpp_facade_pool_failures(tmp_path):
    cxx = os.environ.get("CXX", "g++")
    if shutil.which(cxx) is None:
        pytest.skip("no C++ compiler")
    out = str(tmp_path / "pool_failure_check")
    wrapped = ["vqm_cu_ss2_batch_create", "vqm_cu_ss2_batch_destroy",
               "vqm_cu_ss2_batch_submit_borrowed", "vqm_cu_ss2_batch_finish",
               "vqm_cu_last_error"]
    libdir = os.path.join(ROOT, "vqm_b200")
    cmd = [cxx, "-std=c++20", "-O1", "-Wall", "-Wextra", "-Werror",
           "-I" + os.path.join(ROOT, "include"),
           os.path.join(ROOT, "tests", "cpp", "pool_failure_check.cc"), "-L" + libdir,
           "-lvqm_ss2", "-Wl,-rpath," + libdir, "-Wl," + ",".join(f"--wrap={w}" for w in wrapped),
           "-o", out]
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    r = subprocess.run([out], capture_output=True, text=True, timeout=60)
    assert r.returncode == 0, r.stdout + r.stderr


@pytest.mark.gpu
def test_invalid_image_in_a_real_list():
    """A real list with an image of the wrong byte count in its third chunk:
    the first chunks are drained, the validation error propagates, and the
    pool then scores the list correctly."""
    from tests import synthetic
    good = [synthetic.rgb_pair(96, 64, 700 + i)[:2] for i in range(8)]
    o, d = good[5]
    broken = ss2.Image(o.width, o.height, o.format, o.data[:-4])
    bad = list(good)
    bad[5] = (broken, d)
    pool, batch = ss2.Ssimulacra2Pool(workers=2, chunk=2), ss2.Ssimulacra2Batch(max_pairs=8)
    try:
        with pytest.raises(ss2.InvalidArgument, match="data size does not match"):
            pool.compute_many(bad)
        got = pool.compute_many(good)
        want = batch.compute_many(good)
    finally:
        pool.close()
        batch.close()
    for g, w in zip(got, want):
        assert np.array_equal(g.norms, w.norms)
