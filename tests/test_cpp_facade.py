"""The C++ API in include/vqm_cuda.hpp, compiled as a VQM caller would
compile it (g++ -std=c++20, linked against libvqm_ss2.so).

The host checks run without a device; the GPU check scores the reference's
32x32 gradient pairs through Ssimulacra2Pipeline (pixels and Upload) and
Ssimulacra2Pool and compares each result with the FP32 oracle.
"""

import json
import os
import shutil
import subprocess

import numpy as np
import pytest

from tests import helpers

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
SOURCE = os.path.join(ROOT, "tests", "cpp", "facade_check.cc")
LIBDIR = os.path.join(ROOT, "vqm_b200")


@pytest.fixture(scope="module")
def facade_binary(tmp_path_factory):
    cxx = os.environ.get("CXX", "g++")
    if shutil.which(cxx) is None:
        pytest.skip("no C++ compiler")
    out = str(tmp_path_factory.mktemp("facade") / "facade_check")
    cmd = [cxx, "-std=c++20", "-O1", "-Wall", "-Wextra", "-Werror",
           "-I" + os.path.join(ROOT, "include"), SOURCE, "-L" + LIBDIR, "-lvqm_ss2",
           "-Wl,-rpath," + LIBDIR, "-o", out]
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    return out


def test_facade_compiles_and_host_checks(facade_binary):
    r = subprocess.run([facade_binary, "host"], capture_output=True, text=True, timeout=60)
    assert r.returncode == 0, r.stderr


@pytest.mark.gpu
def test_facade_scores_match_oracle(facade_binary):
    r = subprocess.run([facade_binary, "gpu"], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr
    results = [json.loads(line) for line in r.stdout.splitlines() if line.startswith("{")]
    assert [x["path"] for x in results] == (["pipeline"] * 3 + ["uploaded"] + ["pool"] * 3 +
                                            ["recursive"] * 2 + ["recursive_pool"] * 2 +
                                            ["metrics"] * 3 + ["metrics_image"])
    base = helpers.gradient(0)
    expected, recursive = {}, {}
    for v in range(3):
        expected[v] = helpers.oracle_compute(base, helpers.gradient(v))
        recursive[v] = helpers.oracle_compute(base, helpers.gradient(v), blur=1)
    # Pool pairs are (base, base), (base, 1), (base, 2).
    for x in results:
        norms, score = (recursive if x["path"].startswith("recursive") else expected)[x["variant"]]
        if "norms" in x:
            got = np.asarray(x["norms"], dtype=np.float64).reshape(norms.shape)
            bad = helpers.feature_mismatch(got, norms)
            assert not bad, (x["path"], x["variant"], bad[:6])
        assert abs(x["score"] - score) <= helpers.SCORE_TOL, (x["path"], x["score"], score)
    # The recursive blur moves the scores away from the sampled blur's.
    for k in (1, 2):
        assert abs(results[6 + k]["score"] - results[k]["score"]) > 1e-3
    # The unified facade returns the pipeline's score bit for bit.
    for k in range(3):
        assert results[11 + k]["score"] == results[k]["score"]
    assert results[14]["score"] == results[1]["score"]
    assert results[0]["score"] == 100.0
    assert results[4]["score"] == 100.0
