"""AddressSanitizer and UndefinedBehaviorSanitizer over the library's host
code (vqm_b200/csrc/ss2_host.cc) and the CPU oracle (oracle/ss2_oracle.cc):
tests/cpp/sanitize_check.cc drives formats, decode constants, scale plans,
taps, the score and the oracle over odd sizes, every pixel type and family,
alpha, chroma subsampling and filters, both blur modes and the oracle's
three precisions; any sanitizer report fails the run. (Device code has no
sanitizer here: compute-sanitizer is closed on the GPU pool.)"""

import os
import shutil
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _sanitizing_compiler(tmp_path):
    """The first C++ compiler that links ASan and UBSan runtimes."""
    probe = tmp_path / "probe.cc"
    probe.write_text("int main() { return 0; }\n")
    for cxx in (os.environ.get("CXX_SANITIZE"), "/usr/bin/g++", os.environ.get("CXX"), "g++"):
        if not cxx or shutil.which(cxx) is None:
            continue
        r = subprocess.run([cxx, "-fsanitize=address,undefined", str(probe), "-o",
                            str(tmp_path / "probe")], capture_output=True, timeout=120)
        if r.returncode == 0:
            return cxx
    return None


def test_host_code_and_oracle_under_asan_and_ubsan(tmp_path):
    cxx = _sanitizing_compiler(tmp_path)
    if cxx is None:
        pytest.skip("no C++ compiler with the ASan and UBSan runtimes")
    exe = str(tmp_path / "sanitize_check")
    cmd = [cxx, "-std=c++20", "-O1", "-g", "-fno-omit-frame-pointer", "-ffp-contract=off",
           "-fsanitize=address,undefined", "-fno-sanitize-recover=all",
           "-I/usr/local/cuda/include", "-o", exe,
           os.path.join(ROOT, "tests", "cpp", "sanitize_check.cc"),
           os.path.join(ROOT, "vqm_b200", "csrc", "ss2_host.cc"),
           os.path.join(ROOT, "oracle", "ss2_oracle.cc")]
    build = subprocess.run(cmd, capture_output=True, text=True, timeout=600)
    assert build.returncode == 0, build.stderr[-3000:]
    env = dict(os.environ, ASAN_OPTIONS="detect_leaks=1:abort_on_error=1",
               UBSAN_OPTIONS="print_stacktrace=1:halt_on_error=1")
    env.pop("LD_PRELOAD", None)
    run = subprocess.run([exe], capture_output=True, text=True, timeout=900, env=env)
    assert run.returncode == 0, (run.stdout[-2000:], run.stderr[-4000:])
    assert "sanitize ok" in run.stdout
    assert "runtime error" not in run.stderr
