import os
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200, sm_100a)")
    # Build the extension and the oracle if a fresh checkout has neither.
    lib = os.path.join(ROOT, "vqm_b200", "libvqm_ss2.so")
    if not os.path.exists(lib):
        subprocess.run([sys.executable, "-m", "vqm_b200.build"], cwd=ROOT, check=True)
    from oracle import binding
    if not os.path.exists(binding.LIB_PATH):
        binding.build(reference=bool(binding.REFERENCE_CHECKOUT))


def cuda_available() -> bool:
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


def pytest_collection_modifyitems(config, items):
    if cuda_available():
        return
    skip = pytest.mark.skip(reason="no CUDA device")
    for item in items:
        if "gpu" in item.keywords:
            item.add_marker(skip)
