import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200, sm_100a)")


@pytest.fixture(scope="session", autouse=True)
def _built_libraries():
    """Build the native libraries in-tree once per session if they are missing
    (nvcc cross-compiles here; the GPU box has the same toolchain)."""
    from compute_vp9_b200 import build as B
    need = [os.path.join(B.LIB, "libcvp9_cuda.so"), os.path.join(B.LIB, "libcvp9_synth.so"),
            os.path.join(ROOT, "oracle", "liboracle.so")]
    if not all(os.path.exists(p) for p in need):
        B.build(oracle=True)
    yield


def gpu_available():
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False
