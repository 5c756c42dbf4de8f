"""Test configuration: marker registration and import paths.

`gpu`-marked tests need a CUDA device and call the engine through the C ABI;
everything else runs on the CPU (oracle, golden fixtures, host logic, ABI
symbol checks)."""
import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
for p in (os.path.join(ROOT, "algo-fft_b200"), os.path.join(ROOT, "oracle"), ROOT):
    if p not in sys.path:
        sys.path.insert(0, p)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200) and runs the sm_100a kernels")


def _have_gpu() -> bool:
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


HAVE_GPU = _have_gpu()


def pytest_collection_modifyitems(config, items):
    if HAVE_GPU:
        return
    skip = pytest.mark.skip(reason="no CUDA device")
    for it in items:
        if "gpu" in it.keywords:
            it.add_marker(skip)


@pytest.fixture(scope="session", autouse=True)
def _built_library():
    """Builds libgfft.so and the oracle if they are missing (a no-op when the
    in-tree builds are current)."""
    lib = os.path.join(ROOT, "algo-fft_b200", "libgfft.so")
    if not os.path.exists(lib):
        import build  # algo-fft_b200/build.py
        build.build()
    import oracle
    oracle.build()
    yield
