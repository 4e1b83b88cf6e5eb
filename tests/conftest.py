"""Shared test setup: import paths and the `gpu` marker.

`-m "not gpu"` runs here without a GPU (oracle vs reference, golden fixtures,
host logic, C-ABI exports); `-m gpu` runs the CUDA parity tests on a B200.
"""
import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

# Autotuners record launch shapes in a cache file; the tests use a file of their
# own (one per session) instead of the user's cache directory.
if "GG_TUNE_CACHE" not in os.environ:
    import tempfile
    os.environ["GG_TUNE_CACHE"] = os.path.join(tempfile.mkdtemp(prefix="gg_tune_"), "tune.tsv")
for p in (ROOT, os.path.join(ROOT, "graphgolf-cuda_b200"), os.path.join(ROOT, "oracle"),
          os.path.join(ROOT, "tests")):
    if p not in sys.path:
        sys.path.insert(0, p)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200); runs the engine")


def has_gpu():
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


@pytest.fixture(scope="session")
def gpu_available():
    return has_gpu()
