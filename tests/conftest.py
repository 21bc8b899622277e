import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
# Root of the reference project's sources, read only by the tests that use
# its own mesh files (skipped where it is absent); the oracle's Makefile reads
# the same variable to compile the reference's kernels.
REFERENCE_ROOT = os.environ.get("EBEM_REFERENCE_ROOT", "/root/reference")


def reference_file(*parts) -> str:
    """Path of a file of the reference project, or skip the calling test
    when the reference sources are not present on this machine."""
    path = os.path.join(REFERENCE_ROOT, *parts)
    if not os.path.exists(path):
        pytest.skip(f"reference file not available: {os.path.join(*parts)}")
    return path


sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "oracle"))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200) and the built libebem.so")


def cuda_available() -> bool:
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


@pytest.fixture(scope="session")
def oracle():
    import oracle as O
    O.build()
    return O
