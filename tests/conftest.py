import os
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

GOLDEN = os.path.join(ROOT, "tests", "golden")
if GOLDEN not in sys.path:
    sys.path.insert(0, GOLDEN)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200) and the built library")


def _have_ref_sources() -> bool:
    from oracle import oracle as O
    return O.have_reference_sources()


@pytest.fixture(scope="session")
def oracle_port():
    """The C restatement of the reference (built here if needed)."""
    from oracle import oracle as O
    if not os.path.exists(O.LIB_PATHS["port"]):
        O.build("port")
    return O


@pytest.fixture(scope="session")
def oracle_ref():
    """The reference's own sources compiled against the shim; skipped when
    neither the build nor the sources are present."""
    from oracle import oracle as O
    if not os.path.exists(O.LIB_PATHS["reference"]):
        if not _have_ref_sources():
            pytest.skip("reference build not present")
        O.build("ref")
    return O


@pytest.fixture(scope="session")
def gpu_lib():
    """The CUDA library; GPU tests fail (not skip) when it is missing."""
    import torch
    from mosscap_b200 import capi
    assert torch.cuda.is_available(), "GPU tests need a CUDA device"
    return capi.load()
