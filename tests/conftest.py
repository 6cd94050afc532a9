import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
for p in (ROOT, os.path.join(ROOT, "oracle")):
    if p not in sys.path:
        sys.path.insert(0, p)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200, sm_100a)")
    # temporary files of the tests stay inside the repository (git-ignored)
    if config.option.basetemp is None:
        config.option.basetemp = os.path.join(ROOT, "tests", ".tmp")


def has_gpu() -> bool:
    try:
        import torch

        return torch.cuda.is_available()
    except Exception:
        return False


@pytest.fixture(scope="session")
def ref_oracle():
    """The reference built from its own sources (oracle/_ref); skipped when absent."""
    import mercury_oracle

    if not mercury_oracle.available():
        pytest.skip("oracle/_ref/mercury_ref not built (make -C oracle REF=<reference sources>)")
    return mercury_oracle
