import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
for p in (ROOT, os.path.join(ROOT, "oracle"), os.path.join(ROOT, "tests")):
    if p not in sys.path:
        sys.path.insert(0, p)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200, sm_100a)")
    config.addinivalue_line("markers", "slow: long-running CPU case")


@pytest.fixture(scope="session")
def gpu_lib():
    """The CUDA library, built and loaded; skips nothing -- a GPU test that
    reaches here without a device fails loudly."""
    import torch
    if not torch.cuda.is_available():
        pytest.fail("gpu test collected on a machine without a CUDA device")
    from flowmol_b200 import build as fb
    fb.build()
    from flowmol_b200 import api
    return api.lib()
