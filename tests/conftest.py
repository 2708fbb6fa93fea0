"""Shared fixtures.  GPU tests carry @pytest.mark.gpu; everything else runs
on a CPU-only machine."""
import os
import sys

import pytest

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
for p in (REPO, os.path.join(REPO, "oracle"), os.path.join(REPO, "1d-mctdhb_b200")):
    if p not in sys.path:
        sys.path.insert(0, p)

GOLDEN = os.path.join(REPO, "tests", "golden")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200)")


@pytest.fixture(scope="session")
def oracle():
    from oracle import Oracle

    return Oracle()


@pytest.fixture(scope="session")
def reference():
    from oracle import REF_SO, Reference

    if not os.path.exists(REF_SO):
        pytest.skip("compiled reference (oracle/_ref) not built on this machine")
    return Reference()


@pytest.fixture(scope="session")
def gpu():
    import torch

    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    import mctdhb_b200

    mctdhb_b200.load()
    return mctdhb_b200
