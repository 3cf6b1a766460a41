import os
import sys

import pytest

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
for p in (REPO, os.path.join(REPO, "parallelkde.jl_b200")):
    if p not in sys.path:
        sys.path.insert(0, p)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200) and the built library")


@pytest.fixture(scope="session")
def oracle():
    from oracle import gradepro as og
    og.build_oracle()
    return og


@pytest.fixture(scope="session")
def pk():
    """The host package with the CUDA library loaded (GPU tests only)."""
    import pkde_b200
    pkde_b200.load()
    pkde_b200.context(0)
    return pkde_b200
