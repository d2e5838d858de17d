"""Shared test setup: import paths, the `gpu` marker and GPU fixtures."""
import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
for p in (os.path.join(ROOT, "ssmproblems.jl_b200"), os.path.join(ROOT, "oracle"), ROOT):
    if p not in sys.path:
        sys.path.insert(0, p)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA B200 (runs the libgfb200 kernels)")


@pytest.fixture(scope="session")
def ctx():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    import gfb200
    c = gfb200.default_context(0)
    yield c


@pytest.fixture(scope="session")
def oracle():
    import oracle as O
    O.build()
    return O
