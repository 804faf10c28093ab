"""Shared pytest setup: paths, the `gpu` marker, oracle build."""
import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
for p in (ROOT, os.path.join(ROOT, "quantumclifford.jl_b200"), os.path.join(ROOT, "oracle"), os.path.join(ROOT, "tests")):
    if p not in sys.path:
        sys.path.insert(0, p)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200) and the built libqcb200")


@pytest.fixture(scope="session")
def orc():
    import oracle as _o

    _o.L()
    return _o


@pytest.fixture(scope="session")
def qcb():
    import torch

    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    import qcb200

    qcb200.ensure_init(0)
    return qcb200
