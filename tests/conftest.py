"""Shared test set-up: the package and the oracle on the path, and the `gpu` marker.

Tests marked `gpu` need a B200 and the built library; they fail, never skip, when either is missing, so
a run on a GPU box cannot pass on a fallback. Everything else runs on the CPU.
"""

import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, os.path.join(ROOT, "dinara-align_b200"))
sys.path.insert(0, os.path.join(ROOT, "oracle"))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a B200 and the built CUDA library")


@pytest.fixture(scope="session")
def oracle():
    import oracle as module

    module.lib()
    return module


@pytest.fixture(scope="session")
def da():
    import torch

    assert torch.cuda.is_available(), "a GPU test ran without a GPU"
    import dinara_align

    dinara_align._native.lib()
    return dinara_align
