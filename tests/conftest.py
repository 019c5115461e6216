"""Shared pytest setup.

Markers: ``gpu`` -- needs a CUDA device (run with ``-m gpu``); everything else
runs on CPU.  The CPU oracle (``oracle/``) is the checker for the CUDA path.
"""
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG = os.path.join(ROOT, "fmm4rbgpu.jl_b200")
for p in (ROOT, PKG):
    if p not in sys.path:
        sys.path.insert(0, p)

NTHREADS = max(1, min(16, os.cpu_count() or 1))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: test needs a CUDA GPU (B200)")


@pytest.fixture(scope="session")
def oracle_mod():
    import oracle

    oracle.lib()
    return oracle


@pytest.fixture(scope="session")
def gpu_ctx():
    import torch

    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    import fmmb200

    ctx = fmmb200.Context(0)
    yield ctx
    ctx.close()


@pytest.fixture
def rng():
    return np.random.default_rng(1234)
