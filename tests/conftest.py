"""Shared test set-up.

``gpu`` marks tests that need a CUDA device; everything else runs on CPU.
The oracle library (oracle/liboracle.so) is the checker; the engine under
test is sph_playground_b200/_lib/libsph.so.  Both are built on demand.
"""
import os
import subprocess
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

ORACLE_SO = os.path.join(ROOT, "oracle", "liboracle.so")
ENGINE_SO = os.path.join(ROOT, "sph_playground_b200", "_lib", "libsph.so")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200)")


def _build(target_dir, so):
    if not os.path.exists(so):
        subprocess.run(["make", "-C", target_dir], check=True, capture_output=True)
    return so


@pytest.fixture(scope="session")
def oracle_lib():
    from sph_playground_b200 import abi
    return abi.load(_build(os.path.join(ROOT, "oracle"), ORACLE_SO))


@pytest.fixture(scope="session")
def engine_lib():
    from sph_playground_b200 import abi
    return abi.load(_build(os.path.join(ROOT, "sph_playground_b200", "csrc"), ENGINE_SO))


@pytest.fixture(scope="session")
def cuda_ok():
    import torch
    if not torch.cuda.is_available():
        pytest.fail("a gpu-marked test ran without a CUDA device")
    return True
