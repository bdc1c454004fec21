"""Shared fixtures.  GPU tests carry @pytest.mark.gpu; everything else runs on
a machine without a CUDA device (oracle, geometry, host logic, ABI exports)."""
import os
import sys

import pytest

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG = os.path.join(REPO, "multi-block-lbm-gpu_b200")
for p in (PKG, os.path.join(REPO, "oracle"), os.path.join(REPO, "oracle", "ref_harness"), REPO):
    if p not in sys.path:
        sys.path.insert(0, p)
GOLDEN = os.path.join(REPO, "tests", "golden")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200)")
    config.addinivalue_line("markers", "slow: long-running check")


def _ensure_built():
    import build  # multi-block-lbm-gpu_b200/build.py

    if not os.path.exists(build.ORACLE_LIB):
        build.build_oracle()
    if not os.path.exists(build.LIB):
        build.build_lib()


_ensure_built()


@pytest.fixture(scope="session")
def mb():
    import mblbm

    mblbm.load()
    return mblbm


@pytest.fixture(scope="session")
def orc():
    import oracle

    oracle.load()
    return oracle


@pytest.fixture(scope="session")
def cuda_device():
    import torch

    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    return torch.device("cuda:0")
