"""Shared fixtures: paths, the CPU oracles (checkers only) and the GPU library."""
from __future__ import annotations

import os
import subprocess
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG = os.path.join(ROOT, "electron-phonon-hmc_b200")
ORACLE = os.path.join(ROOT, "oracle")
GOLDEN = os.path.join(ROOT, "tests", "golden")
for p in (PKG, ORACLE):
    if p not in sys.path:
        sys.path.insert(0, p)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200) and libephmc_cuda.so")
    config.addinivalue_line("markers", "slow: long-running")


def golden(name):
    return np.load(os.path.join(GOLDEN, name), allow_pickle=False)


@pytest.fixture(scope="session")
def restated():
    """The project's C restatement of the path (oracle/liboracle.so)."""
    from oracle import RESTATED_SO, Restated
    if not os.path.exists(RESTATED_SO):
        subprocess.run(["make", "-C", ORACLE, "restated"], check=True, capture_output=True)
    return Restated()


@pytest.fixture(scope="session")
def reference():
    """The reference compiled unmodified (oracle/_ref); skipped where it was not built."""
    from oracle import REFERENCE_SO, Reference
    if not os.path.exists(REFERENCE_SO):
        pytest.skip("oracle/_ref not built (needs the reference sources)")
    return Reference()


@pytest.fixture(scope="session")
def gpu():
    """libephmc_cuda.so on a CUDA device; fails loudly when either is missing."""
    import torch
    if not torch.cuda.is_available():
        raise RuntimeError("GPU test requested but no CUDA device is visible")
    import ephmc
    return ephmc.load_library()


def model_from_golden(g):
    from oracle import Model
    return Model(int(g["l1"]), int(g["l2"]), int(g["nt"]), np.array(g["t"]), np.array(g["kappa"]),
                 float(g["mu"]), float(g["omega"]), int(g["flavors"]), beta=float(g["beta"]))
