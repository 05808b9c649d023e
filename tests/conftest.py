"""Test configuration.

Tests marked ``gpu`` need a B200 and are run with ``-m gpu``; everything else
runs on the CPU.  The checker for the CUDA path is the oracle (oracle/): the
C restatement always, the reference's own compiled route A where it was built.
"""

from __future__ import annotations

import sys
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parents[1]
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200, sm_100a)")
    config.addinivalue_line("markers", "slow: minutes rather than seconds")


@pytest.fixture(scope="session")
def oracle():
    from oracle.oracle import Oracle

    return Oracle("restatement")


@pytest.fixture(scope="session")
def reference():
    from oracle.oracle import Oracle, reference_available

    if not reference_available():
        pytest.skip("the reference's route A is not built here (oracle/_ref)")
    return Oracle("reference")


@pytest.fixture(scope="session")
def dp():
    """The drop-in module.  On a GPU run the CUDA library must load and a
    device must be present -- a missing one is a failure, not a skip."""
    from nricp_b200 import nricp_dp

    return nricp_dp


@pytest.fixture(scope="session")
def device(dp):
    info = dp.device_info()
    assert info["available"], f"no CUDA device: {info['device']}"
    return info


def diagonal(points) -> float:
    p = np.asarray(points)
    return float(np.linalg.norm(p.max(0) - p.min(0)))
