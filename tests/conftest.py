"""Shared fixtures. GPU tests carry @pytest.mark.gpu; everything else runs on CPU."""
from __future__ import annotations

import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

GOLDEN = os.path.join(ROOT, "tests", "golden")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (run on the B200 box)")
    config.addinivalue_line("markers", "slow: longer CPU test")


@pytest.fixture(scope="session")
def oracle_lib():
    """The CPU oracle (test infrastructure): C restatement of the reference."""
    from camille_b200 import api
    from oracle import build_oracle
    return api.Library(build_oracle.build(), "orc_")


@pytest.fixture(scope="session")
def product_lib():
    """The CUDA library. Built if missing; never replaced by a CPU path."""
    from camille_b200 import api, build
    if not os.path.isfile(api.PRODUCT_LIB):
        build.build()
    return api.product_library()


def load_golden(name: str) -> dict:
    d = np.load(os.path.join(GOLDEN, f"{name}.npz"))
    return {k: d[k] for k in d.files}


def golden_case(name: str):
    from tests.golden.make_golden import OVERSET_WORKLOADS, WORKLOADS
    return (WORKLOADS[name] if name in WORKLOADS else OVERSET_WORKLOADS[name])()
