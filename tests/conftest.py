"""Test configuration: `gpu` marks tests that need a B200 (run with -m gpu)."""
import sys
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parent.parent
GOLDEN = ROOT / "tests" / "golden"
sys.path.insert(0, str(ROOT))

FIXTURES = ["flow.net", "flow.txt", "directNet_1k_sm_mu_03.txt", "small_planted.txt"]


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200); run with -m gpu")


def golden(name: str) -> dict:
    with np.load(GOLDEN / (name + ".ref.npz")) as z:
        return {k: z[k] for k in z.files}


@pytest.fixture(scope="session")
def built_lib():
    from relaxmap_b200 import LIB_PATH
    if not LIB_PATH.exists():
        from relaxmap_b200.build import build
        build()
    return LIB_PATH


@pytest.fixture(scope="session")
def oracle_mod():
    from oracle import oracle as O
    O.lib()
    return O
