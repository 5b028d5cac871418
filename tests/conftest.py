"""Shared pytest configuration.

Markers:
  gpu -- needs a CUDA device and the built library (run on the B200 box with
         `pytest -m gpu`); everything else runs on a CPU-only machine.
"""
import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))
GOLDEN = Path(__file__).resolve().parent / "golden"


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU and the built lcbinint_b200 library")


@pytest.fixture(scope="session")
def oracle_lib():
    from oracle.oracle import Oracle
    return Oracle()


@pytest.fixture(scope="session")
def ref_lib():
    from oracle.oracle import Reference, have_reference
    if not have_reference():
        pytest.skip("oracle/_ref not built (make -C oracle ref needs the reference sources)")
    return Reference()


@pytest.fixture(scope="session")
def golden():
    import numpy as np

    def load(name):
        return dict(np.load(GOLDEN / name))
    return load
