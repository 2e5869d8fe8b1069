import os
import subprocess
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)
GOLDEN = os.path.join(ROOT, "tests", "golden")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (run with -m gpu on a B200)")


@pytest.fixture(scope="session")
def oracle_lib():
    """Build the oracle (C restatement) if needed; it compiles anywhere gcc exists."""
    from oracle import orc
    if not os.path.exists(orc.LIB_PATH):
        subprocess.run(["make", "-C", os.path.join(ROOT, "oracle"), "oracle"], check=True, capture_output=True)
    return orc


@pytest.fixture(scope="session")
def ref_lib():
    """The reference build; only present where the reference sources were compiled."""
    from oracle import ref
    if not ref.available():
        pytest.skip("reference build (oracle/_ref/libstormref.so) not present")
    return ref


def golden(name):
    return dict(np.load(os.path.join(GOLDEN, name)))
