import glob
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "oracle"))

GOLDEN = os.path.join(ROOT, "tests", "golden")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200, sm_100a)")


def golden_cases():
    return sorted(glob.glob(os.path.join(GOLDEN, "ref_*.npz")))


def load_golden(path):
    d = np.load(path)
    return {k: d[k] for k in d.files}


@pytest.fixture(scope="session")
def handle():
    import mxc_b200 as m

    h = m.Handle(0)
    yield h
    h.close()
