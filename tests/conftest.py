import json
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

GOLDEN = os.path.join(ROOT, "tests", "golden")
KAT_NAMES = ["h2_sonly", "interface_h2", "h2_ccpvdz", "h2o_ccpvdz"]


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200)")


def load_kat(name):
    with open(os.path.join(GOLDEN, name + ".json")) as f:
        d = json.load(f)
    for k in ("exponents", "coef_s", "coef_p", "coef_d", "coef_f", "coords", "schwrz", "density", "fa_ref"):
        d[k] = np.asarray(d[k], dtype=np.float64)
    return d


@pytest.fixture(scope="session")
def kats():
    return {n: load_kat(n) for n in KAT_NAMES}
