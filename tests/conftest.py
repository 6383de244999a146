import json
import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

GOLDEN = os.path.join(ROOT, "tests", "golden")
# Where the reference repository is mounted (read-only; its golden data are read in place).
# Set CABANADEM_REFERENCE to another checkout; tests that need it skip when it is absent.
REFERENCE = os.environ.get("CABANADEM_REFERENCE", "/root/reference")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200); run with -m gpu")


@pytest.fixture(scope="session")
def example_inputs():
    from cabanadem_b200.inputs import Inputs
    with open(os.path.join(GOLDEN, "example_inputs.json")) as f:
        raw = json.load(f)
    return {k: Inputs(v) for k, v in raw.items()}


@pytest.fixture(scope="session")
def validation_data():
    """The reference's golden curves (examples/validation_data/*.csv), read in place."""
    d = os.path.join(REFERENCE, "examples", "validation_data")
    if not os.path.isdir(d):
        pytest.skip("reference validation data not mounted here")
    import numpy as np
    out = {}
    for f in os.listdir(d):
        if f.endswith(".csv"):
            out[f[:-4]] = np.loadtxt(os.path.join(d, f), delimiter=",")
    return out
