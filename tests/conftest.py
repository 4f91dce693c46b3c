import json
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG_DIR = os.path.join(ROOT, "neighborlist-rs_b200")
for p in (ROOT, PKG_DIR):
    if p not in sys.path:
        sys.path.insert(0, p)

GOLDEN = os.path.join(ROOT, "tests", "golden")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200)")


@pytest.fixture(scope="session")
def fixtures():
    """Reference fixture structures: name -> (positions, cell_rows or None)."""
    z = np.load(os.path.join(GOLDEN, "fixtures.npz"))
    out = {}
    for key in z.files:
        if key.endswith("_pos"):
            name = key[:-4]
            cell = z[name + "_cell"]
            out[name] = (z[key], None if not cell.any() else cell)
    return out


@pytest.fixture(scope="session")
def golden_counts():
    with open(os.path.join(GOLDEN, "golden_counts.json")) as f:
        return json.load(f)["counts"]


@pytest.fixture(scope="session")
def oracle():
    import oracle as O

    O.build()
    return O
