import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "oracle"))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200); parity tests of the CUDA path")


@pytest.fixture(scope="session")
def golden():
    import numpy as np

    path = os.path.join(ROOT, "tests", "golden", "ref_vectors.npz")
    z = np.load(path)
    names = [str(x) for x in z["_names"]]
    cases = []
    for nm in names:
        c = {k.split("/", 1)[1]: z[k] for k in z.files if k.startswith(nm + "/")}
        c["name"] = nm
        cases.append(c)
    return cases
