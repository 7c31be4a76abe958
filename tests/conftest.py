import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

GOLDEN = os.path.join(ROOT, "tests", "golden")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200) and the built CUDA library")


def golden_cases(prefix=None, kind="nufft"):
    names = sorted(f[:-4] for f in os.listdir(GOLDEN) if f.endswith(".npz"))
    toep = [n for n in names if n.startswith("toep")]
    lowrank = [n for n in names if n.startswith("lowrank")]
    sparse = [n for n in names if n.startswith("sparse")]
    cgsense = [n for n in names if n.startswith("cgsense")]
    calib = [n for n in names if n.startswith("calib")]
    dcf = [n for n in names if n.startswith("dcf")]
    if kind == "dcf":
        return dcf
    if kind == "cgsense":
        return cgsense
    if kind == "calib":
        return calib
    if kind == "toeplitz":
        return toep
    if kind == "lowrank":
        return lowrank
    if kind == "sparse":
        return sparse
    other = set(toep) | set(lowrank) | set(sparse) | set(cgsense) | set(calib) | set(dcf)
    return [n for n in names if n not in other]


@pytest.fixture
def load_golden():
    import numpy as np

    def _load(name):
        return dict(np.load(os.path.join(GOLDEN, name + ".npz")))

    return _load
