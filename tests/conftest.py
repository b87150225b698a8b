import os
import subprocess
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

GOLDEN = os.path.join(ROOT, "tests", "golden", "reference_fixtures.npz")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200); run with -m gpu")


def _ensure_built():
    lib = os.path.join(ROOT, "bootcmatchgx_b200", "lib", "libbcmgx.so")
    if not os.path.exists(lib):
        subprocess.run(["make", "-s", "-C", os.path.join(ROOT, "bootcmatchgx_b200", "csrc"), "-j8"], check=True)
    oso = os.path.join(ROOT, "oracle", "_build", "liboracle.so")
    if not os.path.exists(oso):
        subprocess.run(["make", "-s", "-C", os.path.join(ROOT, "oracle")], check=True)


_ensure_built()


@pytest.fixture(scope="session")
def golden():
    return dict(np.load(GOLDEN, allow_pickle=False))


@pytest.fixture(scope="session")
def oracle():
    from oracle import pyoracle
    return pyoracle


@pytest.fixture(scope="session")
def bx():
    import bootcmatchgx_b200
    return bootcmatchgx_b200


@pytest.fixture(scope="session")
def cuda():
    import torch
    if not torch.cuda.is_available():
        pytest.fail("a CUDA device is required for -m gpu tests")
    return torch.device("cuda:0")


def golden_mtx(golden, name):
    key = "mtx__" + name
    n, m = golden[key + "__shape"]
    import scipy.sparse as sp
    A = sp.csr_matrix((golden[key + "__val"], (golden[key + "__row"], golden[key + "__col"])), shape=(n, m))
    A.sort_indices()
    return A
