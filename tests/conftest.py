import sys
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parents[1]
sys.path.insert(0, str(ROOT))

GOLDEN = Path(__file__).resolve().parent / "golden" / "golden.npz"


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200, sm_100a)")
    config.addinivalue_line("markers", "ref: needs the reference-built oracle (oracle/_ref)")


@pytest.fixture(scope="session")
def golden():
    return dict(np.load(GOLDEN))


@pytest.fixture(scope="session")
def ctx():
    from mtl4_b200 import mtl
    c = mtl.context(0)
    mtl._DEFAULT[0] = c
    yield c


def csr_from(golden, prefix):
    from mtl4_b200.problems import CSR
    rp, ci, v = golden[prefix + "_rp"], golden[prefix + "_ci"], golden[prefix + "_val"]
    return CSR(rp.size - 1, rp.size - 1, rp.astype(np.int64), ci.astype(np.int32), v.astype(np.float64))


@pytest.fixture(scope="session")
def need_ref():
    from oracle import oracle as O
    if not O.ref_available():
        pytest.skip("reference-built oracle not present (oracle/_ref)")
    return O
