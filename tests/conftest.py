import json
import sys
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parent.parent
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))

GOLDEN = Path(__file__).resolve().parent / "golden"


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200) and libscxpca.so")


@pytest.fixture(scope="session")
def fixtures():
    return json.loads((GOLDEN / "reference_fixtures.json").read_text())


@pytest.fixture(scope="session")
def csr_10x5(fixtures):
    from oracle.rpca import Csr

    c = fixtures["csr_10x5"]
    return Csr(c["indptr"], c["indices"], np.asarray(c["data"], dtype=np.float32), c["shape"])
