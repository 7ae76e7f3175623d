import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200); run with -m gpu")


@pytest.fixture(scope="session")
def oracle():
    from oracle import oracle as O

    O.lib()
    return O


@pytest.fixture(scope="session")
def golden():
    import json

    import numpy as np

    g = ROOT / "tests" / "golden"
    return {"kat": json.loads((g / "kat.json").read_text()), "merkle": dict(np.load(g / "merkle_ref_cpu.npz"))}
