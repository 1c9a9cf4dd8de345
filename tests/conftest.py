import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

GOLDEN = os.path.join(ROOT, "tests", "golden")
GOLDEN_INPUTS = sorted(f for f in os.listdir(GOLDEN)
                       if f.endswith((".hgr", ".snn", ".axh")) and os.path.exists(os.path.join(GOLDEN, f + ".ref.npz")))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200); run with -m gpu")


@pytest.fixture(scope="session")
def ctx():
    import axoncuda_b200 as ax
    c = ax.Context(0, 8 << 30)
    yield c
    c.close()
