import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parent.parent
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (run with -m gpu on a B200)")


@pytest.fixture(scope="session")
def built():
    """Builds the CUDA library and the CPU checkers once per session."""
    from sol_b200 import build
    build.build()
    import oracle
    oracle.build(ref=True)
    return True
