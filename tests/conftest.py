import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]
sys.path.insert(0, str(ROOT))
sys.path.insert(0, str(ROOT / "oracle"))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200) and the built library")


@pytest.fixture(scope="session")
def oracle():
    import py_oracle
    return py_oracle.Oracle()


@pytest.fixture(scope="session")
def reference():
    import py_oracle
    if not py_oracle.Reference.available():
        pytest.skip("reference build oracle/_ref not present (make -C oracle ref)")
    return py_oracle.Reference()
