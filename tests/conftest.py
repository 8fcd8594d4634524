import json
import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200); runs through libumapb200.so")


@pytest.fixture(scope="session")
def orc():
    from oracle import oracle

    oracle.load()
    return oracle


@pytest.fixture(scope="session")
def pins():
    return json.loads((ROOT / "tests/golden/reference_pins.json").read_text())
