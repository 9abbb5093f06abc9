import gzip
import hashlib
import json
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

GOLDEN = os.path.join(ROOT, "tests", "golden")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200) and the built libmnmgdl.so")


def load_expected() -> dict:
    with open(os.path.join(GOLDEN, "expected.json")) as f:
        return json.load(f)


def load_input(name: str) -> np.ndarray:
    with gzip.open(os.path.join(GOLDEN, "data", name + ".gz"), "rb") as f:
        raw = f.read()
    return np.frombuffer(raw, dtype="<i4")[: (len(raw) // 8) * 2].reshape(-1, 2).copy()


def sha_rows(rows) -> str:
    return hashlib.sha256(np.ascontiguousarray(rows, dtype="<i4").tobytes()).hexdigest()


@pytest.fixture(scope="session")
def expected():
    return load_expected()


@pytest.fixture(scope="session")
def engine():
    from mnmgdatalog_b200 import Engine
    eng = Engine(0)
    yield eng
    eng.close()
