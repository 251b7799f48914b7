import json
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
GOLDEN = os.path.join(ROOT, "tests", "golden")
for p in (ROOT, os.path.join(ROOT, "oracle")):
    if p not in sys.path:
        sys.path.insert(0, p)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200) and the built libqubo_b200.so")
    config.addinivalue_line("markers", "slow: long-running full-size case")


def load_golden(name: str) -> dict:
    with open(os.path.join(GOLDEN, name)) as f:
        return json.load(f)


def dec_q(rec: dict) -> np.ndarray:
    dt = np.dtype(rec["dtype"])
    if np.issubdtype(dt, np.integer):
        return np.array(rec["data"], dtype=np.int64).astype(dt)
    return np.array([[float.fromhex(v) for v in row] for row in rec["data"]], dtype=np.float64).astype(dt)


def bits_to_int(s: str) -> int:
    return int(s, 2) if s else 0


@pytest.fixture(scope="session")
def cuda_ok():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    return True
