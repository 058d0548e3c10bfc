import json
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "oracle"))

GOLDEN_DIR = os.path.join(ROOT, "tests", "golden")
sys.path.insert(0, GOLDEN_DIR)  # snap_cases


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a B200 (sm_100a) GPU")
    config.addinivalue_line("markers", "slow: long-running")


@pytest.fixture(scope="session")
def golden():
    with open(os.path.join(GOLDEN_DIR, "golden.json")) as f:
        return json.load(f)


@pytest.fixture(scope="session")
def snap_golden():
    with open(os.path.join(GOLDEN_DIR, "snap_golden.json")) as f:
        return json.load(f)


@pytest.fixture(scope="session")
def order_golden():
    with open(os.path.join(GOLDEN_DIR, "order_golden.json")) as f:
        return json.load(f)


@pytest.fixture(scope="session")
def golden_ranks():
    return dict(np.load(os.path.join(GOLDEN_DIR, "golden_ranks.npz")))


@pytest.fixture(scope="session")
def oracle():
    import oracle_py
    return oracle_py


@pytest.fixture(scope="session")
def gb():
    import graph_analytics_applesilicon_b200 as G
    G.lib()
    return G


def ref_test_sources(n: int) -> list:
    """The reference's exhaustive-check sources (tests/test_main.cpp:286-291)."""
    s = [0, n // 2, n - 1]
    x = 12345
    for _ in range(3):
        x = (x * 6364136223846793005 + 1442695040888963407) & 0xFFFFFFFFFFFFFFFF
        s.append((x >> 33) % n)
    return s


def sha(a) -> str:
    import hashlib
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()
