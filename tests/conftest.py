"""Shared test setup: import paths, the `gpu` marker, seeded inputs."""
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
for sub in ("oracle", "linear-massiv_b200"):
    p = os.path.join(ROOT, sub)
    if p not in sys.path:
        sys.path.insert(0, p)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a B200 (sm_100a) GPU")


def philox(seed: int) -> np.random.Generator:
    """Seeded counter-based generator (numpy Philox4x64) for test inputs."""
    return np.random.Generator(np.random.Philox(seed))


@pytest.fixture(scope="session")
def ctx():
    import lmb200

    return lmb200.default_context(0)


@pytest.fixture(scope="session")
def golden_known():
    import json

    with open(os.path.join(ROOT, "tests", "golden", "known_answers.json")) as f:
        return json.load(f)


@pytest.fixture(scope="session")
def golden_regression():
    return np.load(os.path.join(ROOT, "tests", "golden", "oracle_regression.npz"))
