"""Shared fixtures.  GPU tests are marked ``gpu``; everything else runs on CPU."""
import json
import sys
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parent.parent
GOLDEN = ROOT / "tests" / "golden"
sys.path.insert(0, str(ROOT))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200)")


def golden_json(name):
    return json.loads((GOLDEN / name).read_text())


def golden_links(name):
    return np.fromfile(GOLDEN / name)


@pytest.fixture(scope="session")
def ctx():
    from msc_project_b200 import Context
    c = Context(0)
    yield c
    c.close()


def q_err(a, b):
    """|dQ| / max(1, |Q|) -- the tolerance measure for Q, which can be ~0."""
    a, b = np.asarray(a), np.asarray(b)
    return float(np.max(np.abs(a - b) / np.maximum(1.0, np.abs(b))))


def rel_err(a, b):
    a, b = np.asarray(a), np.asarray(b)
    return float(np.max(np.abs(a - b) / np.abs(b)))
