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


def random_gauge(U, shape, seed):
    """U'_mu(x) = g(x) U_mu(x) g(x+mu)^dag with random SU(3) g (host numpy)."""
    from oracle import oracle as O
    V = O.volume(shape)
    g = O.generate_G(shape, seed, 1.0).reshape(V, 4, 18)[:, 0]
    G = g[:, 0::2] + 1j * g[:, 1::2]
    G = G.reshape(V, 3, 3)
    M = (U.reshape(V, 4, 18)[:, :, 0::2] + 1j * U.reshape(V, 4, 18)[:, :, 1::2]).reshape(V, 4, 3, 3)
    idx = np.arange(V).reshape(shape)
    out = np.empty_like(M)
    for mu in range(4):
        nb = np.roll(idx, -1, axis=mu).reshape(-1)
        out[:, mu] = G @ M[:, mu] @ np.conj(np.transpose(G[nb], (0, 2, 1)))
    r = np.empty((V, 4, 9, 2))
    r[..., 0] = out.reshape(V, 4, 9).real
    r[..., 1] = out.reshape(V, 4, 9).imag
    return r.reshape(-1)
