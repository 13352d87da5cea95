import sys
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parents[1]
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))
GOLDEN = Path(__file__).resolve().parent / "golden"


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200) and the built libvrc.so")


@pytest.fixture(scope="session")
def ctx():
    from varrcwa_b200.capi import Context
    c = Context(0)
    yield c
    c.close()


def golden(name):
    return dict(np.load(GOLDEN / f"{name}.npz"))


def relerr(a, b):
    a = np.asarray(a)
    b = np.asarray(b)
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


def fourier_blocks(r):
    """Basis-invariant S-matrix view of a device result dict."""
    W0i = np.linalg.inv(r["W0"])
    W1i = np.linalg.inv(r["W1"])
    return {"Tuu": r["W1"] @ r["Tuu"] @ W0i, "Tdd": r["W0"] @ r["Tdd"] @ W1i,
            "Rdu": r["W0"] @ r["Rdu"] @ W0i, "Rud": r["W1"] @ r["Rud"] @ W1i}
