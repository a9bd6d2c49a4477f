import os
import subprocess
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "oracle"))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200)")


@pytest.fixture(scope="session")
def oracle():
    lib = os.path.join(ROOT, "oracle", "liboracle.so")
    src = os.path.join(ROOT, "oracle", "rte_oracle.cpp")
    if not os.path.exists(lib) or os.path.getmtime(lib) < os.path.getmtime(src):
        subprocess.run(["bash", os.path.join(ROOT, "oracle", "build.sh")], check=True,
                       env=dict(os.environ, RTE_REFERENCE_DIR="/nonexistent"))
    import oracle as O
    return O


@pytest.fixture(scope="session")
def rte():
    import doi_b200
    from doi_b200 import build
    build.build()
    return doi_b200


def real_to_complex(u, L):
    """Reference complex SH coefficients of the real function with real-basis coefficients u."""
    u = np.asarray(u, np.float64)
    w = np.zeros(u.shape, np.complex128)
    s2 = np.sqrt(2.0)
    for l in range(L + 1):
        c0 = l * l + l
        w[..., c0] = u[..., c0]
        for m in range(1, l + 1):
            wp = (u[..., c0 + m] - 1j * u[..., c0 - m]) / s2
            w[..., c0 + m] = wp
            w[..., c0 - m] = (-1) ** m * np.conj(wp)
    return w


def rel(a, b):
    a = np.asarray(a)
    b = np.asarray(b)
    nb = np.linalg.norm(b)
    return float(np.linalg.norm(a - b) / (nb if nb > 0 else 1.0))
