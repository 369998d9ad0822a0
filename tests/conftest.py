import math
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200) and libtbpm_b200.so")
    config.addinivalue_line("markers", "slow: long-running test")


def bessel_series(time_scaled, precision=1e-14, bessel_max=250):
    """Solver._get_bessel_series (tbpm/solver.py:194-224) for tests."""
    import scipy.special as spec
    out = []
    for i in range(bessel_max):
        v = spec.jv(i, time_scaled)
        if abs(v) > precision or abs(spec.jv(i + 1, time_scaled)) > precision:
            out.append(v)
        else:
            return out
    raise ValueError("Bessel_max too low")


def unit_states(n_states, n, seed=1337):
    rng = np.random.default_rng(seed)
    wf = np.exp(2j * np.pi * rng.random((n_states, n)))
    return wf / np.linalg.norm(wf, axis=1, keepdims=True)


def rel_err(a, b):
    a = np.asarray(a)
    b = np.asarray(b)
    return float(np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300))


@pytest.fixture(scope="session")
def graphene_small():
    import tbplas_b200 as tb
    s = tb.make_graphene_sample(16, 12, disorder=1.0, rescale=9.0, seed=7)
    return s


@pytest.fixture(scope="session")
def dos_bes():
    return bessel_series(math.pi)   # dt*rescale = 2*pi/(2*rescale)*rescale


@pytest.fixture(scope="session")
def ac_bes():
    return bessel_series(math.pi / 2)
