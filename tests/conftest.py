import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

GOLDEN = os.path.join(ROOT, "tests", "golden")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200); runs the parity tests through the C ABI")


def golden(name):
    return np.load(os.path.join(GOLDEN, name), allow_pickle=False)


def nonfinite_cases(n=24, seed=11):
    """S with a NaN antenna (whole row and column) and its zero-antenna twin, S with a NaN
    above the diagonal only, and S with NaN/Inf in one kept entry of the lower triangle,
    the imaginary part of a diagonal entry included (returned as a dict): the reference drops the first two antennas alike, never reads
    the upper triangle and raises EigensolverError on the last three."""
    rng = np.random.default_rng(seed)
    a = rng.standard_normal((n, n)) + 1j * rng.standard_normal((n, n))
    s = a @ a.conj().T / n
    np.fill_diagonal(s, 0)
    xyz = rng.uniform(-50, 50, (n, 3))
    zero_ant, nan_ant = s.copy(), s.copy()
    zero_ant[:, 5] = zero_ant[5, :] = 0
    nan_ant[:, 5] = nan_ant[5, :] = np.nan
    upper, lower, both, inf, diag = s.copy(), s.copy(), s.copy(), s.copy(), s.copy()
    upper[3, 7] = np.nan
    lower[7, 3] = np.nan
    both[7, 3] = both[3, 7] = np.nan
    inf[7, 3] = np.inf
    diag[4, 4] = complex(0.5, np.nan)
    return xyz, zero_ant, nan_ant, upper, {"lower": lower, "both": both, "inf": inf, "diag_imag": diag}


@pytest.fixture(scope="session")
def ctx():
    import bipp_b200 as bipp

    c = bipp.Context("GPU")
    yield c
    c.close()
