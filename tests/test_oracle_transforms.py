"""The oracle's half-integer transforms against the golden vectors
(scipy.fft type-4 DCT/DST = FFTW REDFT11/RODFT11) and the reference's own
transform-harness inputs (surfaceFFT.cu:383-473)."""
import os

import numpy as np
import pytest

from tertia_b200.abi import QS_REDFT11, QS_RODFT11

G = np.load(os.path.join(os.path.dirname(__file__), "golden", "dtt_golden.npz"))


def rel(a, b):
    return np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300)


@pytest.mark.parametrize("n", [1, 2, 3, 5, 8, 16, 24, 64, 128])
@pytest.mark.parametrize("direct", [False, True])
def test_dtt1d_golden(oracle_lib, n, direct):
    x = G[f"d1_in_{n}"]
    assert rel(oracle_lib.dtt1d(x, QS_REDFT11, direct), G[f"d1_dct4_{n}"]) < 1e-13
    assert rel(oracle_lib.dtt1d(x, QS_RODFT11, direct), G[f"d1_dst4_{n}"]) < 1e-13


@pytest.mark.parametrize("shape", [(4, 4), (8, 16), (32, 32), (16, 48)])
def test_dtt2d_golden(oracle_lib, shape):
    nz, ny = shape
    x = G[f"d2_in_{nz}x{ny}"]
    for kz in (0, 1):
        for ky in (0, 1):
            y = oracle_lib.transform2d(x, kz, ky)
            assert rel(y, G[f"d2_{kz}{ky}_{nz}x{ny}"]) < 1e-13


@pytest.mark.parametrize("n", [4, 8])
def test_reference_harness_patterns(oracle_lib, n):
    for tag, kz, ky in (("p", 1, 0), ("m", 0, 1)):
        x = G[f"harness_{tag}_{n}_in"]
        y = oracle_lib.transform2d(x, kz, ky)
        assert rel(y, G[f"harness_{tag}_{n}_out"]) < 1e-13


@pytest.mark.parametrize("n", [8, 64, 256])
def test_involution(oracle_lib, n):
    """REDFT11 and RODFT11 are their own inverses up to 2n (the reference
    normalises by 4*ny*nz after a forward and an inverse 2-D transform,
    movefieldshydrolinlayersplit.cpp:1010)."""
    rng = np.random.default_rng(n)
    x = rng.standard_normal(n)
    for kind in (QS_REDFT11, QS_RODFT11):
        y = oracle_lib.dtt1d(oracle_lib.dtt1d(x, kind), kind)
        assert rel(y / (2 * n), x) < 1e-13
    X = rng.standard_normal((n // 2, n))
    for kz in (0, 1):
        for ky in (0, 1):
            Y = oracle_lib.transform2d(oracle_lib.transform2d(X, kz, ky), kz, ky)
            assert rel(Y / (4 * n * (n // 2)), X) < 1e-13


def test_fast_matches_direct_large(oracle_lib):
    rng = np.random.default_rng(5)
    x = rng.standard_normal((64, 256))
    for kz in (0, 1):
        for ky in (0, 1):
            a = oracle_lib.transform2d(x, kz, ky)
            b = oracle_lib.transform2d(x, kz, ky, direct=True)
            assert rel(a, b) < 1e-11
