"""The host eigenbasis of the pressure operator (cavity_eigenbasis, host QL) on the CPU: S S^T = W^-1, and the
operator K = W S diag(lambda) S^T W it implies is the axis's Neumann Laplacian: tridiagonal, symmetric, zero row
sums, couplings 1/spacing and widths from the grid of the oracle (whose grid is bit-identical to the product's)."""
import ctypes as ct

import numpy as np
import pytest

from les_impulse3d_64_b200 import workloads
from les_impulse3d_64_b200.api import Solver, load_library, make_config


@pytest.mark.parametrize('n,beta', [(8, None), (24, 1.5), (64, 1.5), (130, 2.0)])
def test_host_eigenbasis_is_the_axis_operator(n, beta, oracle_libs):
    lib = load_library()
    lib.cavity_eigenbasis.argtypes = [ct.c_void_p, ct.c_int, ct.c_int, ct.c_void_p, ct.c_void_p]
    lib.cavity_eigenbasis.restype = ct.c_int
    s = workloads.settings(n, 1000.0, beta=beta)
    lam, S = np.empty(n), np.empty((n, n))
    assert lib.cavity_eigenbasis(ct.byref(make_config(s)), 0, 0, lam.ctypes.data, S.ctypes.data) == 0

    oracle = Solver(s, library=oracle_libs['fp64'])
    try:
        faces, centres = oracle.grid['x']
    finally:
        oracle.close()

    assert lam.max() == 0.0 and np.sum(lam == 0.0) == 1 and np.all(lam[lam != 0.0] < 0)
    inv_w = S @ S.T
    d = np.diag(inv_w)
    assert np.abs(inv_w - np.diag(d)).max() <= 1e-12 * d.max()
    W = np.diag(1.0 / d)
    K = W @ S @ np.diag(lam) @ S.T @ W
    scale = np.abs(K).max()
    far = np.abs(np.triu(K, 2)).max() if n > 2 else 0.0
    assert far <= 1e-10 * scale
    assert np.abs(K - K.T).max() <= 1e-10 * scale
    assert np.abs(K.sum(axis=1)).max() <= 1e-10 * scale
    # widths and spacings of the grid: the oracle reports faces and centres rounded to float, so their differences
    # carry up to a float ulp of the coordinates
    ulp = 2.0 ** -23 * max(np.abs(faces).max(), 1.0)
    assert np.abs(1.0 / d - np.diff(faces)).max() <= 2 * ulp
    assert np.abs(1.0 / np.diag(K, 1) - np.diff(centres)).max() <= 2 * ulp
