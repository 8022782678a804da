"""The pressure operator's eigenbasis computed on the GPU (bisection and inverse iteration, the set-up with
CAVITY_EIGEN=gpu) against the host's implicit-shift QL, and a solver set up with it against one set up on the host."""
import ctypes as ct

import numpy as np
import pytest

from les_impulse3d_64_b200 import workloads
from les_impulse3d_64_b200.api import Solver, load_library, make_config

pytestmark = pytest.mark.gpu


def eigenbasis(lib, settings, on_gpu):
    n = settings['nx']
    lam, S = np.empty(n), np.empty((n, n))
    lib.cavity_eigenbasis.argtypes = [ct.c_void_p, ct.c_int, ct.c_int, ct.c_void_p, ct.c_void_p]
    lib.cavity_eigenbasis.restype = ct.c_int
    config = make_config(settings)
    assert lib.cavity_eigenbasis(ct.byref(config), 0, int(on_gpu), lam.ctypes.data, S.ctypes.data) == 0, \
        lib.cavity_last_error().decode()
    return lam, S


@pytest.mark.parametrize('n,beta', [(8, None), (32, None), (64, 1.5), (130, 2.0), (512, 2.0)])
def test_gpu_eigenbasis_matches_host(n, beta):
    lib = load_library()
    s = workloads.settings(n, 1000.0, beta=beta)
    lam_h, S_h = eigenbasis(lib, s, False)
    lam_g, S_g = eigenbasis(lib, s, True)
    order = np.argsort(lam_h, kind='stable')
    lam_h, S_h = lam_h[order], S_h[:, order]
    scale = np.abs(lam_h).max()
    assert np.abs(lam_g - lam_h).max() <= 1e-12 * scale
    assert lam_g[-1] == 0.0                                   # the constant mode, set to exactly zero
    # S S^T = W^-1 (diagonal) for both
    inv_w = S_h @ S_h.T
    assert np.abs(S_g @ S_g.T - inv_w).max() <= 1e-11 * np.abs(np.diag(inv_w)).max()
    # the eigen-equation K S = W S diag(lambda), with K = W S_h diag(lambda_h) S_h^T W from the host's basis.  The
    # vectors themselves are compared only through it: on a symmetric stretched grid the modes held in the small
    # wall cells come in pairs whose eigenvalues agree to rounding, and any rotation within a pair is a valid basis.
    W = np.diag(1.0 / np.diag(inv_w))
    K = W @ S_h @ np.diag(lam_h) @ S_h.T @ W
    resid = K @ S_g - W @ S_g @ np.diag(lam_g)
    assert np.abs(resid).max() <= 1e-11 * np.abs(K).max() * np.abs(S_g).max()


def test_solver_with_gpu_eigenbasis_matches_host(monkeypatch):
    s = workloads.settings(32, 1000.0, beta=1.5)
    v, w = workloads.initial_noise({'v': (32, 33, 32), 'w': (33, 32, 32)}, 1e-3, 0)
    out = {}
    for mode in ('host', 'gpu'):
        monkeypatch.setenv('CAVITY_EIGEN', mode)
        sim = Solver(s, precision='fp64')
        try:
            sim.initialize(v, w)
            passes = [sim.step()['phi_passes'] for _ in range(10)]
            out[mode] = (passes, {k: sim.field64(k) for k in ('u', 'v', 'w', 'phi')})
        finally:
            sim.close()
    assert out['gpu'][0] == out['host'][0]
    for k, a in out['host'][1].items():
        b = out['gpu'][1][k]
        assert np.abs(b - a).max() <= 1e-10 * max(np.abs(a).max(), 1e-30), k
