"""The standalone fast-diagonalisation pass (cavity_fdm_pass) against NumPy on random operands."""
import ctypes as ct

import numpy as np
import pytest

from les_impulse3d_64_b200.api import load_library

pytestmark = pytest.mark.gpu


def device(a):
    import torch
    return torch.from_numpy(np.ascontiguousarray(a)).to('cuda')


def fdm_reference(S, r, inv_lambda, phi):
    """phi + S_x S_y S_z (inv_lambda .* S_z^T S_y^T S_x^T r) on [z][y][x] arrays."""
    t = np.einsum('zyi,ij->zyj', r, S[0])
    t = np.einsum('ij,zix->zjx', S[1], t)
    t = np.einsum('ij,iyx->jyx', S[2], t)
    t = t * inv_lambda
    t = np.einsum('ij,jyx->iyx', S[2], t)
    t = np.einsum('ij,zjx->zix', S[1], t)
    t = np.einsum('zyj,ij->zyi', t, S[0])
    return phi + t


def random_operands(nx, ny, nz, seed):
    rng = np.random.default_rng(seed)
    S = [np.linalg.qr(rng.standard_normal((n, n)))[0] for n in (nx, ny, nz)]
    inv_lambda = rng.uniform(0.1, 1.0, (nz, ny, nx))
    r = rng.standard_normal((nz, ny, nx))
    phi = rng.standard_normal((nz, ny, nx))
    return S, inv_lambda, r, phi


def call_fdm(lib, name, S, inv_lambda, r, phi):
    nz, ny, nx = r.shape
    ds = [device(s) for s in S]
    dst = [device(s.T.copy()) for s in S]
    dil, dr, dphi = device(inv_lambda), device(r), device(phi)
    sp = (ct.c_void_p * 3)(*[t.data_ptr() for t in ds])
    stp = (ct.c_void_p * 3)(*[t.data_ptr() for t in dst])
    fn = getattr(lib, name)
    fn.argtypes = [ct.c_int, ct.c_int, ct.c_int, ct.c_void_p, ct.c_void_p, ct.c_void_p, ct.c_void_p, ct.c_void_p,
                   ct.c_void_p]
    rc = fn(nx, ny, nz, sp, stp, dil.data_ptr(), dr.data_ptr(), dphi.data_ptr(), None)
    if rc:
        raise RuntimeError(lib.cavity_last_error().decode())
    return dphi.cpu().numpy()


@pytest.mark.parametrize('fused', ['0', '1'])
@pytest.mark.parametrize('dims', [(8, 8, 5), (24, 24, 16), (40, 40, 33), (64, 64, 64), (96, 80, 70)])
def test_fdm_pass_matches_numpy(dims, fused, monkeypatch):
    """The FP64 pass as six launches (CAVITY_FDM_FUSED=0) and as one cooperative launch with grid barriers
    between the transforms (=1), each against NumPy; and the two bit for bit against each other."""
    monkeypatch.setenv('CAVITY_FDM_FUSED', fused)
    lib = load_library()
    lib.cavity_last_error.restype = ct.c_char_p
    S, il, r, phi = random_operands(*dims, seed=sum(dims))
    out = call_fdm(lib, 'cavity_fdm_pass', S, il, r, phi)
    ref = fdm_reference(S, r, il, phi)
    assert np.abs(out - ref).max() <= 1e-12 * np.abs(ref).max()
    monkeypatch.setenv('CAVITY_FDM_FUSED', '1' if fused == '0' else '0')
    assert np.array_equal(call_fdm(lib, 'cavity_fdm_pass', S, il, r, phi), out)


@pytest.mark.parametrize('dims', [(8, 8, 5), (24, 24, 16), (40, 40, 33), (64, 64, 64), (128, 96, 130)])
def test_fdm_pass_tf32_matches_numpy(dims):
    """The mixed form's pass on the tensor cores (3xTF32, float S, r scaled to rms 1): the update agrees with
    the FP64 pass to FP32 level (1e-5 of its largest entry)."""
    lib = load_library()
    lib.cavity_last_error.restype = ct.c_char_p
    S, il, r, phi = random_operands(*dims, seed=sum(dims) + 1)
    out = call_fdm(lib, 'cavity_fdm_pass_tf32', S, il, r, phi)
    ref = fdm_reference(S, r, il, phi)
    upd = ref - phi
    assert np.abs(out - ref).max() <= 1e-5 * np.abs(upd).max()


def test_fdm_pass_tf32_rejects_unaligned_rows():
    lib = load_library()
    lib.cavity_last_error.restype = ct.c_char_p
    S, il, r, phi = random_operands(6, 6, 5, seed=3)
    with pytest.raises(RuntimeError, match='multiple of 4'):
        call_fdm(lib, 'cavity_fdm_pass_tf32', S, il, r, phi)
