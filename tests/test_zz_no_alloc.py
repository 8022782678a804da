"""cavity_fdm_pass_noalloc, the pressure pass for callers that cannot allocate device memory (hosts whose
device memory belongs to their own pool allocator, or processes running with the device nearly full): it
must give the result of cavity_fdm_pass, which allocates its intermediates, on two calls in a row through
the same shared device array, and refuse grids beyond its 262144-cell limit.  Collected last so that a run
stopping at the first failure has already run every other test."""
import ctypes as ct

import numpy as np
import pytest

from les_impulse3d_64_b200.api import load_library
from test_gpu_fdm import device, random_operands

pytestmark = pytest.mark.gpu


def _fn(lib, name):
    fn = getattr(lib, name)
    fn.argtypes = [ct.c_int, ct.c_int, ct.c_int, ct.c_void_p, ct.c_void_p, ct.c_void_p, ct.c_void_p, ct.c_void_p,
                   ct.c_void_p]
    return fn


@pytest.mark.parametrize('shape', [(40, 40, 33), (64, 64, 64)])
def test_noalloc_pass_matches_allocating_pass_twice(shape):
    """A ragged grid, and 64^3, the full size of the shared device array."""
    lib = load_library()
    lib.cavity_last_error.restype = ct.c_char_p
    S, il, r, phi = random_operands(*shape, seed=11)
    nz, ny, nx = r.shape
    ds = [device(s) for s in S]
    dst = [device(s.T.copy()) for s in S]
    sp = (ct.c_void_p * 3)(*[t.data_ptr() for t in ds])
    stp = (ct.c_void_p * 3)(*[t.data_ptr() for t in dst])
    dil, dr = device(il), device(r)
    phi_alloc, phi_static = device(phi), device(phi)
    for call in range(2):
        for name, out in (('cavity_fdm_pass', phi_alloc), ('cavity_fdm_pass_noalloc', phi_static)):
            rc = _fn(lib, name)(nx, ny, nz, sp, stp, dil.data_ptr(), dr.data_ptr(), out.data_ptr(), None)
            assert rc == 0, lib.cavity_last_error().decode()
        a, b = phi_alloc.cpu().numpy(), phi_static.cpu().numpy()
        assert np.abs(a - b).max() <= 1e-12 * np.abs(a).max(), f'call {call + 1}'


@pytest.mark.parametrize('shape, message', [((65, 64, 64), b'exceeds the maximum of 262144'),
                                            ((2048, 64, 1), b'1 <= nx, ny, nz <= 1024'),
                                            ((2, 2, 65536), b'1 <= nx, ny, nz <= 1024'),
                                            ((0, 8, 8), b'1 <= nx, ny, nz <= 1024')])
def test_noalloc_pass_rejects_grids_beyond_its_limit(shape, message):
    """Over the cell limit, or one axis over 1024 cells with fewer than 262144 cells in all: rejected with a
    message before anything is launched (the pointers here are never dereferenced)."""
    lib = load_library()
    lib.cavity_last_error.restype = ct.c_char_p
    sp = (ct.c_void_p * 3)(1, 1, 1)
    rc = _fn(lib, 'cavity_fdm_pass_noalloc')(*shape, sp, sp, 1, 1, 1, None)
    assert rc == 1
    assert message in lib.cavity_last_error()
