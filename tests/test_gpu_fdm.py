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


@pytest.mark.parametrize('fused', ['0', '1', '2'])
@pytest.mark.parametrize('dims', [(8, 8, 5), (7, 9, 11), (24, 24, 16), (40, 40, 33), (33, 64, 50), (64, 64, 64),
                                  (96, 80, 70)])
def test_fdm_pass_matches_numpy(dims, fused, monkeypatch):
    """The FP64 pass as six launches (CAVITY_FDM_FUSED=0), as one cooperative launch with grid barriers between
    the transforms (=1) and as three launches of two chained transforms each (=2, the default where no axis
    exceeds 64 cells; six launches above), each against NumPy; and each bit for bit against the six launches."""
    monkeypatch.setenv('CAVITY_FDM_FUSED', fused)
    lib = load_library()
    lib.cavity_last_error.restype = ct.c_char_p
    S, il, r, phi = random_operands(*dims, seed=sum(dims))
    out = call_fdm(lib, 'cavity_fdm_pass', S, il, r, phi)
    ref = fdm_reference(S, r, il, phi)
    assert np.abs(out - ref).max() <= 1e-12 * np.abs(ref).max()
    monkeypatch.setenv('CAVITY_FDM_FUSED', '2' if fused == '0' else '0')
    assert np.array_equal(call_fdm(lib, 'cavity_fdm_pass', S, il, r, phi), out)


def test_fdm_pass_default_is_the_paired_pass(monkeypatch):
    """Without CAVITY_FDM_FUSED a pass on axes of at most 64 cells is the paired one (bit for bit equal to it)."""
    lib = load_library()
    lib.cavity_last_error.restype = ct.c_char_p
    S, il, r, phi = random_operands(48, 40, 36, seed=11)
    monkeypatch.delenv('CAVITY_FDM_FUSED', raising=False)
    out = call_fdm(lib, 'cavity_fdm_pass', S, il, r, phi)
    monkeypatch.setenv('CAVITY_FDM_FUSED', '2')
    assert np.array_equal(call_fdm(lib, 'cavity_fdm_pass', S, il, r, phi), out)


FIELDS = ('u', 'v', 'w', 'mx', 'my', 'mz', 'phi')


def solver_run(settings, precision, form, steps=3):
    """`steps` steps of a random state, the solver created with CAVITY_FDM_FUSED=form (None: unset)."""
    import os

    from cases import random_state
    from les_impulse3d_64_b200.api import Solver
    old = os.environ.pop('CAVITY_FDM_FUSED', None)
    if form is not None:
        os.environ['CAVITY_FDM_FUSED'] = form
    try:
        sim = Solver(settings, precision=precision)
    finally:
        os.environ.pop('CAVITY_FDM_FUSED', None)
        if old is not None:
            os.environ['CAVITY_FDM_FUSED'] = old
    try:
        sim.initialize()
        for name, a in random_state(sim.shapes, 9, True).items():
            sim.set_field(name, a)
        reps = [sim.step() for _ in range(steps)]
        return reps, {k: sim.field64(k) for k in FIELDS}
    finally:
        sim.close()


@pytest.mark.parametrize('precision', ['fp64', 'mixed'])
@pytest.mark.parametrize('grid', [dict(nx=16, ny=16, nz=8), dict(nx=22, ny=22, nz=9),
                                  dict(nx=40, ny=40, nz=13, grid_stretch=1, grid_dx_wall=0.01),
                                  dict(nx=64, ny=64, nz=64, grid_stretch=1, grid_dx_wall=0.0049)])
def test_paired_pass_steps_equal_six_launch_steps(precision, grid):
    """Whole steps (initial projection, refinement loops with their guess and pass decisions) with the paired
    pass and with six launches per pass: the same reports and the same fields bit for bit."""
    from cases import base_settings
    s = base_settings(adaptive_dt=1, dt_max=0.01, nu=0.002, **grid)
    rp, fp = solver_run(s, precision, '2')
    rs, fs = solver_run(s, precision, '0')
    rd, fd = solver_run(s, precision, None)
    for a, b, c in zip(rp, rs, rd):
        assert a == b == c
    for k in FIELDS:
        assert np.array_equal(fp[k], fs[k]), k
        assert np.array_equal(fp[k], fd[k]), k


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


WIDTH_CHECK = r'''
import os, sys
import numpy as np
sys.path[:0] = [{tests!r}, {root!r}]
import test_gpu_fdm as t
from les_impulse3d_64_b200.api import load_library
import ctypes as ct
lib = load_library()
lib.cavity_last_error.restype = ct.c_char_p
for dims in ((8, 8, 5), (7, 9, 11), (40, 40, 33), (64, 64, 64)):
    S, il, r, phi = t.random_operands(*dims, seed=sum(dims) + 5)
    os.environ['CAVITY_FDM_FUSED'] = '2'
    a = t.call_fdm(lib, 'cavity_fdm_pass', S, il, r, phi)
    os.environ['CAVITY_FDM_FUSED'] = '0'
    b = t.call_fdm(lib, 'cavity_fdm_pass', S, il, r, phi)
    assert np.array_equal(a, b), dims
print('ok')
'''


@pytest.mark.parametrize('width', ['16', '32'])
def test_paired_pass_widths(width):
    """The paired pass with CTAs 16 or 32 columns wide (CAVITY_PAIR_W, read once per process: a child process
    each) equals the six-launch pass bit for bit."""
    import os
    import subprocess
    import sys
    from pathlib import Path
    tests = Path(__file__).resolve().parent
    code = WIDTH_CHECK.format(tests=str(tests), root=str(tests.parent))
    env = dict(os.environ, CAVITY_PAIR_W=width)
    res = subprocess.run([sys.executable, '-c', code], env=env, capture_output=True, text=True, timeout=300)
    assert res.returncode == 0 and 'ok' in res.stdout, res.stdout + res.stderr


@pytest.mark.parametrize('per', ['3', '64'])
def test_paired_pass_tiles_per_cta(per):
    """The paired pass with several tiles per CTA (CAVITY_PAIR_PER: planes, or plane-column blocks, taken in a row
    by one CTA with its bases staged once, as large batches run it; read once per process: a child process each),
    the last CTA of an axis taking fewer, equals the six-launch pass bit for bit."""
    import os
    import subprocess
    import sys
    from pathlib import Path
    tests = Path(__file__).resolve().parent
    code = WIDTH_CHECK.format(tests=str(tests), root=str(tests.parent))
    env = dict(os.environ, CAVITY_PAIR_PER=per)
    res = subprocess.run([sys.executable, '-c', code], env=env, capture_output=True, text=True, timeout=300)
    assert res.returncode == 0 and 'ok' in res.stdout, res.stdout + res.stderr


TC_KERNEL_RUN = r'''
import sys
import numpy as np
sys.path[:0] = [{tests!r}, {root!r}]
import test_gpu_fdm as t
from les_impulse3d_64_b200.api import load_library
import ctypes as ct
lib = load_library()
lib.cavity_last_error.restype = ct.c_char_p
out = {{}}
for dims in ((8, 8, 5), (24, 24, 16), (40, 40, 33), (128, 96, 130), (132, 20, 36)):
    S, il, r, phi = t.random_operands(*dims, seed=sum(dims) + 7)
    out['x'.join(map(str, dims))] = t.call_fdm(lib, 'cavity_fdm_pass_tf32', S, il, r, phi)
np.savez({path!r}, **out)
'''


def test_tc_kernels_agree(tmp_path):
    """The two tensor-core transform kernels, the register-pipelined one and the staged one (CAVITY_TC_KERNEL
    selects, read once per process: a child process each), give the same pass bit for bit: the same split
    operands and the same MMA sequence for every output element, whatever the tile width."""
    import os
    import subprocess
    import sys
    from pathlib import Path
    tests = Path(__file__).resolve().parent
    res = {}
    for kind in ('staged', 'panel'):
        path = str(tmp_path / f'{kind}.npz')
        code = TC_KERNEL_RUN.format(tests=str(tests), root=str(tests.parent), path=path)
        env = dict(os.environ, CAVITY_TC_KERNEL=kind)
        r = subprocess.run([sys.executable, '-c', code], env=env, capture_output=True, text=True, timeout=300)
        assert r.returncode == 0, r.stdout + r.stderr
        res[kind] = dict(np.load(path))
    for k in res['panel']:
        assert np.array_equal(res['staged'][k], res['panel'][k]), k
