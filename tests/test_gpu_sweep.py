"""The momentum sweep's three kernels give the same step: the z-march (CAVITY_SWEEP=march, sweep_march.cuh)
against the shared-memory tile kernel (the default) and the face-by-face kernel (CAVITY_SWEEP=face), from the same
random O(1) state, on grids that exercise every edge of the march: tiles cut by the grid's x and y ends, short
z-chunks, odd nz, 2nd-order stencils, both precision forms and a batch of cavities."""
import os

import numpy as np
import pytest

from cases import base_settings, random_state
from les_impulse3d_64_b200.api import Solver

pytestmark = pytest.mark.gpu
FIELDS = ('u', 'v', 'w', 'mx', 'my', 'mz', 'phi')


def run(settings, precision, env, steps=2):
    old = {k: os.environ.get(k) for k in env}
    os.environ.update(env)
    try:
        sim = Solver(settings, precision=precision)
    finally:
        for k, v in old.items():
            if v is None:
                os.environ.pop(k, None)
            else:
                os.environ[k] = v
    try:
        sim.initialize()
        for name, a in random_state(sim.shapes, 5, True).items():
            sim.set_field(name, a)
        reps = [sim.step() for _ in range(steps)]
        return reps, {k: sim.field64(k) for k in FIELDS}
    finally:
        sim.close()


GRIDS = [
    dict(nx=16, ny=16, nz=8),                                       # one tile, partial in x and y
    dict(nx=40, ny=40, nz=13, grid_stretch=1, grid_dx_wall=0.01),    # tiles cut in x and y, odd nz
    dict(nx=64, ny=64, nz=64, grid_stretch=1, grid_dx_wall=0.0049),  # C2-like
    dict(nx=24, ny=24, nz=5, impulse_order=2),                      # smallest nz, 2nd order
    dict(nx=32, ny=32, nz=40, impulse_order4_ramp=3.0, lid_shaped=0),
]


@pytest.mark.parametrize('precision', ['fp64', 'mixed'])
@pytest.mark.parametrize('grid', range(len(GRIDS)))
@pytest.mark.parametrize('other', ['tile', 'face'])     # CAVITY_SWEEP=tile: the default
def test_march_matches_other_sweeps(precision, grid, other):
    s = base_settings(adaptive_dt=1, dt_max=0.01, nu=0.002, **GRIDS[grid])
    rm, fm = run(s, precision, {'CAVITY_SWEEP': 'march'})
    ro, fo = run(s, precision, {'CAVITY_SWEEP': other})
    tol = 1e-12 if precision == 'fp64' else 2e-6
    for a, b in zip(rm, ro):
        assert a['dt_reason'] == b['dt_reason'] and a['phi_passes'] == b['phi_passes']
    for k in FIELDS:
        err = float(np.abs(fm[k] - fo[k]).max() / max(np.abs(fo[k]).max(), 1e-30))
        assert err <= tol, (k, err)


@pytest.mark.parametrize('chunks', ['1', '3', '16'])
def test_march_chunks_do_not_change_the_step(chunks):
    """Any split of z into chunks gives the same fields bit for bit (each chunk recomputes its halo planes)."""
    s = base_settings(adaptive_dt=1, dt_max=0.01, nu=0.002, nx=32, ny=32, nz=33, grid_stretch=1, grid_dx_wall=0.01)
    _, ref = run(s, 'fp64', {'CAVITY_SWEEP': 'march', 'CAVITY_MARCH_CHUNKS': '2'})
    _, f = run(s, 'fp64', {'CAVITY_SWEEP': 'march', 'CAVITY_MARCH_CHUNKS': chunks})
    for k in FIELDS:
        assert np.array_equal(f[k], ref[k]), k


@pytest.mark.parametrize('grid', range(len(GRIDS)))
def test_packed_pair_sweep_matches_tile_sweep(grid):
    """The FP32 sweep with two cells per thread in packed FP32x2 arithmetic (CAVITY_SWEEP=pair, sweep_pair.cuh)
    against the one-cell-per-thread tile kernel: the same expressions and sums, so the mixed form's fields agree
    to FP32 rounding."""
    s = base_settings(adaptive_dt=1, dt_max=0.01, nu=0.002, **GRIDS[grid])
    rp, fp = run(s, 'mixed', {'CAVITY_SWEEP': 'pair'})
    rt, ft = run(s, 'mixed', {'CAVITY_SWEEP': 'tile'})
    for a, b in zip(rp, rt):
        assert a['dt_reason'] == b['dt_reason'] and a['phi_passes'] == b['phi_passes']
    for k in FIELDS:
        err = float(np.abs(fp[k] - ft[k]).max() / max(np.abs(ft[k]).max(), 1e-30))
        assert err <= 2e-6, (k, err)


def test_packed_pair_sweep_in_a_batch():
    """A mixed-form batch of cavities of three sizes with the packed FP32x2 sweep equals the same batch with the
    tile sweep to FP32 rounding."""
    from les_impulse3d_64_b200 import workloads
    from les_impulse3d_64_b200.ensemble import Ensemble
    cases = workloads.ensemble_cases(count=6, seed=13, sizes=(16, 24, 40), re_range=(100.0, 2000.0))
    out = {}
    for kind in ('pair', 'tile'):
        old = os.environ.get('CAVITY_SWEEP')
        os.environ['CAVITY_SWEEP'] = kind
        try:
            ens = Ensemble(cases, group='precision')
        finally:
            if old is None:
                os.environ.pop('CAVITY_SWEEP', None)
            else:
                os.environ['CAVITY_SWEEP'] = old
        try:
            ens.advance(3, chunk=3)
            out[kind] = [ens.fields(i) for i in range(len(cases))]
        finally:
            ens.close()
    for i in range(len(cases)):
        for k in out['tile'][i]:
            a, b = out['pair'][i][k], out['tile'][i][k]
            err = float(np.abs(a - b).max() / max(np.abs(b).max(), 1e-30))
            assert err <= 2e-6, (i, k, err)
