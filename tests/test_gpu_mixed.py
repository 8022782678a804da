"""The mixed form (FP32 fields, FDM transforms on the tcgen05 tensor cores) against the FP64 oracle and against
its own FP64-transform variant, at the benchmark grids."""
import os

import numpy as np
import pytest

from les_impulse3d_64_b200 import workloads
from les_impulse3d_64_b200.api import Solver

pytestmark = pytest.mark.gpu


def rel_l2(a, b):
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


def run(make, settings, steps, noise, seed):
    sim = make(settings)
    try:
        sim.initialize(*workloads.initial_noise(sim.shapes, noise, seed))
        reps = [sim.step() for _ in range(steps)]
        fields = {k: sim.field64(k) for k in ('u', 'v', 'w', 'phi')}
        diag = sim.diagnostics()
    finally:
        sim.close()
    return reps, fields, diag


def with_env(name, value, fn):
    old = os.environ.get(name)
    os.environ[name] = value
    try:
        return fn()
    finally:
        if old is None:
            del os.environ[name]
        else:
            os.environ[name] = old


@pytest.mark.parametrize('n, steps', [(32, 40), (64, 20)])
def test_tensor_core_transforms_match_fp64_transforms(n, steps):
    """Mixed form, tcgen05 3xTF32 transforms vs the FP64 DMMA transforms (CAVITY_FDM=dmma): both refine the
    pressure to fdm_rtol, so the fields agree to FP32 level."""
    s = workloads.settings(n, 1000.0, beta=1.5, cfl=0.5)
    r_tc, f_tc, d_tc = with_env('CAVITY_FDM', 'tc', lambda: run(lambda x: Solver(x, precision='mixed'), s, steps,
                                                                  1e-3, 0))
    r_dm, f_dm, d_dm = with_env('CAVITY_FDM', 'dmma', lambda: run(lambda x: Solver(x, precision='mixed'), s, steps,
                                                                    1e-3, 0))
    for a, b in zip(r_tc, r_dm):
        assert a['phi_rel'] <= 1e-9 and b['phi_rel'] <= 1e-9
        assert abs(a['dt'] - b['dt']) <= 1e-6 * b['dt']
    for k in ('u', 'v', 'w'):
        assert rel_l2(f_tc[k], f_dm[k]) <= 1e-5, k
    assert d_tc['div_rms'] <= 1e-5


@pytest.mark.parametrize('fdm', ['tc', 'dmma'])
@pytest.mark.parametrize('workload, steps', [('c1_32cube_re400', 100), ('c2_64cube_re1000', 30)])
def test_mixed_matches_fp64_oracle(oracle_libs, workload, steps, fdm):
    """Mixed form, with either transform path, vs the FP64 oracle on the same seeded run: velocity within 1e-5
    relative L2; the divergence invariant of the reference's own check (div_rms < 1e-5)."""
    w = workloads.WORKLOADS[workload]
    r_gpu, f_gpu, d_gpu = with_env('CAVITY_FDM', fdm, lambda: run(lambda x: Solver(x, precision='mixed'),
                                                                   w['settings'], steps, w['noise'], w['seed']))
    r_orc, f_orc, _ = run(lambda x: Solver(x, library=oracle_libs['fp64']), w['settings'], steps, w['noise'],
                          w['seed'])
    assert [r['dt_reason'] for r in r_gpu] == [r['dt_reason'] for r in r_orc]
    for k in ('u', 'v', 'w'):
        assert rel_l2(f_gpu[k], f_orc[k]) <= 1e-5, (k, rel_l2(f_gpu[k], f_orc[k]))
    assert d_gpu['div_rms'] < 1e-5
