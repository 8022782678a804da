"""GPU parity of the B200 build (both precision forms) against the reference's golden fixtures and the CPU
oracle, through the C ABI (ctypes, the reference's binding interface)."""
from pathlib import Path

import numpy as np
import pytest

from cases import CASES, run_case
from les_impulse3d_64_b200 import workloads
from les_impulse3d_64_b200.api import Solver
from parity import compare, max_rel

GOLDEN = Path(__file__).resolve().parent / 'golden'
pytestmark = pytest.mark.gpu


@pytest.mark.parametrize('name', sorted(CASES))
def test_fp64_matches_reference_fixture(name):
    ref = dict(np.load(GOLDEN / f'{name}.npz'))
    out = run_case(lambda s: Solver(s, precision='fp64'), CASES[name])
    assert compare(out, ref, field_rtol=2e-5, passes='at_most', div_atol=1e-5) == []


@pytest.mark.parametrize('name', sorted(CASES))
def test_mixed_matches_reference_fixture(name):
    ref = dict(np.load(GOLDEN / f'{name}.npz'))
    out = run_case(lambda s: Solver(s, precision='mixed'), CASES[name])
    assert compare(out, ref, field_rtol=2e-5, passes='any', div_atol=1e-5) == []


@pytest.mark.parametrize('name', sorted(CASES))
def test_mixed_tensor_core_transforms_match_reference_fixture(name, monkeypatch):
    """The mixed form with its FDM transforms forced onto the tcgen05 tensor cores (the default below 128^3
    cells is the FP64 DMMA transforms)."""
    monkeypatch.setenv('CAVITY_FDM', 'tc')
    ref = dict(np.load(GOLDEN / f'{name}.npz'))
    out = run_case(lambda s: Solver(s, precision='mixed'), CASES[name])
    assert compare(out, ref, field_rtol=2e-5, passes='any', div_atol=1e-5) == []


def _run_steps(make, case_settings, steps, noise, seed):
    sim = make(case_settings)
    try:
        sim.initialize(*workloads.initial_noise(sim.shapes, noise, seed))
        reports = [sim.step() for _ in range(steps)]
        fields = {k: sim.field64(k) for k in ('u', 'v', 'w', 'mx', 'my', 'mz', 'phi')}
        probes = sim.probes()
    finally:
        sim.close()
    return reports, fields, probes


@pytest.mark.parametrize('name, steps', [('one_step_o4_uniform', 1), ('two_steps_o4_stretched', 2),
                                         ('three_steps_o2_lag', 3)])
def test_fp64_matches_fp64_oracle_bitwise_level(oracle_libs, name, steps):
    """Same random state, same steps: FP64 GPU vs FP64 oracle to 1e-12 relative (double fields)."""
    case = CASES[name]
    outs = []
    for make in (lambda s: Solver(s, precision='fp64'), lambda s: Solver(s, library=oracle_libs['fp64'])):
        sim = make(case['settings'])
        try:
            sim.initialize()
            from cases import random_state
            for k, a in random_state(sim.shapes, case['script'][0][1], case['script'][0][2]).items():
                sim.set_field(k, a)
            reps = [sim.step() for _ in range(steps)]
            outs.append((reps, {k: sim.field64(k) for k in ('u', 'v', 'w', 'mx', 'my', 'mz', 'phi')}))
        finally:
            sim.close()
    (rg, fg), (ro, fo) = outs
    for a, b in zip(rg, ro):
        assert a['dt_reason'] == b['dt_reason'] and a['phi_passes'] == b['phi_passes']
        assert abs(a['dt'] - b['dt']) <= 1e-14 * abs(b['dt'])
    for k in fg:
        assert max_rel(fg[k], fo[k]) <= 1e-12, k


def test_c1_500_steps_fp64_vs_oracle(oracle_libs):
    """C1 (32^3, Re 400, polynomial lid, fixed dt, 500 steps): FP64 GPU vs FP64 oracle <= 1e-10."""
    w = workloads.C1
    rg, fg, pg = _run_steps(lambda s: Solver(s, precision='fp64'), w['settings'], w['steps'], w['noise'], w['seed'])
    ro, fo, po = _run_steps(lambda s: Solver(s, library=oracle_libs['fp64']), w['settings'], w['steps'], w['noise'],
                            w['seed'])
    assert [r['dt_reason'] for r in rg] == [r['dt_reason'] for r in ro]
    assert [r['phi_passes'] for r in rg] == [r['phi_passes'] for r in ro]
    for k in fg:
        assert max_rel(fg[k], fo[k]) <= 1e-10, (k, max_rel(fg[k], fo[k]))
    assert np.array_equal(pg, po) or max_rel(pg, po) <= 1e-6
