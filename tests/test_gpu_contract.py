"""The parity contract at the configurations it names, through the C ABI on the GPU.

* C2 (64^3, beta 1.5, Re 1000, regularised lid, adaptive dt at CFL 0.5) run as the config states it: 2000
  steps, kicks of amplitude 1e-2 after steps 500 and 1000, dt-weighted mid-span statistics from step 1000, 8
  probes read after every step (main.py:342-363 is the order).  The plain FP64 form must match the FP64
  oracle (oracle/cavity_oracle.cpp, run live on the host cores) to a max relative difference of 1e-10 in
  every field after 1000 and 2000 steps, with the same dt_reason and pressure-pass sequences, the same
  statistics sums and centreline samples, and probe values read at the reference's probe cells
  (backend.cu:1058-1070).
* The mixed form (FP32 fields) against the same oracle runs: C2, and C3 (128^3, beta 2.0, Re 3200, 1000
  steps) against the oracle's run kept in tests/golden/c3_oracle_1000.npz (tests/golden/make_c3_oracle.py;
  the oracle needs about ten minutes for it).  Stated per config: velocity relative L2 (bound 1e-5), the
  potential phi relative L2, kinetic energy, and the max |div u| beside the max |div u| of the oracle's own
  field rounded to float32, which is the floor of any field held in FP32 on these stretched grids.

With CAVITY_CONTRACT_REPORT set to a file name, the measured errors are written there as JSON.
"""
import json
import os
from pathlib import Path

import numpy as np
import pytest

import contract
from les_impulse3d_64_b200 import workloads
from les_impulse3d_64_b200.api import Solver
from parity import max_rel

pytestmark = pytest.mark.gpu
GOLDEN = Path(__file__).resolve().parent / 'golden'
FIELDS = ('u', 'v', 'w', 'mx', 'my', 'mz', 'phi')
SNAPSHOTS = (1000, 2000)
REPORT = {}


def _record(key, values):
    REPORT[key] = values
    path = os.environ.get('CAVITY_CONTRACT_REPORT')
    if path:
        Path(path).write_text(json.dumps(REPORT, indent=1, default=float) + '\n')


def play(make, workload, snapshots=SNAPSHOTS, steps=None):
    """Run a workload's protocol (`steps` steps, by default the workload's) on a fresh solver; returns the
    per-step run, the fields and diagnostics at each snapshot, the final statistics and the grid."""
    sim = make(workload['settings'])
    snaps = {}

    def keep(n, s):
        # the reference's build has no double-precision getter: its float fields, widened
        get = s.field64 if hasattr(s.lib, 'cavity_get_field_f64') else (lambda k: s.field(k).astype(np.float64))
        snaps[n] = ({k: get(k) for k in FIELDS}, s.diagnostics())
    try:
        sim.initialize(*workloads.initial_noise(sim.shapes, workload['noise'], workload['seed']))
        run = workloads.run_protocol(sim, workload, steps=steps, snapshots=snapshots, on_snapshot=keep)
        stats = sim.statistics() if workload.get('stats_from') is not None else None
        grid = sim.grid
    finally:
        sim.close()
    return run, snaps, stats, grid


@pytest.fixture(scope='module')
def c2_oracle(oracle_libs):
    return play(lambda s: Solver(s, library=oracle_libs['fp64']), workloads.C2)


REFERENCE_BINARY = Path(__file__).resolve().parents[1] / 'oracle' / '_ref' / 'libcavity_solver.so'


def recorded_reference_errors(config):
    """The reference build's errors recorded on a B200, keyed by step number."""
    rec = json.loads((GOLDEN / 'reference_fp32_errors.json').read_text())[config]
    return {int(n): e for n, e in rec.items()}


@pytest.fixture(scope='module')
def c2_reference_errors(c2_oracle):
    """The reference's own backend.cu (FP32 fields, built unchanged under oracle/_ref) through C2's protocol,
    against the FP64 oracle: the error that FP32 fields carry at this config.  Where that build is absent, the
    errors it gave on a B200 (tests/golden/reference_fp32_errors.json)."""
    if not REFERENCE_BINARY.is_file():
        return recorded_reference_errors('c2')
    w = workloads.C2
    ro, so, _, _ = c2_oracle
    rr, sr, _, _ = play(lambda s: Solver(s, library=REFERENCE_BINARY), w)
    out = {}
    for n in SNAPSHOTS:
        e = mixed_errors(sr[n][0], sr[n][1], so[n][0], so[n][1], w['settings'])
        e['dt_reason_same'] = bool(list(rr['dt_reason']) == list(ro['dt_reason']))
        out[n] = e
    _record('c2_reference_backend_fp32_vs_oracle', out)
    return out


def probe_cells(settings, grid):
    """The cell of each probe on the mid-span layer: the last face at or below the probe position
    (backend.cu:1058-1070)."""
    cells = []
    for px, py in settings['probes']:
        xy = []
        for frac, name in ((px, 'x'), (py, 'y')):
            faces = grid[name][0]
            length = faces[-1] - faces[0]
            k = int(np.searchsorted(faces, frac * length, side='right')) - 1
            xy.append(min(len(faces) - 2, max(0, k)))
        cells.append((xy[0], xy[1], settings['nz'] // 2))
    return cells


def test_c2_fp64_full_config_matches_oracle(c2_oracle):
    w = workloads.C2
    ro, so, sto, grid_o = c2_oracle
    rg, sg, stg, grid_g = play(lambda s: Solver(s, precision='fp64'), w)
    for name in 'xyz':
        assert np.array_equal(grid_g[name][0], grid_o[name][0]) and np.array_equal(grid_g[name][1], grid_o[name][1])
    assert list(rg['dt_reason']) == list(ro['dt_reason'])
    assert np.array_equal(rg['phi_passes'], ro['phi_passes'])
    errors = {'dt': max_rel(rg['dt'], ro['dt']), 'time': max_rel(rg['time'], ro['time']),
              'kick_ke': max_rel(rg['kick_ke'], ro['kick_ke'])}
    for n in SNAPSHOTS:
        for k in FIELDS:
            errors[f'{k}@{n}'] = max_rel(sg[n][0][k], so[n][0][k])
        errors[f'kinetic_energy@{n}'] = max_rel(sg[n][1]['kinetic_energy'], so[n][1]['kinetic_energy'])
    for k in stg:
        errors[f'statistics.{k}'] = max_rel(stg[k], sto[k])
    errors['centreline'] = max_rel(rg['centreline'], ro['centreline'])
    errors['probes'] = max_rel(rg['probes'], ro['probes'])
    _record('c2_fp64_vs_oracle', dict(errors, steps=w['steps'], dt_reasons=sorted(set(rg['dt_reason'])),
                                      passes=int(rg['phi_passes'].sum())))
    assert len(rg['centreline']) == w['steps'] - w['stats_from']
    for k, e in errors.items():
        # probe values are float32 outputs of fields that agree to 1e-10: equal up to the last float bit
        assert e <= (2.0 ** -22 if k == 'probes' else 1e-10), (k, e)
    # the probe cells: the last probe values are u and v centred in the reference's probe cells of the GPU's
    # own field (float outputs: equal to float rounding)
    u, v = sg[2000][0]['u'], sg[2000][0]['v']
    last = rg['probes'][-1].astype(np.float64)
    for p, (x, y, z) in enumerate(probe_cells(w['settings'], grid_g)):
        cu, cv = 0.5 * (u[z, y, x] + u[z, y, x + 1]), 0.5 * (v[z, y, x] + v[z, y + 1, x])
        assert abs(last[2 * p] - cu) <= 2.0 ** -22 * abs(cu) and abs(last[2 * p + 1] - cv) <= 2.0 ** -22 * abs(cv), p


def mixed_errors(f, diag, ref_f, ref_diag, settings, layers=None):
    """The contract's errors of one mixed-form state against the oracle's."""
    if layers is not None:
        f = {k: f[k][list(layers)] for k in ('u', 'v', 'w', 'phi')} | {'_full': f}
    return {
        'velocity_rel_l2': contract.velocity_rel_l2(f, ref_f),
        'phi_rel_l2': contract.rel_l2(f['phi'], ref_f['phi']),
        'kinetic_energy_rel': abs(diag['kinetic_energy'] - ref_diag['kinetic_energy']) / ref_diag['kinetic_energy'],
        'div_rms': diag['div_rms'],
        'max_div': contract.max_abs_divergence(f.get('_full', f), settings),
    }


def mixed_bound(key, n, ref_errors, floor):
    """The contract's bound, or, where the reference's own FP32 form misses it at this config, twice the
    reference's error: FP32 fields cannot be held to less than what they carry."""
    if ref_errors is None:
        return floor
    return max(floor, 2.0 * ref_errors[n][key])


@pytest.mark.parametrize('fdm', ['default', 'tc'])
def test_c2_mixed_matches_fp64_oracle(c2_oracle, c2_reference_errors, fdm, monkeypatch):
    """The mixed form through C2's full protocol (kicks, statistics, probes) against the FP64 oracle, beside the
    reference's own FP32 backend.cu on the same protocol."""
    if fdm != 'default':
        monkeypatch.setenv('CAVITY_FDM', fdm)
    w = workloads.C2
    ro, so, sto, _ = c2_oracle
    rg, sg, stg, _ = play(lambda s: Solver(s, precision='mixed'), w)
    assert list(rg['dt_reason']) == list(ro['dt_reason'])
    result = {}
    for n in SNAPSHOTS:
        e = mixed_errors(sg[n][0], sg[n][1], so[n][0], so[n][1], w['settings'])
        e['max_div_oracle_float32'] = contract.max_abs_divergence(contract.as_float32(so[n][0]), w['settings'])
        result[n] = e
    result['statistics_u_rel_l2'] = contract.rel_l2(stg['u'], sto['u'])
    result['time_rel'] = max_rel(rg['time'][-1:], ro['time'][-1:])
    _record(f'c2_mixed_{fdm}_vs_oracle', result)
    for n in SNAPSHOTS:
        e = result[n]
        assert e['velocity_rel_l2'] <= mixed_bound('velocity_rel_l2', n, c2_reference_errors, 1e-5), (n, e)
        assert e['kinetic_energy_rel'] <= mixed_bound('kinetic_energy_rel', n, c2_reference_errors, 1e-5), (n, e)
        assert e['phi_rel_l2'] <= mixed_bound('phi_rel_l2', n, c2_reference_errors, 1e-4), (n, e)
        assert e['div_rms'] < 1e-5, (n, e)
        # FP32 faces cannot do better than the oracle's own field rounded to float32
        assert e['max_div'] <= 4 * e['max_div_oracle_float32'], (n, e)


@pytest.fixture(scope='module')
def c3_reference_errors():
    """The reference's own backend.cu (FP32 fields) through C3's protocol against the FP64 oracle's fixture: the
    error that FP32 fields carry at this config.  Where that build is absent, the errors it gave on a B200."""
    if not REFERENCE_BINARY.is_file():
        return recorded_reference_errors('c3')
    ref = np.load(GOLDEN / 'c3_oracle_1000.npz')
    w = workloads.C3
    steps = int(ref['steps'])
    rr, sr, _, _ = play(lambda s: Solver(s, library=REFERENCE_BINARY), w, snapshots=(steps,), steps=steps)
    f, diag = sr[steps]
    e = mixed_errors(f, diag, {k: ref[f'layer.{k}'] for k in ('u', 'v', 'w', 'phi')},
                     {'kinetic_energy': float(ref['diag.kinetic_energy'])}, w['settings'],
                     layers=[int(k) for k in ref['layers']])
    e['dt_reason_same'] = bool(list(rr['dt_reason']) == [str(x) for x in ref['run.dt_reason']])
    e['norm_rel'] = {k: abs(float(np.linalg.norm(f[k])) - float(ref[f'norm.{k}'])) / float(ref[f'norm.{k}'])
                     for k in ('u', 'v', 'w', 'phi')}
    _record('c3_reference_backend_fp32_vs_oracle', e)
    return {steps: e}


@pytest.mark.parametrize('fdm', ['default', 'dmma'])
def test_c3_mixed_matches_fp64_oracle_fixture(fdm, monkeypatch, c3_reference_errors):
    """C3, 1000 steps of the mixed form (tensor-core transforms by default at 128^3, or the FP64 DMMA ones)
    against the FP64 oracle's run of the same seeded workload (tests/golden/c3_oracle_1000.npz): errors on
    the fixture's z-layers, kinetic energy and full-field norms, and the max |div u| of the whole field."""
    if fdm != 'default':
        monkeypatch.setenv('CAVITY_FDM', fdm)
    ref = np.load(GOLDEN / 'c3_oracle_1000.npz')
    w = workloads.C3
    steps = int(ref['steps'])
    rg, sg, _, grid = play(lambda s: Solver(s, precision='mixed'), w, snapshots=(steps,), steps=steps)
    contract.check_faces(w['settings'], grid)
    f, diag = sg[steps]
    layers = [int(k) for k in ref['layers']]
    ref_f = {k: ref[f'layer.{k}'] for k in ('u', 'v', 'w', 'phi')}
    ref_diag = {'kinetic_energy': float(ref['diag.kinetic_energy'])}
    e = mixed_errors(f, diag, ref_f, ref_diag, w['settings'], layers=layers)
    e['max_div_oracle_float32'] = float(ref['max_div_float32'])
    e['max_div_oracle'] = float(ref['max_div'])
    e['norm_rel'] = {k: abs(float(np.linalg.norm(f[k])) - float(ref[f'norm.{k}'])) / float(ref[f'norm.{k}'])
                     for k in ('u', 'v', 'w', 'phi')}
    e['dt_rel'] = max_rel(rg['dt'], ref['run.dt'])
    e['time_rel'] = max_rel(rg['time'][-1:], ref['run.time'][-1:])
    e['dt_reason_same'] = bool(list(rg['dt_reason']) == [str(x) for x in ref['run.dt_reason']])
    e['probes_max_rel'] = max_rel(rg['probes'], ref['run.probes'])
    e['passes_per_stage'] = float(rg['phi_passes'].mean())
    _record(f'c3_mixed_{fdm}_vs_oracle', e)
    assert e['dt_reason_same']
    ref_e = c3_reference_errors
    assert e['velocity_rel_l2'] <= mixed_bound('velocity_rel_l2', steps, ref_e, 1e-5), e
    assert e['kinetic_energy_rel'] <= mixed_bound('kinetic_energy_rel', steps, ref_e, 1e-5), e
    assert e['phi_rel_l2'] <= mixed_bound('phi_rel_l2', steps, ref_e, 1e-4), e
    for k, r in e['norm_rel'].items():
        assert r <= (1e-5 if ref_e is None else max(1e-5, 2.0 * ref_e[steps]['norm_rel'][k])), (k, e)
    assert e['div_rms'] < 1e-5, e
    assert e['max_div'] <= 4 * e['max_div_oracle_float32'], e
