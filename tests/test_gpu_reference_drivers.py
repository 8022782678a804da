"""The reference's own front end drives this build unchanged.

The reference's `python_api.py`, `main.py` and `validate_gpu.py` are copied from the reference checkout
named by CAVITY_REFERENCE_DIR into a temporary folder beside this build's `libcavity_solver.so` (python_api
loads the library from its own folder, python_api.py:43-53).  Skipped when CAVITY_REFERENCE_DIR is unset:
the checkout is not part of this repository.

* `python validate_gpu.py` runs unchanged and passes its checks (validate_gpu.py:37-58: finite fields,
  div_rms < 1e-5, zero wall faces, dt * cfl_rate = 0.4 when the step is CFL-limited).
* `main.advance` (main.py:342-363) runs a short TEST-mesh run with two kicks and the statistics window, then
  `save_checkpoint` / `load_checkpoint` (main.py:159-191), once on this build and once on the FP64 oracle
  under the same file name; the probe histories, statistics and fields agree to 1e-10.
"""
import json
import os
import shutil
import subprocess
import sys
from pathlib import Path

import numpy as np
import pytest

from les_impulse3d_64_b200.api import DEFAULT_LIBRARY

pytestmark = pytest.mark.gpu
ROOT = Path(__file__).resolve().parents[1]
DRIVERS = ('python_api.py', 'main.py', 'validate_gpu.py')


def reference_dir():
    folder = os.environ.get('CAVITY_REFERENCE_DIR')
    if not folder or not all((Path(folder) / f).is_file() for f in DRIVERS):
        pytest.skip('CAVITY_REFERENCE_DIR does not name a reference checkout with ' + ', '.join(DRIVERS))
    return Path(folder)


def stage(tmp, library):
    tmp.mkdir(parents=True, exist_ok=True)
    for f in DRIVERS:
        shutil.copy(reference_dir() / f, tmp / f)
    shutil.copy(library, tmp / 'libcavity_solver.so')
    return tmp


def run_python(folder, *args, timeout=600):
    return subprocess.run([sys.executable, *args], cwd=folder, capture_output=True, text=True, timeout=timeout)


def test_validate_gpu_passes_unchanged(tmp_path):
    folder = stage(tmp_path / 'ours', DEFAULT_LIBRARY)
    res = run_python(folder, 'validate_gpu.py')
    out = res.stdout + res.stderr
    assert res.returncode == 0, out
    for line in ('PASS  finite after 60 steps', 'PASS  divergence-free', 'PASS  no flow through the walls',
                 'PASS  CFL-limited dt', 'ALL CHECKS PASSED'):
        assert line in out, out


# a short run of the reference's front end: kicks after t = 0.02 and 0.06, statistics from t = 0.03, then a
# checkpoint written and read back by main.py's own functions
FRONT_END_RUN = r'''
import json, sys
import numpy as np
import main as front
from python_api import Solver
s = dict(vars(front))
s.update(MESH='TEST', LID_RAMP_T=0.0, KICK_T=0.02, KICK_COUNT=2, KICK_EVERY=0.04, KICK_AMP=0.01,
         STATS_START_T=0.03, STATS_WINDOW_T=0.05)
sim = Solver(front.native_settings(s))
sim.initialize(*front.initial_noise(sim, s))
run = front.Run(sim, s)
reports = [front.advance(run) for _ in range(40)]
front.save_checkpoint(run, 'ck.npz')
sim2 = Solver(front.native_settings(s))
sim2.initialize()
run2 = front.Run(sim2, s)
front.load_checkpoint(run2, 'ck.npz')
reports += [front.advance(run2) for _ in range(5)]
out = {k: sim2.field(k) for k in ('u', 'v', 'w', 'mx', 'my', 'mz', 'phi')}
out.update({'stat_' + k: v for k, v in sim2.statistics().items()})
out['probes'] = np.array(run2.probe_v)
out['window'] = run2.window.mean()
np.savez('front_end.npz', **out)
json.dump([{k: r[k] for k in ('steps', 'time', 'dt', 'dt_reason', 'phi_passes')} for r in reports],
          open('reports.json', 'w'))
sim.close(); sim2.close()
'''


def test_main_advance_with_kicks_statistics_and_checkpoint_matches_oracle(tmp_path, oracle_libs):
    results = {}
    for name, library in (('ours', DEFAULT_LIBRARY), ('oracle', oracle_libs['fp64'])):
        folder = stage(tmp_path / name, library)
        (folder / 'front_end_run.py').write_text(FRONT_END_RUN)
        res = run_python(folder, 'front_end_run.py')
        assert res.returncode == 0, res.stdout + res.stderr
        assert '[kick 1/2]' in res.stdout and '[kick 2/2]' in res.stdout, res.stdout
        results[name] = (dict(np.load(folder / 'front_end.npz')), json.loads((folder / 'reports.json').read_text()))
    (ours, rep_ours), (orc, rep_orc) = results['ours'], results['oracle']
    assert [(r['steps'], r['dt_reason'], r['phi_passes']) for r in rep_ours] == \
           [(r['steps'], r['dt_reason'], r['phi_passes']) for r in rep_orc]
    assert np.abs(ours['stat_u']).max() > 0
    for k, b in orc.items():
        a = ours[k]
        tol = 2.0 ** -22 if a.dtype == np.float32 else 1e-10     # float outputs: to the last float bit
        err = float(np.abs(a.astype(np.float64) - b).max() / max(np.abs(b).max(), 1e-30))
        assert err <= tol, (k, err)
