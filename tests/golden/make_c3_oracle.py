"""Generate tests/golden/c3_oracle_1000.npz: the FP64 oracle's run of the C3 workload (128^3, beta 2.0,
Re 3200, CFL 0.5, seeded noise 1e-3), 1000 steps.

The oracle (oracle/cavity_oracle.cpp, FP64) needs about ten minutes on sixteen cores for this run, too long
for a test, so its result is kept as a fixture, reduced to what the contract test compares:
  - the per-step dt, time, dt_reason and pressure-pass count;
  - the probe history;
  - after step 1000: the volume diagnostics (kinetic energy, div_rms, ...), the L2 norms of u, v, w and phi
    over the whole field, the max |div u| of the oracle's field and of that field rounded to float32 (the
    floor of any FP32 field), and the z-layers of tests/contract.py C3_LAYERS of u, v, w and phi as float32.

Usage, from the repository root, on any machine with the oracle built (oracle/build_oracle.py):

    OMP_NUM_THREADS=<cores> python tests/golden/make_c3_oracle.py [steps]
"""
import sys
import time
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
ROOT = HERE.parents[1]
for p in (ROOT, ROOT / 'tests', ROOT / 'oracle'):
    sys.path.insert(0, str(p))

import build_oracle  # noqa: E402
import contract  # noqa: E402
from les_impulse3d_64_b200 import workloads  # noqa: E402
from les_impulse3d_64_b200.api import Solver  # noqa: E402

OUT = HERE / 'c3_oracle_1000.npz'


def main():
    steps = int(sys.argv[1]) if len(sys.argv) > 1 else workloads.C3['steps']
    build_oracle.build_oracle()
    w = workloads.C3
    sim = Solver(w['settings'], library=ROOT / 'oracle' / 'libcavity_oracle.so')
    t0 = time.time()
    try:
        sim.initialize(*workloads.initial_noise(sim.shapes, w['noise'], w['seed']))

        def progress(n, _):
            print(f'step {n}: {time.time() - t0:.0f} s', flush=True)

        run = workloads.run_protocol(sim, w, steps=steps, snapshots=range(50, steps + 1, 50), on_snapshot=progress)
        fields = {k: sim.field64(k) for k in ('u', 'v', 'w', 'phi')}
        diag = sim.diagnostics()
        grid = sim.grid
    finally:
        sim.close()
    contract.check_faces(w['settings'], grid)      # the widths behind max_div are the solver's
    out = {f'run.{k}': (v.astype(str) if k == 'dt_reason' else v) for k, v in run.items()
           if k not in ('kick_ke', 'centreline')}
    out.update({f'diag.{k}': np.float64(v) for k, v in diag.items()})
    out.update({f'norm.{k}': np.float64(np.linalg.norm(a)) for k, a in fields.items()})
    out['max_div'] = np.float64(contract.max_abs_divergence(fields, w['settings']))
    out['max_div_float32'] = np.float64(contract.max_abs_divergence(contract.as_float32(fields), w['settings']))
    out.update({f'layer.{k}': a for k, a in contract.c3_layers(fields).items()})
    out['layers'] = np.asarray(contract.C3_LAYERS)
    out['steps'] = np.int64(steps)
    np.savez_compressed(OUT, **out)
    print(f'wrote {OUT} ({OUT.stat().st_size / 1e6:.1f} MB) after {time.time() - t0:.0f} s', flush=True)


if __name__ == '__main__':
    main()
