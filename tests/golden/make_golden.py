"""Generate the golden fixtures of tests/golden/ from the reference's own solver.

Runs every case of `cases.py` through the reference's backend.cu, built unchanged for sm_100a by
`oracle/build_oracle.py` into `oracle/_ref/libcavity_solver.so`, and stores all outputs as
`tests/golden/<case>.npz`.  It needs a CUDA GPU (the reference has no CPU path).  Usage, from the
repository root on a GPU machine:

    python tests/golden/make_golden.py [output_dir]

Inputs are not stored: `cases.py` regenerates them from integer seeds.
"""
import sys
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))
sys.path.insert(0, str(Path(__file__).resolve().parent))

from cases import CASES, run_case  # noqa: E402
from les_impulse3d_64_b200.api import Solver  # noqa: E402

REFERENCE_LIBRARY = ROOT / 'oracle' / '_ref' / 'libcavity_solver.so'


def main():
    out_dir = Path(sys.argv[1]) if len(sys.argv) > 1 else Path(__file__).resolve().parent
    out_dir.mkdir(parents=True, exist_ok=True)
    for name, case in CASES.items():
        res = run_case(lambda s: Solver(s, library=REFERENCE_LIBRARY), case)
        np.savez_compressed(out_dir / f'{name}.npz', **res)
        print(f'{name}: {len(res)} arrays, final t={float(res["final.time"]):.6g} '
              f'passes={int(res["final.phi_passes"])}', flush=True)


if __name__ == '__main__':
    main()
