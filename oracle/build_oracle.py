"""Build recipe for the test-side checkers (test infrastructure, never part of the product).

* `oracle/libcavity_oracle.so`   - the CPU restatement of the reference's time step in FP64
                                   (`cavity_oracle.cpp` with ORACLE_REAL=double), OpenMP.
* `oracle/libcavity_oracle32.so` - the same restatement carrying the fields in FP32, the precision the
                                   reference's backend.cu uses (ORACLE_REAL=float); it pins the
                                   restatement against the reference's own outputs at float level.
* `oracle/_ref/libcavity_solver.so` - the reference's own `backend.cu`, compiled unchanged from the
                                   reference checkout with its own flags (build_windows.bat:4:
                                   `-O2 -std=c++17 --fmad=false ... -lcublas`) plus the sm_100a target.
                                   Built only where the checkout exists; the .so then travels with the
                                   repository snapshot to the GPU machine, where it produces the golden
                                   fixtures and serves as a parity and timing point.

Both oracle builds export the same 18 `solver_*` functions as the reference, so one ctypes binding
drives the oracle, the reference and the B200 build.
"""
import os
import shutil
import subprocess
import sys
from pathlib import Path

HERE = Path(__file__).resolve().parent
# the reference checkout: CAVITY_REFERENCE_DIR, by default where this machine keeps it
REFERENCE_SOURCE = Path(os.environ.get('CAVITY_REFERENCE_DIR', '/root/reference')) / 'backend.cu'
CUDA_HOME = Path(os.environ.get('CUDA_HOME', '/usr/local/cuda'))


def _stale(target, sources):
    return not target.exists() or any(s.stat().st_mtime > target.stat().st_mtime for s in sources)


def _run(cmd):
    print(' '.join(str(c) for c in cmd), flush=True)
    subprocess.run([str(c) for c in cmd], check=True)


def build_oracle(force=False):
    src = HERE / 'cavity_oracle.cpp'
    for real, name in (('double', 'libcavity_oracle.so'), ('float', 'libcavity_oracle32.so')):
        out = HERE / name
        if force or _stale(out, [src, Path(__file__)]):
            # -ffp-contract=off: no fused multiply-add, as the reference's --fmad=false
            _run(['g++', '-O2', '-std=c++17', '-fopenmp', '-ffp-contract=off', '-fPIC', '-shared',
                  f'-DORACLE_REAL={real}', src, '-o', out])


def build_reference(force=False):
    """Compile the reference's backend.cu for sm_100a into oracle/_ref (skipped without the checkout)."""
    if not REFERENCE_SOURCE.is_file():
        return False
    out_dir = HERE / '_ref'
    out_dir.mkdir(exist_ok=True)
    out = out_dir / 'libcavity_solver.so'
    if force or _stale(out, [REFERENCE_SOURCE, Path(__file__)]):
        nvcc = shutil.which('nvcc') or str(CUDA_HOME / 'bin' / 'nvcc')
        _run([nvcc, '-O2', '-std=c++17', '--fmad=false', '-shared', '-Xcompiler', '-fPIC',
              '-gencode', 'arch=compute_100a,code=sm_100a', REFERENCE_SOURCE, '-o', out,
              '-lcublas', f'-L{CUDA_HOME / "lib64"}', f'-Xlinker', f'-rpath={CUDA_HOME / "lib64"}'])
    return True


def build(force=False):
    build_oracle(force)
    build_reference(force)


if __name__ == '__main__':
    build(force='--force' in sys.argv)
