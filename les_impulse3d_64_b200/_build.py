"""Build of libcavity_solver.so for sm_100a (nvcc, in-tree, no JIT cache)."""
import os
import shutil
import subprocess
from pathlib import Path

PACKAGE = Path(__file__).resolve().parent
ROOT = PACKAGE.parent
CSRC = PACKAGE / 'csrc'
LIBRARY = PACKAGE / 'libcavity_solver.so'
CUDA_HOME = Path(os.environ.get('CUDA_HOME', '/usr/local/cuda'))
ARCH = ['-gencode', 'arch=compute_100a,code=sm_100a']


def sources():
    return sorted(CSRC.glob('*.cu')) + sorted(CSRC.glob('*.cpp'))


def _stale(target, deps):
    return not target.exists() or any(d.stat().st_mtime > target.stat().st_mtime for d in deps)


def nvcc():
    return shutil.which('nvcc') or str(CUDA_HOME / 'bin' / 'nvcc')


def build(force=False, verbose_ptxas=False):
    """Compile the CUDA library if any source changed; returns its path."""
    deps = sources() + sorted(CSRC.glob('*.cuh')) + sorted(CSRC.glob('*.h')) + [ROOT / 'include' / 'cavity_solver.h',
                                                                                Path(__file__)]
    if not force and not _stale(LIBRARY, deps):
        return LIBRARY
    cmd = [nvcc(), *ARCH, '-O3', '-std=c++17', '-lineinfo', '-Xcompiler', '-fPIC,-O2', '-shared',
           f'-I{ROOT / "include"}', f'-I{CSRC}', *[str(s) for s in sources()], '-o', str(LIBRARY)]
    if verbose_ptxas:
        cmd[1:1] = ['-Xptxas', '-v']
    print(' '.join(cmd), flush=True)
    subprocess.run(cmd, check=True)
    return LIBRARY


if __name__ == '__main__':
    import sys
    build(force='--force' in sys.argv, verbose_ptxas='-v' in sys.argv)
