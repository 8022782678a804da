"""B200-native cavity solver: the time step of an Eulerian-impulse lid-driven-cavity Navier-Stokes solver
(staggered MAC grid, 4th-order Lamb vector, SSP-RK3, fast-diagonalisation pressure projection) as sm_100a
CUDA kernels behind the reference's `solver_*` C ABI (libcavity_solver.so in this folder).

`api.Solver` is the ctypes binding (the reference's python_api.Solver interface); `build()` compiles the
library.  There is no CPU path: without the compiled library or a GPU the calls fail.
"""
from .api import Config, Diagnostics, Report, Solver, load_library  # noqa: F401
from ._build import LIBRARY, build  # noqa: F401

__all__ = ['Config', 'Diagnostics', 'Report', 'Solver', 'load_library', 'build', 'LIBRARY']
