"""Fault injection through the inputs on the B200 build: no device fault is involved; the errors are the
device-side decisions of the step (NaN CFL rate, NaN right-hand side, no convergence) read back by the host."""
import pytest

from faults import SCENARIOS
from les_impulse3d_64_b200.api import Solver

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize('precision', ['fp64', 'mixed'])
@pytest.mark.parametrize('name', sorted(SCENARIOS))
def test_gpu_fault(name, precision):
    SCENARIOS[name](lambda s: Solver(s, precision=precision))
