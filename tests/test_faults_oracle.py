"""Fault injection through the inputs, on the CPU oracle (the GPU build runs the same scenarios)."""
import pytest

from faults import SCENARIOS
from les_impulse3d_64_b200.api import Solver


@pytest.mark.parametrize('name', sorted(SCENARIOS))
def test_oracle_fault(oracle_libs, name):
    SCENARIOS[name](lambda s: Solver(s, library=oracle_libs['fp64']))
