"""The CPU oracle against the golden fixtures made by the reference's own backend.cu on a B200.

The float build carries the fields in float like the reference, so it must agree to float rounding of a
few operations; the FP64 build differs from the reference by the reference's own float rounding.
"""
from pathlib import Path

import numpy as np
import pytest

from cases import CASES, run_case
from les_impulse3d_64_b200.api import Solver
from parity import compare

GOLDEN = Path(__file__).resolve().parent / 'golden'


@pytest.mark.parametrize('name', sorted(CASES))
def test_oracle_fp32_matches_reference(oracle_libs, name):
    ref = dict(np.load(GOLDEN / f'{name}.npz'))
    out = run_case(lambda s: Solver(s, library=oracle_libs['fp32']), CASES[name])
    assert compare(out, ref, field_rtol=1e-6, passes='exact') == []


@pytest.mark.parametrize('name', sorted(CASES))
def test_oracle_fp64_matches_reference(oracle_libs, name):
    ref = dict(np.load(GOLDEN / f'{name}.npz'))
    out = run_case(lambda s: Solver(s, library=oracle_libs['fp64']), CASES[name])
    assert compare(out, ref, field_rtol=2e-5, passes='at_most', div_atol=1e-5) == []
