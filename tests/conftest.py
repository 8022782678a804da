"""Test configuration: the `gpu` marker, and import paths for the package, the oracle build and the cases."""
import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]
for p in (ROOT, ROOT / 'tests', ROOT / 'tests' / 'golden'):
    if str(p) not in sys.path:
        sys.path.insert(0, str(p))


def pytest_configure(config):
    config.addinivalue_line('markers', 'gpu: needs a CUDA GPU (B200); run with -m gpu')


@pytest.fixture(scope='session')
def oracle_libs():
    """Paths of the two oracle builds (built on demand with g++)."""
    sys.path.insert(0, str(ROOT / 'oracle'))
    import build_oracle
    build_oracle.build_oracle()
    return {'fp64': ROOT / 'oracle' / 'libcavity_oracle.so', 'fp32': ROOT / 'oracle' / 'libcavity_oracle32.so'}
