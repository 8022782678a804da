"""The C ABI without a GPU: every symbol include/cavity_solver.h declares is exported by the built library,
the record layouts match the reference's (byte sizes and offsets), and calls without a solver fail cleanly."""
import ctypes as ct
import os
import re
from pathlib import Path

import pytest

from les_impulse3d_64_b200 import _build
from les_impulse3d_64_b200.api import Config, Diagnostics, Report, load_library

ROOT = Path(__file__).resolve().parents[1]
HEADER = ROOT / 'include' / 'cavity_solver.h'


def declared_functions():
    text = re.sub(r'/\*.*?\*/', '', HEADER.read_text(), flags=re.S)
    names = re.findall(r'\b((?:solver|cavity)_[a-z0-9_]+)\s*\(', text)
    return sorted(set(names))


@pytest.fixture(scope='module')
def lib():
    _build.build()
    return load_library()


def test_library_exports_every_declared_symbol(lib):
    names = declared_functions()
    assert len([n for n in names if n.startswith('solver_')]) == 18
    missing = [n for n in names if not hasattr(lib, n)]
    assert missing == []


def test_record_layouts():
    assert ct.sizeof(Config) == 288 and Config.length.offset == 48
    assert ct.sizeof(Report) == 48 and ct.sizeof(Diagnostics) == 64


def _our_layouts():
    return {name: {'size': ct.sizeof(rec), 'fields': [[n, getattr(rec, n).offset] for n, _ in rec._fields_]}
            for name, rec in (('Config', Config), ('Report', Report), ('Diagnostics', Diagnostics))}


def test_layouts_match_reference_binding():
    """The reference's own python_api records (python_api.py:11-28), as recorded in
    tests/golden/record_layouts.json by tests/golden/make_layouts.py; and, when CAVITY_REFERENCE_DIR names a
    reference checkout, read live from it as well."""
    import json
    assert _our_layouts() == json.loads((ROOT / 'tests' / 'golden' / 'record_layouts.json').read_text())
    folder = os.environ.get('CAVITY_REFERENCE_DIR')
    if folder and (Path(folder) / 'python_api.py').is_file():
        from make_layouts import layouts
        assert _our_layouts() == layouts(Path(folder) / 'python_api.py')


def test_calls_without_solver_fail_with_message(lib):
    r = Report()
    assert lib.solver_report(ct.byref(r)) == 1
    assert lib.solver_last_error() == b'no solver: call solver_create first'
    assert lib.solver_destroy() == 0


def test_field_output_buffer_is_checked():
    """`field(name, out=...)` copies into a caller's buffer only when it has the field's shape and dtype."""
    import numpy as np
    from les_impulse3d_64_b200.api import _field_buffer
    a = np.zeros((4, 3, 5), dtype=np.float32)
    assert _field_buffer((4, 3, 5), 'u', a) is a
    assert _field_buffer((4, 3, 5), 'phi', None).dtype == np.float64
    for bad in (np.zeros((4, 3, 5), dtype=np.float64), np.zeros((4, 3, 6), dtype=np.float32),
                np.zeros((4, 5, 3), dtype=np.float32).transpose(0, 2, 1)):
        with pytest.raises(ValueError):
            _field_buffer((4, 3, 5), 'u', bad)


def test_config_from_settings():
    """make_config copies the settings by field name and packs up to 8 probes (python_api.py's Config record)."""
    from les_impulse3d_64_b200 import workloads
    from les_impulse3d_64_b200.api import make_config
    s = workloads.C2['settings']
    c = make_config(s)
    for name in ('nx', 'ny', 'nz', 'lid_shaped', 'impulse_order', 'adaptive_dt', 'grid_stretch'):
        assert getattr(c, name) == s[name], name
    for name in ('nu', 'grid_dx_wall', 'cfl_target', 'dt_max', 'reinit_r'):
        assert getattr(c, name) == s[name], name
    assert c.n_probes == 8
    assert [(c.probe_x[k], c.probe_y[k]) for k in range(8)] == list(workloads.PROBES8)
    many = make_config(dict(s, probes=list(workloads.PROBES8) + [(0.3, 0.3)]))
    assert many.n_probes == 8
    assert make_config(dict(s, probes=())).n_probes == 0
