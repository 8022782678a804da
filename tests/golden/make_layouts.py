"""Record the reference binding's record layouts as a fixture (tests/golden/record_layouts.json).

Reads the reference's `python_api.py` (its ctypes records Config, Report and Diagnostics,
python_api.py:11-28) and writes each record's byte size and (field name, offset) list, so that the ABI test
pins this build's records against the reference's without the reference present.  Usage:

    python tests/golden/make_layouts.py <reference checkout folder>

or with the folder in the environment variable CAVITY_REFERENCE_DIR.
"""
import ctypes as ct
import importlib.util
import json
import os
import sys
from pathlib import Path

OUT = Path(__file__).resolve().parent / 'record_layouts.json'


def layouts(python_api):
    spec = importlib.util.spec_from_file_location('reference_python_api', python_api)
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return {name: {'size': ct.sizeof(rec), 'fields': [[n, getattr(rec, n).offset] for n, _ in rec._fields_]}
            for name, rec in (('Config', mod.Config), ('Report', mod.Report), ('Diagnostics', mod.Diagnostics))}


def main():
    folder = sys.argv[1] if len(sys.argv) > 1 else os.environ.get('CAVITY_REFERENCE_DIR')
    if not folder:
        sys.exit('usage: make_layouts.py <reference checkout folder>')
    OUT.write_text(json.dumps(layouts(Path(folder) / 'python_api.py'), indent=1) + '\n')
    print(f'wrote {OUT}')


if __name__ == '__main__':
    main()
