"""Comparison rules for case outputs (see tests/golden/cases.py) between builds of the solver ABI."""
import numpy as np

EXACT_SUFFIXES = ('.steps', '.dt_reason')
CLOCK_SUFFIXES = ('.dt', '.time', '.cfl')


def max_rel(a, b):
    """max |a - b| / max |b| (0 for empty arrays)."""
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    if a.shape != b.shape:
        return np.inf
    if a.size == 0:
        return 0.0
    return float(np.abs(a - b).max() / max(np.abs(b).max(), 1e-30))


def compare(out, ref, field_rtol, passes='exact', fdm_rtol=1e-9, clock_rtol=1e-6, div_atol=1e-6, keys=None):
    """Failures (list of strings) of `out` against `ref` key by key.

    field_rtol  - max relative difference for fields, probes, statistics, diagnostics
    passes      - 'exact': same number of pressure passes; 'at_most': no more passes than `ref`;
                  'any': not compared (a different transform precision converges in a different count)
    """
    bad = []
    for key in (ref.keys() if keys is None else keys):
        if key not in out:
            bad.append(f'{key}: missing')
            continue
        a, b = np.asarray(out[key]), np.asarray(ref[key])
        if key.endswith('.phi_rel'):
            if not float(a) <= fdm_rtol:
                bad.append(f'{key}: {float(a):.3e} > {fdm_rtol}')
        elif key.endswith('.phi_passes'):
            if passes == 'exact' and int(a) != int(b):
                bad.append(f'{key}: {int(a)} != {int(b)}')
            elif passes == 'at_most' and int(a) > int(b):
                bad.append(f'{key}: {int(a)} > {int(b)}')
        elif key.endswith(EXACT_SUFFIXES) or key.startswith('grid.'):
            if not np.array_equal(a, b):
                bad.append(f'{key}: {a} != {b}')
        elif key.endswith(CLOCK_SUFFIXES):
            if max_rel(a, b) > clock_rtol:
                bad.append(f'{key}: rel {max_rel(a, b):.2e}')
        elif key == 'diag.div_rms':
            if abs(float(a) - float(b)) > div_atol:
                bad.append(f'{key}: {float(a):.3e} vs {float(b):.3e}')
        elif key in ('diag.gauge_x', 'diag.gauge_y'):
            continue        # location of a maximum: ties between faces may break either way
        else:
            r = max_rel(a, b)
            if not r <= field_rtol:
                bad.append(f'{key}: rel {r:.2e}')
    return bad
