"""Error measures of the north-star parity contract, shared by the contract tests and the fixture script
tests/golden/make_c3_oracle.py: relative L2 differences, the cell divergence of a velocity field, the kinetic
energy, and the z-layers of the reduced C3 fixture."""
import numpy as np

# z-layers of u, v, w and phi kept in the C3 fixture: every 16th layer, and the two mid-span layers
C3_LAYERS = (0, 16, 32, 48, 63, 64, 80, 96, 112, 127)
VELOCITY = ('u', 'v', 'w')


def rel_l2(a, b):
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


def velocity_rel_l2(f, ref):
    """|u - u_ref| / |u_ref| over the three components together."""
    num = sum(float(np.sum((np.asarray(f[k], np.float64) - np.asarray(ref[k], np.float64)) ** 2)) for k in VELOCITY)
    den = sum(float(np.sum(np.asarray(ref[k], np.float64) ** 2)) for k in VELOCITY)
    return float(np.sqrt(num / max(den, 1e-300)))


def _linspace(a, b, count):
    step = (b - a) / (count - 1)
    v = [i * step + a for i in range(count)]
    v[-1] = b
    return v


def axis_faces(n, length, dx_wall):
    """The solver's unrounded face positions of one axis: tanh stretching with the first cell dx_wall found by
    200 bisections, uniform when dx_wall is not below length / n (backend.cu:643-666)."""
    import math
    if dx_wall >= length / n * (1 - 1e-12):
        return _linspace(0.0, length, n + 1)
    xi = _linspace(0.0, 1.0, n + 1)

    def faces(beta):
        return [length * 0.5 * (1.0 + math.tanh(beta * (2 * x - 1)) / math.tanh(beta)) for x in xi]
    lo, hi = 1e-8, 30.0
    for _ in range(200):
        mid = 0.5 * (lo + hi)
        f = faces(mid)
        if f[1] - f[0] < dx_wall:
            hi = mid
        else:
            lo = mid
    f = faces(0.5 * (lo + hi))
    f[0], f[n], f[n // 2] = 0.0, length, 0.5 * length
    return f


def _axis_faces_of(settings, axis):
    n = settings[('nx', 'ny', 'nz')[axis]]
    length = settings['length'] if axis < 2 else n * (settings['lz'] / n)
    dx_wall = min(settings['grid_dx_wall'], length / n) if settings['grid_stretch'] else 1e300
    return axis_faces(n, length, dx_wall)


def check_faces(settings, grid):
    """The restated faces, rounded to float, are the solver's own (solver_grid), bit for bit."""
    for a, name in enumerate('xyz'):
        f = np.asarray(_axis_faces_of(settings, a)).astype(np.float32).astype(np.float64)
        assert np.array_equal(f, grid[name][0]), f'axis {name}: restated faces differ from the solver grid'


def cell_widths(settings, axis):
    """Cell widths of one axis as the solver holds them: differences of the unrounded faces, rounded to float
    (backend.cu:667-699; the aspect cap is not used by these workloads)."""
    assert not settings.get('grid_max_aspect', 0.0) > 0
    f = _axis_faces_of(settings, axis)
    n = len(f) - 1
    return np.asarray([f[i + 1] - f[i] for i in range(n)], np.float64).astype(np.float32).astype(np.float64)


def divergence(f, settings):
    """div u per cell (1/time) on the staggered grid: face differences over the solver's float-rounded cell
    widths, in double arithmetic; u (nz, ny, nx+1), v (nz, ny+1, nx), w (nz+1, ny, nx)."""
    wx, wy, wz = (cell_widths(settings, a) for a in range(3))
    u, v, w = (np.asarray(f[k], np.float64) for k in VELOCITY)
    return (np.diff(u, axis=2) / wx[None, None, :] + np.diff(v, axis=1) / wy[None, :, None]
            + np.diff(w, axis=0) / wz[:, None, None])


def max_abs_divergence(f, settings):
    return float(np.abs(divergence(f, settings)).max())


def as_float32(f):
    return {k: np.asarray(a, np.float32) for k, a in f.items()}


def c3_layers(f):
    """The fixture's z-layers of u, v, w (w on its z-faces of the same index) and phi, float32."""
    return {k: np.asarray(f[k][list(C3_LAYERS)], np.float32) for k in ('u', 'v', 'w', 'phi')}
