"""Host-side binding of the cavity solver's C ABI (ctypes).

This module mirrors the reference's Python binding, `python_api.py:1-161`, name for name: the same
`Config` / `Report` / `Diagnostics` records (byte layout fixed by backend.cu:584-597 and
python_api.py:11-28), the same `Solver` methods with the same argument meaning, NumPy shapes and error
behaviour (a non-zero return code raises `RuntimeError` carrying `solver_last_error()`,
python_api.py:82-84).  Code written against the reference's binding runs unchanged against this one.

By default it loads `libcavity_solver.so` from this package (the B200 build).  The `library=` argument
selects another build of the same ABI, e.g. the CPU oracle under `oracle/` or the reference's own
`backend.cu` built under `oracle/_ref/`; tests use that to drive all three through one code path.
"""
import ctypes as ct
import os
from pathlib import Path

import numpy as np

PACKAGE_DIR = Path(__file__).resolve().parent
DEFAULT_LIBRARY = PACKAGE_DIR / 'libcavity_solver.so'


class Config(ct.Structure):
    """Solver settings: 11 int32, 14 double, probe_x[8], probe_y[8]; 288 bytes (backend.cu:584-589)."""
    _fields_ = ([(name, ct.c_int) for name in
                 ('nx', 'ny', 'nz', 'lid_shaped', 'impulse_order', 'adaptive_dt', 'dt_lag', 'phi_extrapolate',
                  'fdm_max_passes', 'grid_stretch', 'n_probes')]
                + [(name, ct.c_double) for name in
                   ('length', 'u_lid', 'nu', 'lz', 'lid_ramp_t', 'reinit_r', 'impulse_order4_ramp',
                    'grid_dx_wall', 'grid_max_aspect', 'dt_fixed', 'dt_max', 'cfl_target', 'diffusion_limit',
                    'fdm_rtol')]
                + [('probe_x', ct.c_double * 8), ('probe_y', ct.c_double * 8)])


class Report(ct.Structure):
    """State of the clock after a step: 48 bytes (backend.cu:590-594)."""
    _fields_ = [('steps', ct.c_longlong), ('time', ct.c_double), ('dt', ct.c_double), ('cfl', ct.c_double),
                ('phi_rel', ct.c_double), ('dt_reason', ct.c_int), ('phi_passes', ct.c_int)]


class Diagnostics(ct.Structure):
    """Volume-averaged diagnostics: 8 doubles (backend.cu:595-597)."""
    _fields_ = [(name, ct.c_double) for name in
                ('kinetic_energy', 'enstrophy', 'umax', 'div_rms', 'cfl_rate', 'gauge_ratio', 'gauge_x', 'gauge_y')]


DT_REASONS = ('fixed_DT', 'DT_MAX', 'CFL', 'viscous')
FIELD_NUMBER = {'u': 0, 'v': 1, 'w': 2, 'mx': 3, 'my': 4, 'mz': 5, 'phi': 6}
FIELD_NAMES = ('u', 'v', 'w', 'mx', 'my', 'mz', 'phi')
# precision forms of the B200 build (cavity_set_precision); other builds ignore it
PRECISION = {'fp64': 0, 'mixed': 1}


def pointer(a):
    """C pointer to a NumPy array's data; None stays None (= NULL)."""
    return None if a is None else a.ctypes.data_as(ct.c_void_p)


def load_library(library=None):
    """Open a build of the solver ABI and declare the argument types that need one."""
    library = Path(DEFAULT_LIBRARY if library is None else library)
    if not library.is_file():
        raise FileNotFoundError(f'solver library not built: {library} (run __graft_entry__.build())')
    lib = ct.CDLL(str(library))
    lib.solver_last_error.restype = ct.c_char_p
    lib.solver_set_clock.argtypes = [ct.c_double, ct.c_longlong, ct.c_double]
    lib.solver_kick.argtypes = [ct.c_void_p, ct.c_void_p, ct.c_void_p, ct.c_double, ct.c_int]
    lib.solver_add_statistics.argtypes = [ct.c_double, ct.c_void_p]
    if hasattr(lib, 'cavity_set_precision'):
        lib.cavity_set_precision.argtypes = [ct.c_int]
    return lib


def _field_buffer(shape, name, out):
    """`out`, checked, or a new array for a field: float64 for phi, float32 for the others (python_api.py)."""
    dtype = np.float64 if name == 'phi' else np.float32
    if out is None:
        return np.empty(shape, dtype=dtype)
    if out.shape != tuple(shape) or out.dtype != dtype or not out.flags['C_CONTIGUOUS']:
        raise ValueError(f'{name}: output buffer must be C-contiguous {dtype.__name__} of shape {tuple(shape)}')
    return out


def make_config(settings):
    """Config record from a settings dict, copying fields by name; `probes` is a list of (x/L, y/L)."""
    config = Config()
    for name, _ in Config._fields_:
        if name in settings:
            setattr(config, name, settings[name])
    probes = list(settings.get('probes', ()))[:8]
    config.n_probes = len(probes)
    for k, (px, py) in enumerate(probes):
        config.probe_x[k], config.probe_y[k] = px, py
    return config


class Solver:
    """One cavity on the device.  Create, `initialize()`, then `step()` in a loop (python_api.py:40-161).

    `precision` selects the form of the B200 build ('fp64' default, or 'mixed'); it is ignored by
    builds of the ABI that have a single form (the oracle, the reference).
    """

    def __init__(self, settings, library=None, precision=None):
        self.lib = load_library(library)
        if precision is not None and hasattr(self.lib, 'cavity_set_precision'):
            self.call('cavity_set_precision', PRECISION[precision])
        config = make_config(settings)
        self.config = config
        self.call('solver_create', ct.byref(config))
        nx, ny, nz = config.nx, config.ny, config.nz
        self.nx, self.ny, self.nz = nx, ny, nz
        # NumPy shapes [z, y, x] of every field (python_api.py:73-74)
        self.shapes = {'u': (nz, ny, nx + 1), 'v': (nz, ny + 1, nx), 'w': (nz + 1, ny, nx), 'phi': (nz, ny, nx)}
        self.shapes.update(mx=self.shapes['u'], my=self.shapes['v'], mz=self.shapes['w'])
        self.grid = {}
        for axis, (name, n) in enumerate((('x', nx), ('y', ny), ('z', nz))):
            faces, centres = np.empty(n + 1), np.empty(n)
            self.call('solver_grid', axis, pointer(faces), pointer(centres))
            self.grid[name] = (faces, centres)

    def call(self, name, *args):
        if getattr(self.lib, name)(*args):
            raise RuntimeError(self.lib.solver_last_error().decode())

    def initialize(self, v_noise=None, w_noise=None):
        v = None if v_noise is None else np.ascontiguousarray(v_noise, dtype=np.float64)
        w = None if w_noise is None else np.ascontiguousarray(w_noise, dtype=np.float64)
        self.call('solver_initialize', pointer(v), pointer(w))

    def step(self):
        r = Report()
        self.call('solver_step', ct.byref(r))
        return self._as_dict(r)

    def report(self):
        r = Report()
        self.call('solver_report', ct.byref(r))
        return self._as_dict(r)

    @staticmethod
    def _as_dict(r):
        d = {name: getattr(r, name) for name, _ in Report._fields_}
        d['dt_reason'] = DT_REASONS[r.dt_reason]
        return d

    def kick(self, noise, amplitude, passes):
        n = [np.ascontiguousarray(a, dtype=np.float64) for a in noise]
        self.call('solver_kick', pointer(n[0]), pointer(n[1]), pointer(n[2]), float(amplitude), int(passes))

    def diagnostics(self):
        d = Diagnostics()
        self.call('solver_diagnostics', ct.byref(d))
        return {name: getattr(d, name) for name, _ in Diagnostics._fields_}

    def field(self, name, out=None):
        """A field as python_api returns it; `out` (an addition): a C-contiguous array of the field's shape and
        dtype to copy into, so that a caller reading fields repeatedly reuses its buffers."""
        out = _field_buffer(self.shapes[name], name, out)
        self.call('solver_get_field', FIELD_NUMBER[name], pointer(out))
        return out

    def field64(self, name):
        """A field in double precision (an addition of the B200 build and the oracle)."""
        out = np.empty(self.shapes[name], dtype=np.float64)
        self.call('cavity_get_field_f64', FIELD_NUMBER[name], pointer(out))
        return out

    def set_field(self, name, values):
        a = np.ascontiguousarray(values, dtype=np.float64 if name == 'phi' else np.float32)
        if a.shape != self.shapes[name]:
            raise ValueError(f'{name}: shape {a.shape}, expected {self.shapes[name]}')
        self.call('solver_set_field', FIELD_NUMBER[name], pointer(a))

    def set_clock(self, time, steps, last_dt):
        self.call('solver_set_clock', float(time), int(steps), float(last_dt))

    def probes(self):
        out = np.zeros(2 * self.config.n_probes, dtype=np.float32)
        self.call('solver_probes', pointer(out))
        return out

    def add_statistics(self, weight):
        """Add the mid-span field to the statistics; returns the centreline sample (u, v, uu, vv, ww)."""
        line = np.empty((5, self.nx))
        self.call('solver_add_statistics', float(weight), pointer(line))
        return line

    def statistics(self):
        sums = np.empty((6, self.ny, self.nx))
        self.call('solver_get_statistics', pointer(sums))
        return dict(zip(('u', 'v', 'uu', 'vv', 'ww', 'uv'), sums))

    def set_statistics(self, sums):
        a = np.ascontiguousarray([sums[k] for k in ('u', 'v', 'uu', 'vv', 'ww', 'uv')], dtype=np.float64)
        self.call('solver_set_statistics', pointer(a))

    def midplane(self):
        out = np.empty((4, self.ny, self.nx), dtype=np.float32)
        self.call('solver_midplane', pointer(out))
        return out

    def q_volume(self, colour_w=True):
        q = np.empty((self.nz, self.ny, self.nx), dtype=np.float32)
        colour = np.empty_like(q)
        self.call('solver_q_volume', int(bool(colour_w)), pointer(q), pointer(colour))
        return q, colour

    def close(self):
        self.call('solver_destroy')


class Cavity:
    """Handle API of the B200 build (cavity_* functions): one of several independent cavities.

    Same operations as `Solver` on an explicit handle, plus asynchronous stepping, device-memory
    accounting and device-timed benchmark steps.
    """

    def __init__(self, settings, precision='fp64', library=None):
        self.lib = load_library(library)
        L = self.lib
        L.cavity_create.argtypes = [ct.c_void_p, ct.c_int, ct.POINTER(ct.c_void_p)]
        for name in ('cavity_destroy', 'cavity_initialize', 'cavity_step', 'cavity_step_async', 'cavity_sync',
                     'cavity_get_field', 'cavity_set_field', 'cavity_probes', 'cavity_diagnostics',
                     'cavity_time_steps'):
            getattr(L, name).restype = ct.c_int
        L.cavity_destroy.argtypes = [ct.c_void_p]
        L.cavity_initialize.argtypes = [ct.c_void_p, ct.c_void_p, ct.c_void_p]
        L.cavity_step.argtypes = [ct.c_void_p, ct.c_void_p]
        L.cavity_step_async.argtypes = [ct.c_void_p, ct.c_int]
        L.cavity_sync.argtypes = [ct.c_void_p, ct.c_void_p]
        L.cavity_get_field.argtypes = [ct.c_void_p, ct.c_int, ct.c_void_p]
        L.cavity_set_field.argtypes = [ct.c_void_p, ct.c_int, ct.c_void_p]
        L.cavity_probes.argtypes = [ct.c_void_p, ct.c_void_p]
        L.cavity_diagnostics.argtypes = [ct.c_void_p, ct.c_void_p]
        L.cavity_device_bytes.argtypes = [ct.c_void_p]
        L.cavity_device_bytes.restype = ct.c_longlong
        L.cavity_estimate_bytes.argtypes = [ct.c_void_p, ct.c_int]
        L.cavity_estimate_bytes.restype = ct.c_longlong
        L.cavity_time_steps.argtypes = [ct.c_void_p, ct.c_int, ct.c_int, ct.c_int, ct.c_void_p, ct.c_void_p]
        L.cavity_kernels_per_step.argtypes = [ct.c_void_p, ct.c_int]
        L.cavity_pressure_passes.argtypes = [ct.c_void_p]
        L.cavity_pressure_passes.restype = ct.c_longlong
        L.cavity_last_error.restype = ct.c_char_p
        self.config = make_config(settings)
        nx, ny, nz = self.config.nx, self.config.ny, self.config.nz
        self.nx, self.ny, self.nz = nx, ny, nz
        self.n_cell = nx * ny * nz
        self.shapes = {'u': (nz, ny, nx + 1), 'v': (nz, ny + 1, nx), 'w': (nz + 1, ny, nx), 'phi': (nz, ny, nx)}
        self.shapes.update(mx=self.shapes['u'], my=self.shapes['v'], mz=self.shapes['w'])
        self.handle = ct.c_void_p()
        self._call('cavity_create', ct.byref(self.config), PRECISION[precision], ct.byref(self.handle))

    def _call(self, name, *args):
        if getattr(self.lib, name)(*args):
            raise RuntimeError(self.lib.cavity_last_error().decode())

    def initialize(self, v_noise=None, w_noise=None):
        v = None if v_noise is None else np.ascontiguousarray(v_noise, dtype=np.float64)
        w = None if w_noise is None else np.ascontiguousarray(w_noise, dtype=np.float64)
        self._call('cavity_initialize', self.handle, pointer(v), pointer(w))

    def step(self):
        r = Report()
        self._call('cavity_step', self.handle, ct.byref(r))
        return Solver._as_dict(r)

    def step_async(self, count=1):
        self._call('cavity_step_async', self.handle, int(count))

    def sync(self):
        r = Report()
        self._call('cavity_sync', self.handle, ct.byref(r))
        return Solver._as_dict(r)

    def field(self, name, out=None):
        out = _field_buffer(self.shapes[name], name, out)
        self._call('cavity_get_field', self.handle, FIELD_NUMBER[name], pointer(out))
        return out

    def set_field(self, name, values):
        dtype = np.float64 if name == 'phi' else np.float32
        a = np.ascontiguousarray(values, dtype=dtype).reshape(self.shapes[name])
        self._call('cavity_set_field', self.handle, FIELD_NUMBER[name], pointer(a))

    def report(self):
        r = Report()
        self.lib.cavity_report.argtypes = [ct.c_void_p, ct.c_void_p]
        self._call('cavity_report', self.handle, ct.byref(r))
        return Solver._as_dict(r)

    def set_clock(self, time, steps, last_dt):
        self.lib.cavity_set_clock.argtypes = [ct.c_void_p, ct.c_double, ct.c_longlong, ct.c_double]
        self._call('cavity_set_clock', self.handle, float(time), int(steps), float(last_dt))

    def probes(self):
        out = np.zeros(2 * self.config.n_probes, dtype=np.float32)
        self._call('cavity_probes', self.handle, pointer(out))
        return out

    def device_bytes(self):
        return int(self.lib.cavity_device_bytes(self.handle))

    def kernels_per_step(self, passes_per_stage):
        return int(self.lib.cavity_kernels_per_step(self.handle, int(passes_per_stage)))

    def pressure_passes(self):
        return int(self.lib.cavity_pressure_passes(self.handle))

    def time_steps(self, warmup, steps, flush_l2=True):
        """Device time (ms) of each of `steps` steps after `warmup`, and of its momentum-sweep launches."""
        ms = np.zeros(steps, dtype=np.float32)
        kms = np.zeros(steps, dtype=np.float32)
        self._call('cavity_time_steps', self.handle, int(warmup), int(steps), int(bool(flush_l2)), pointer(ms),
                   pointer(kms))
        return ms, kms

    def autotune(self, steps=6):
        """Pick the fastest launch shapes for this cavity by timing `steps` steps per candidate (state restored);
        returns (march z-chunks, FP64 transform tile, FP64 pass form (0 six launches, 1 one cooperative launch,
        2 three paired launches, -1 the size rule), ms per step).  See cavity_autotune."""
        L = self.lib
        L.cavity_autotune.argtypes = [ct.c_void_p, ct.c_int, ct.c_void_p, ct.c_void_p, ct.c_void_p, ct.c_void_p]
        chunks, tile, fused, ms = ct.c_int(0), ct.c_int(0), ct.c_int(0), ct.c_float(0)
        self._call('cavity_autotune', self.handle, int(steps), ct.byref(chunks), ct.byref(tile), ct.byref(fused),
                   ct.byref(ms))
        return chunks.value, tile.value, fused.value, ms.value

    def kernel_times(self):
        """Mean device time per step (ms, three stages) of the sweeps, projection starts, residuals of their
        guesses, finishes and the transforms of each stage's first pressure pass, over the last `time_steps`
        call."""
        self.lib.cavity_kernel_times.argtypes = [ct.c_void_p, ct.c_void_p]
        self.lib.cavity_kernel_times.restype = ct.c_int
        ms = np.zeros(5, dtype=np.float64)
        self._call('cavity_kernel_times', self.handle, pointer(ms))
        return dict(zip(('sweep', 'projection_start', 'guess_residual', 'finish', 'transforms'), (float(v) for v in ms)))

    def step_outputs_async(self, count=1, statistics=False):
        """Queue `count` steps, each followed on the device by its probe values and, if `statistics`, by the
        mid-span statistics weighted with that step's dt."""
        self.lib.cavity_step_outputs_async.argtypes = [ct.c_void_p, ct.c_int, ct.c_int]
        self._call('cavity_step_outputs_async', self.handle, int(count), int(bool(statistics)))

    def sync_outputs(self, max_steps=4096):
        """Wait for the queued steps; (report, probe values of each queued step as [steps, 2 * n_probes])."""
        L = self.lib
        L.cavity_sync_outputs.argtypes = [ct.c_void_p, ct.c_void_p, ct.c_void_p, ct.c_int, ct.c_void_p]
        r = Report()
        out = np.zeros((max_steps, 2 * self.config.n_probes), dtype=np.float32)
        n = ct.c_int(0)
        self._call('cavity_sync_outputs', self.handle, ct.byref(r), out.ctypes.data_as(ct.c_void_p), int(max_steps),
                   ct.byref(n))
        return Solver._as_dict(r), out[:n.value]

    def statistics(self):
        out = np.empty(6 * self.nx * self.ny, dtype=np.float64)
        self.lib.cavity_get_statistics.argtypes = [ct.c_void_p, ct.c_void_p]
        self._call('cavity_get_statistics', self.handle, out.ctypes.data_as(ct.c_void_p))
        return out

    def add_statistics(self, weight):
        line = np.empty(5 * self.nx, dtype=np.float64)
        self.lib.cavity_add_statistics.argtypes = [ct.c_void_p, ct.c_double, ct.c_void_p]
        self._call('cavity_add_statistics', self.handle, float(weight), line.ctypes.data_as(ct.c_void_p))
        return line

    def checkpoint(self, device_buffer=None):
        """The complete state (fields, potential history, dt lag, clock, statistics): into a new host array, or
        into `device_buffer` (a device pointer of at least `checkpoint_bytes()` bytes)."""
        L = self.lib
        L.cavity_checkpoint_save.argtypes = [ct.c_void_p, ct.c_void_p, ct.c_int]
        if device_buffer is not None:
            self._call('cavity_checkpoint_save', self.handle, ct.c_void_p(device_buffer), 1)
            return device_buffer
        out = np.empty(self.checkpoint_bytes(), dtype=np.uint8)
        self._call('cavity_checkpoint_save', self.handle, out.ctypes.data_as(ct.c_void_p), 0)
        return out

    def restore(self, checkpoint):
        """Load a state saved by `checkpoint` (a host array, or an int device pointer)."""
        L = self.lib
        L.cavity_checkpoint_load.argtypes = [ct.c_void_p, ct.c_void_p, ct.c_int]
        if isinstance(checkpoint, np.ndarray):
            self._call('cavity_checkpoint_load', self.handle, checkpoint.ctypes.data_as(ct.c_void_p), 0)
        else:
            self._call('cavity_checkpoint_load', self.handle, ct.c_void_p(checkpoint), 1)

    def checkpoint_bytes(self):
        self.lib.cavity_checkpoint_bytes.argtypes = [ct.c_void_p]
        self.lib.cavity_checkpoint_bytes.restype = ct.c_longlong
        return int(self.lib.cavity_checkpoint_bytes(self.handle))

    def close(self):
        if self.handle:
            self._call('cavity_destroy', self.handle)
            self.handle = ct.c_void_p()


class Batch:
    """Cavities of one precision form stepped together (cavity_batch_* functions): every kernel launch of a
    batched step covers all of them, whatever their grid sizes.  With `capacity` above the number of cavities
    the batch has empty slots (its cavities then need one grid size); `set_member` puts a cavity into a slot or
    empties it without rebuilding the batch's graphs.  The cavities stay ordinary `Cavity` handles between steps
    (fields, probes, diagnostics); take a cavity out of the batch, or close the batch, before closing it."""

    def __init__(self, cavities, capacity=None):
        if not cavities:
            raise ValueError('a batch needs at least one cavity')
        cavities = list(cavities)
        capacity = len(cavities) if capacity is None else max(int(capacity), len(cavities))
        self.slots = cavities + [None] * (capacity - len(cavities))
        self.lib = L = cavities[0].lib
        L.cavity_batch_create_slots.argtypes = [ct.c_void_p, ct.c_int, ct.c_int, ct.POINTER(ct.c_void_p)]
        L.cavity_batch_set_member.argtypes = [ct.c_void_p, ct.c_int, ct.c_void_p]
        L.cavity_batch_step_async.argtypes = [ct.c_void_p, ct.c_int]
        L.cavity_batch_sync.argtypes = [ct.c_void_p, ct.c_void_p]
        L.cavity_batch_destroy.argtypes = [ct.c_void_p]
        L.cavity_batch_part_times.argtypes = [ct.c_void_p, ct.c_int, ct.c_void_p]
        handles = (ct.c_void_p * len(cavities))(*[c.handle.value for c in cavities])
        self.handle = ct.c_void_p()
        self._call('cavity_batch_create_slots', handles, len(cavities), capacity, ct.byref(self.handle))

    @property
    def cavities(self):
        return [c for c in self.slots if c is not None]

    def free_slots(self):
        return [i for i, c in enumerate(self.slots) if c is None]

    def set_member(self, slot, cavity):
        """Put `cavity` into slot `slot`, or empty the slot (None); no steps may be queued."""
        self._call('cavity_batch_set_member', self.handle, int(slot), None if cavity is None else cavity.handle)
        self.slots[slot] = cavity

    def _call(self, name, *args):
        if getattr(self.lib, name)(*args):
            raise RuntimeError(self.lib.cavity_last_error().decode())

    def step_async(self, count=1):
        self._call('cavity_batch_step_async', self.handle, int(count))

    def part_times(self, steps=4):
        """Mean device time per step (ms, three stages) of the sweeps, the projection starts with their guesses'
        residuals, the first pressure pass of each stage and the finishes, over `steps` ordinary steps through an
        instrumented graph (cavity_batch_part_times)."""
        ms = (ct.c_double * 4)()
        self._call('cavity_batch_part_times', self.handle, int(steps), ms)
        return dict(zip(('sweep', 'start', 'first_pass', 'finish'), list(ms)))

    def sync(self):
        """Wait for the queued steps; the report of every slot (None for an empty slot)."""
        reports = (Report * len(self.slots))()
        self._call('cavity_batch_sync', self.handle, reports)
        return [Solver._as_dict(r) if c is not None else None for r, c in zip(reports, self.slots)]

    def close(self):
        if self.handle:
            self._call('cavity_batch_destroy', self.handle)
            self.handle = ct.c_void_p()


def estimate_bytes(settings, precision='fp64', library=None):
    """Device bytes a cavity with these settings would hold (for admission against a memory budget)."""
    lib = load_library(library)
    lib.cavity_estimate_bytes.argtypes = [ct.c_void_p, ct.c_int]
    lib.cavity_estimate_bytes.restype = ct.c_longlong
    return int(lib.cavity_estimate_bytes(ct.byref(make_config(settings)), PRECISION[precision]))
