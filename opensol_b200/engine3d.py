"""FDTDEngine3D on the B200: open_sol's 3D Yee engine (open_sol/physics/em3d/engine3d.py:157-554) for a Cartesian
uniform grid with one real field set and float32 fields, as device-resident state behind the os_fdtd3d_* C ABI.

Host side, computed as the reference computes it: the kappa-folded curl spacings (engine3d.py:189-203), the CPML
layer rows of every axis with CPML (physics/em3d/boundaries3d.py:207-243), the hi-face shares
(physics/em/yee_grid.py:119-125), the uint16 material index with its per-id tables and the PEC wall layers
(engine3d.py:337-369, material_index3d.py), the float64 clock, per-step dipole amplitudes and per-sample DFT phases.
Device side: the six fields, psi slabs, material ids and tables, dipoles and the flux monitors' complex128 sums.
``advance(n)`` enqueues n steps with no host synchronisation.
"""
from __future__ import annotations

import ctypes

import numpy as np

from . import _native
from .boundaries import cpml_axis_profiles, cpml_recursion, cpml_side_rows, face_shares  # noqa: F401
from .constants import DTYPE
from .domain3d import AXES
from .material_index3d import build_material_index
from .monitors import dft_phase_table

MAX_MATERIAL_IDS = 65535
REQUIRED_ARRAYS = ('eps_r', 'sigma_e', 'mu_r')
OPTIONAL_ARRAYS = ('eps_xx', 'eps_yy', 'sigma_m')


class CPMLLayers3D:
    """CPML layers of one axis (lo and hi stacked): int32 row maps grid row -> psi row (-1 outside) and float32
    recursion b and gain = a x bulk inverse spacing per psi row, for the 'e' (cell centre) and 'h' (hi face) kinds."""

    def __init__(self, axis, n_rows, row_map_e, b_e, gain_e, row_map_h, b_h, gain_h):
        self.axis, self.n_rows = axis, n_rows
        self.row_map_e, self.b_e, self.gain_e = row_map_e, b_e, gain_e
        self.row_map_h, self.b_h, self.gain_h = row_map_h, b_h, gain_h


def yee_rows_3d(config, shape, widths, periodic, dt):
    """(inv_e per axis, inv_h per axis, {axis: CPMLLayers3D}): the curl spacings with kappa folded in and the layer
    rows (engine3d.py:189-203, boundaries3d.py:207-243)."""
    npml = int(config.cpml_npml)
    inv_e, inv_h, layers = [], [], {}
    for axis_index, axis in enumerate(AXES):
        w = np.asarray(widths[axis_index], dtype=np.float64)
        inverse_e = 1.0 / w
        inverse_h = 1.0 / (0.5 * (w + np.roll(w, -1)))
        if not periodic[axis_index]:
            inverse_h[-1] = 0.0
        n = shape[axis_index]
        pml_dx = float(max(w[0], w[-1]))
        se, ke, ae, sh, kh, ah = cpml_axis_profiles(config, n, axis, pml_dx)
        inv_e.append((inverse_e / ke).astype(DTYPE))
        inv_h.append((inverse_h / kh).astype(DTYPE))
        sides = [cpml_side_rows(side, n, npml) for side in ('lo', 'hi') if config.cpml_sides[f'{axis}_{side}']]
        if not sides:
            continue
        rows = {}
        for kind_index, (kind, sigma, kappa, alpha, inverse) in enumerate((('e', se, ke, ae, inverse_e),
                                                                           ('h', sh, kh, ah, inverse_h))):
            row_map = np.full(n, -1, dtype=np.int32)
            b_rows, gain_rows = [], []
            for position, side in enumerate(sides):
                selected = side[kind_index]
                row_map[selected] = np.arange(position * npml, (position + 1) * npml, dtype=np.int32)
                a, b = cpml_recursion(sigma[selected], kappa[selected], alpha[selected], dt)
                b_rows.append(b)
                gain_rows.append(a * inverse[selected].astype(DTYPE))
            rows[kind] = (row_map, np.concatenate(b_rows).astype(DTYPE), np.concatenate(gain_rows).astype(DTYPE))
        layers[axis_index] = CPMLLayers3D(axis_index, npml * len(sides), *rows['e'], *rows['h'])
    return inv_e, inv_h, layers


class FDTDEngine3D:
    """3D Yee engine of a Domain3D on one B200."""

    def __init__(self, domain, config, precision='single', device=0):
        if precision != 'single':
            raise NotImplementedError('the B200 3D engine steps float32 fields (stepper precision single)')
        config.validate()
        config.require_supported()
        self.domain = domain
        self.config = config
        self.precision = precision
        self.device = int(device)
        self.shape = domain.shape
        self.nx, self.ny, self.nz = self.shape
        self.dt = float(domain.dt)
        self._dt32 = DTYPE(domain.dt)
        self.periodic = tuple(config.periodic(axis) for axis in AXES)
        self.widths = domain.grid_widths
        self.inv_e, self.inv_h, self.cpml = yee_rows_3d(config, self.shape, self.widths, self.periodic, self.dt)
        self.shares = [face_shares(w, p) for w, p in zip(self.widths, self.periodic)]
        self.material_id = None
        self.tables = None
        self.quantisation_errors = {}
        self._quantisation_deltas = {}
        self.time = 0.0
        self.n_step = 0
        self.sample_interval = 1
        self._handle = None
        self._dipoles = []       # (source, device id)
        self._monitors = []      # (monitor, monitor id, [pair ids per plane])
        self.h2d_bytes = 0

    # ---- device handle
    @property
    def handle(self):
        if self._handle is None:
            lib = _native.load()
            grid = _native.OsGrid3D(self.nx, self.ny, self.nz, (ctypes.c_int32 * 3)(*map(int, self.periodic)),
                                    self.device)
            out = ctypes.c_void_p()
            _native.check(lib.os_fdtd3d_create(ctypes.byref(grid), ctypes.byref(out)), 'os_fdtd3d_create')
            self._handle = out.value
            shares = np.concatenate([s for pair in self.shares for s in pair]).astype(DTYPE)
            _native.check(lib.os_fdtd3d_set_rows(self._handle, *(_native.fptr(a) for a in self.inv_e),
                                                 *(_native.fptr(a) for a in self.inv_h), _native.fptr(shares)))
            for axis, layer in self.cpml.items():
                ip = ctypes.POINTER(ctypes.c_int32)
                _native.check(lib.os_fdtd3d_set_cpml_axis(
                    self._handle, axis, layer.n_rows, layer.row_map_e.ctypes.data_as(ip), _native.fptr(layer.b_e),
                    _native.fptr(layer.gain_e), layer.row_map_h.ctypes.data_as(ip), _native.fptr(layer.b_h),
                    _native.fptr(layer.gain_h)))
        return self._handle

    def __del__(self):
        if getattr(self, '_handle', None) is not None:
            try:
                _native.load().os_fdtd3d_destroy(self._handle)
            except Exception:
                pass
            self._handle = None

    # ---- materials (engine3d.py:337-369)
    def material_arrays(self):
        m = self.domain.materials
        names = list(REQUIRED_ARRAYS) + [n for n in OPTIONAL_ARRAYS if m.get(n) is not None]
        return {name: m.array(name) for name in names}

    def rebuild_materials(self):
        """Material index + tables (+ the PEC entry), PEC wall layers, then upload."""
        ids, n_ids = self.build_materials_host()
        t = self.tables
        _native.check(_native.load().os_fdtd3d_set_materials(
            self.handle, ids.ctypes.data_as(ctypes.POINTER(ctypes.c_uint16)), n_ids,
            *(_native.fptr(t[name]) for name in ('t_ex', 't_ey', 't_ez', 't_sig', 't_mu', 't_sm')), self._dt32))
        self.h2d_bytes += ids.nbytes

    def build_materials_host(self):
        """(uint16 ids with the PEC wall layers, ids incl. the PEC entry); sets material_id and tables."""
        arrays = self.material_arrays()
        ids, tables, self.quantisation_errors, deltas = build_material_index(
            arrays, self.shape, MAX_MATERIAL_IDS - 1, self._quantisation_deltas)
        self._quantisation_deltas.update(deltas)
        n_ids = int(tables['eps_r'].size)

        def with_pec(values, pec_value):
            return np.concatenate((values, np.full(1, pec_value, DTYPE))).astype(DTYPE)
        self.tables = {'t_ez': with_pec(tables['eps_r'], -1.0),
                       't_ex': with_pec(tables.get('eps_xx', tables['eps_r']), -1.0),
                       't_ey': with_pec(tables.get('eps_yy', tables['eps_r']), -1.0),
                       't_sig': with_pec(tables['sigma_e'], 0.0), 't_mu': with_pec(tables['mu_r'], 1.0),
                       't_sm': with_pec(tables.get('sigma_m', np.zeros(n_ids, DTYPE)), 0.0)}
        pec_id = np.uint16(n_ids)
        window = self.domain.physical_window()
        for axis_index, axis in enumerate(AXES):
            for side in ('lo', 'hi'):
                if getattr(self.config, f'{axis}_{side}') == 'pec':
                    layer = window[axis_index].start if side == 'lo' else window[axis_index].stop - 1
                    key = [slice(None)] * 3
                    key[axis_index] = slice(layer, layer + 1)
                    ids[tuple(key)] = pec_id
        self.material_id = ids
        return ids, n_ids + 1

    def face_cb(self, component, cell):
        out = ctypes.c_float()
        _native.check(_native.load().os_fdtd3d_face_cb(self.handle, int(component), *map(int, cell),
                                                       ctypes.byref(out)))
        return DTYPE(out.value)

    def face_dual_volume(self, axis, cell) -> float:
        """Dual volume of the E face along axis of cell: the edge between the two centres times the cell face
        (engine3d.py:299-312)."""
        lengths = []
        for other, widths in enumerate(self.widths):
            index = cell[other]
            partner = (index + 1) % widths.size if self.periodic[other] else min(index + 1, widths.size - 1)
            lengths.append(0.5 * (widths[index] + widths[partner]) if other == axis else widths[index])
        return float(np.prod(lengths))

    # ---- sources and monitors on the device
    def attach_dipole(self, source):
        dipole_id = ctypes.c_int32()
        _native.check(_native.load().os_fdtd3d_add_dipole(self.handle, int(source.axis), *map(int, source.cell),
                                                          DTYPE(0.0), ctypes.byref(dipole_id)))
        self._dipoles.append((source, dipole_id.value))

    def set_dipole_weight(self, source):
        for s, dipole_id in self._dipoles:
            if s is source:
                _native.check(_native.load().os_fdtd3d_set_dipole_weight(self.handle, dipole_id, source.weight))

    def attach_flux_monitor(self, monitor):
        lib = _native.load()
        monitor_id = ctypes.c_int32()
        _native.check(lib.os_fdtd3d_add_flux_monitor(self.handle, int(monitor.frequencies.size),
                                                     ctypes.byref(monitor_id)))
        planes = monitor.planes() if hasattr(monitor, 'planes') else [monitor]
        for plane in planes:
            for index, pair in enumerate(plane.pairs):
                pair_id = ctypes.c_int32()
                origin = (ctypes.c_int32 * 3)(*pair['origin'])
                extent = (ctypes.c_int32 * 3)(*pair['extent'])
                _native.check(lib.os_fdtd3d_add_flux_pair(self.handle, monitor_id.value, pair['e_comp'],
                                                          pair['h_comp'], plane.normal_axis, plane.edge, origin,
                                                          extent, ctypes.byref(pair_id)))
                pair['pair_id'] = pair_id.value
            plane._reader = self._pair_reader(plane)
        self._monitors.append(monitor)

    def _pair_reader(self, plane):
        def read(index):
            pair = plane.pairs[index]
            shape = (plane.frequencies.size,) + pair['area'].shape
            e = np.empty(shape, np.complex128)
            h = np.empty(shape, np.complex128)
            _native.check(_native.load().os_fdtd3d_read_flux_pair(
                self.handle, pair['pair_id'], e.view(np.float64).ctypes.data_as(ctypes.POINTER(ctypes.c_double)),
                h.view(np.float64).ctypes.data_as(ctypes.POINTER(ctypes.c_double))))
            return e, h
        return read

    def set_sample_interval(self, m):
        self.sample_interval = int(m)
        _native.check(_native.load().os_fdtd3d_set_sample_interval(self.handle, self.sample_interval))

    # ---- stepping (engine3d.py:497-554)
    def chunk_tables(self, n_steps):
        """(dipole amplitudes (n_dipoles, n_steps), first sample, n_samples, phases, clock after the chunk)."""
        dt = float(self.dt)
        t = self.time
        t_half = np.empty(n_steps)
        t_full = np.empty(n_steps)
        for k in range(n_steps):
            t_half[k] = t + 0.5 * dt
            t = t + dt
            t_full[k] = t
        values = np.empty((len(self._dipoles), n_steps), np.float32)
        for row, (source, _) in enumerate(self._dipoles):
            temporal = source.temporal
            for k in range(n_steps):
                values[row, k] = DTYPE(temporal(float(t_half[k])))
        m = self.sample_interval
        first_q = self.n_step // m + 1
        n_q = max(0, (self.n_step + n_steps) // m - first_q + 1)
        rows = []
        for monitor in self._monitors:
            times = [t_full[q * m - self.n_step - 1] for q in range(first_q, first_q + n_q)]
            table = dft_phase_table(2.0 * np.pi * monitor.frequencies, times, dt * m)
            rows.append(table.reshape(n_q, 2 * monitor.frequencies.size))
        phases = np.concatenate(rows, axis=1).reshape(-1) if rows and n_q else np.zeros(0, np.float32)
        return np.ascontiguousarray(values), first_q, n_q, np.ascontiguousarray(phases, np.float32), t

    def advance(self, n_steps, tables=None):
        n_steps = int(n_steps)
        if n_steps <= 0:
            return
        values, first_q, n_q, phases, t_end = tables if tables is not None else self.chunk_tables(n_steps)
        self.h2d_bytes += values.nbytes + phases.nbytes
        _native.check(_native.load().os_fdtd3d_advance(
            self.handle, n_steps, _native.fptr(values) if values.size else None, first_q, n_q,
            _native.fptr(phases) if phases.size else None))
        self.n_step += n_steps
        self.time = t_end

    def launch_count(self):
        n = ctypes.c_int64()
        _native.check(_native.load().os_fdtd3d_launch_count(self.handle, ctypes.byref(n)))
        return int(n.value)

    def last_advance_ms(self):
        ms = ctypes.c_float()
        _native.check(_native.load().os_fdtd3d_last_advance_ms(self.handle, ctypes.byref(ms)))
        return float(ms.value)

    def synchronize(self):
        _native.check(_native.load().os_fdtd3d_synchronize(self.handle))

    def set_x_chunk(self, planes):
        """x planes per block of the H / E kernels (speed only)."""
        _native.check(_native.load().os_fdtd3d_set_x_chunk(self.handle, int(planes)))

    def set_variant(self, variant):
        """Step form (speed and memory only; results are bit-identical): 0 = the two in-place kernels, 1 = the fused
        kernel on two field and psi sets, 2 = the fused kernel with its planes staged in shared memory by tensor
        copies (rows of a multiple of 8 cells; other grids run form 1), 3 = the lean staged fused kernel (the default:
        four cells a thread, packed arithmetic; z rows of a multiple of 4 cells and at least 144, y at least 17; other
        grids run form 0)."""
        _native.check(_native.load().os_fdtd3d_set_variant(self.handle, int(variant)))

    def set_fused_config(self, config):
        """Launch shape of the fused step kernel of forms 1-3 (0..4, -1 for the form's default; speed only, results
        bit-identical)."""
        _native.check(_native.load().os_fdtd3d_set_fused_config(self.handle, int(config)))

    def interior(self):
        """((i0, i1, j0, j1, k0, k1) of the fused interior box, whether the next advance uses it)."""
        box = (ctypes.c_int32 * 6)()
        fused = ctypes.c_int32()
        _native.check(_native.load().os_fdtd3d_interior(self.handle, box, ctypes.byref(fused)))
        return tuple(int(v) for v in box), bool(fused.value)

    def set_stream(self, cuda_stream):
        _native.check(_native.load().os_fdtd3d_set_stream(self.handle, cuda_stream or None))

    def reset(self):
        _native.check(_native.load().os_fdtd3d_reset(self.handle))
        self.n_step = 0
        self.time = 0.0

    def read_field(self, name):
        out = np.empty(self.shape, dtype=DTYPE)
        _native.check(_native.load().os_fdtd3d_read_field(self.handle, _native.FIELDS_3D.index(name),
                                                          _native.fptr(out)))
        return out

    def write_field(self, name, values):
        values = np.ascontiguousarray(values, dtype=DTYPE)
        if values.shape != self.shape:
            raise ValueError(f'{name} must have shape {self.shape}, got {values.shape}')
        _native.check(_native.load().os_fdtd3d_write_field(self.handle, _native.FIELDS_3D.index(name),
                                                           _native.fptr(values)))

    def state(self):
        return {name: self.read_field(name) for name in _native.FIELDS_3D}
