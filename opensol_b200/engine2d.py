"""FDTDEngine2D_Ez on the B200: the 2D E_z-polarisation Yee engine of open_sol (open_sol/physics/em/solvers/
fdtd_ez_2d.py:11) re-built as device-resident state behind the C ABI of libopensol_fdtd.so.

The host keeps only the float64 clock, the step counter and the setup rows; fields, coefficients, CPML psi slabs,
line-source profiles and monitor spectra stay in HBM.  ``advance(n)`` hands a whole chunk of n steps to the device:
per-step source values and per-sample DFT phases are precomputed on the host into small tables, so no host work sits
between steps.
"""
from __future__ import annotations

import ctypes

import numpy as np

from . import _native
from .boundaries import build_yee_rows, face_shares
from .constants import DTYPE, EPS0, MU0
from .monitors import dft_phase_table
from .poles import pole_face_sets


class FDTDEngine2D_Ez:
    """Device engine of one 2D E_z simulation (real fields, CPML and periodic faces)."""

    polarization = 'ez'
    FIELDS = {'ez': _native.OS_EZ, 'hx': _native.OS_HX, 'hy': _native.OS_HY}
    _CREATE = 'os_fdtd2d_create'
    KERNEL_KINDS = {0: 'ez2d_interior_kernel', 1: 'ez2d_frame_step_kernel | ez2d_tb_kernel (general)',
                    2: 'ez2d_flux_staged_kernel',
                    3: 'ez2d_h_kernel+ez2d_e_kernel'}

    def __init__(self, domain, boundary_config, device: int = 0):
        boundary_config.require_supported('FDTDEngine2D_Ez')
        self.domain = domain
        self.grid = domain.grid
        self.boundary_config = boundary_config
        self.nx, self.ny = self.grid.nx, self.grid.ny
        self.dt = self.grid.dt
        self.device = int(device)
        self.n_step = 0
        self.time = 0.0
        # curl spacings with kappa folded in, CPML rows per active side (float32)
        self.rows = build_yee_rows(boundary_config, (self.nx, self.ny), float(self.grid.dx), float(self.grid.dx),
                                   float(self.dt))
        self._handle = None
        self._lines = []          # LineSource objects in add order
        self._tfsf = []           # TFSFSource boxes in add order (value rows after the line sources')
        self._poles = []          # (pole, box, cropped mask) in add order
        self._line_ids = {}       # id(source) -> native id
        self._profiles_sent = {}  # id(source) -> profile array last uploaded
        self._monitors = []       # FluxMonitor objects in add order
        self._maps = []           # DFTMonitor objects in add order
        self._probes = []         # FieldProbe objects in add order
        self._step_times = []     # engine clock after each step since reset (the probes' times)
        self._monitor_ids = {}
        self._materials_version = None
        self.sample_interval = 1
        self._sample_interval_sent = None
        self.variant, self.steps_per_launch, self.tile_rows = 1, 3, 0
        self._config_sent = None
        self.h2d_bytes = 0   # host-to-device bytes this engine has uploaded (setup, materials, chunk tables)

    # ------------------------------------------------------------------------------------------- native handle
    @property
    def handle(self):
        """The native engine, created on first device use with its spacings and CPML rows."""
        if self._handle is None:
            lib = _native.load()
            sides = sum(_native.OS_SIDE_BITS[face] for face, on in self.boundary_config.cpml_sides.items() if on)
            grid = _native.OsGrid2D(self.nx, self.ny, int(self.boundary_config.periodic_x),
                                    int(self.boundary_config.periodic_y), int(self.boundary_config.cpml_npml),
                                    sides, self.device)
            h = ctypes.c_void_p()
            create = getattr(lib, self._CREATE)
            _native.check(create(ctypes.byref(grid), ctypes.byref(h)), self._CREATE)
            self._handle = h
            c = self.rows.curl
            _native.check(lib.os_fdtd2d_set_spacings(h, _native.fptr(c['inv_dx_e']), _native.fptr(c['inv_dx_h']),
                                                     _native.fptr(c['inv_dy_e']), _native.fptr(c['inv_dy_h'])))
            for side in self.rows.sides:
                _native.check(lib.os_fdtd2d_set_cpml_side(
                    h, _native.OS_SIDE_BITS[side.face], *(_native.fptr(np.ascontiguousarray(getattr(side, n)))
                                                          for n in ('b_e', 'a_e', 'inv_e', 'b_h', 'a_h', 'inv_h'))))
        return self._handle

    def close(self):
        if self._handle is not None:
            _native.load().os_fdtd2d_destroy(self._handle)
            self._handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # ------------------------------------------------------------------------------------------- setup
    def attach_line_source(self, source):
        """Register a line source; its profile and the device copy follow at the next sync."""
        self._lines.append(source)

    def attach_flux_monitor(self, monitor):
        self._monitors.append(monitor)
        monitor._reader = lambda m=monitor: self.read_flux_spectra(m)

    def attach_pole(self, pole, box, cropped_mask):
        """Register a Drude / Lorentz pole on a cell box (cropped_mask: its cells); created at the next sync."""
        self._poles.append((pole, box, np.asarray(cropped_mask, dtype=bool)))

    def _pole_coefficients(self, pole):
        """(kind 0 Drude / 1 Lorentz, damping, restoring, drive) float32 of a pole at this engine's dt."""
        coefficients = pole.ade_coefficients(float(self.dt))
        kind = 0 if len(coefficients) == 2 else 1
        damping, restoring, drive = ((coefficients[0], 0.0, coefficients[1]) if kind == 0 else coefficients)
        return kind, damping, restoring, drive

    def _create_pole(self, lib, h, pole, box, cropped):
        """The pole on the device: its cell box with drive = cell mask x drive coefficient."""
        kind, damping, restoring, drive = self._pole_coefficients(pole)
        drive_box = np.ascontiguousarray(cropped.astype(DTYPE) * DTYPE(drive))
        pid = ctypes.c_int32()
        _native.check(lib.os_fdtd2d_add_pole(h, kind, box[0].start, box[0].stop, box[1].start, box[1].stop,
                                             float(damping), float(restoring), _native.fptr(drive_box),
                                             float(DTYPE(1.0 / float(self.dt))), ctypes.byref(pid)))
        return pid.value

    def attach_tfsf(self, source):
        """Register a TFSF plane-wave box; it is created on the device at the next sync."""
        self._tfsf.append(source)

    def attach_probe(self, probe):
        """Register a FieldProbe; it is created on the device at the next sync and records from the step then."""
        if probe.field_component not in self.FIELDS:
            raise ValueError(f"field probe component must be one of {tuple(self.FIELDS)}, got {probe.field_component!r}")
        self._probes.append(probe)
        probe._reader = lambda p=probe: self.read_probe(p)

    def attach_dft_monitor(self, monitor):
        """Register a field-map DFTMonitor; its device sums are created at the next sync."""
        self._maps.append(monitor)
        monitor._reader = lambda m=monitor: self.read_dft_map(m)

    def set_sample_interval(self, m):
        self.sample_interval = int(m)

    def sync_device(self):
        """Bring the device engine up to date with the host setup: coefficients (when the materials changed), new
        sources and monitors, changed profiles, the sample interval."""
        lib = _native.load()
        h = self.handle
        materials = self.domain.materials
        if self._materials_version != materials.version:
            self._upload_materials(lib, h, materials)
            self._materials_version = materials.version
        for source in self._lines:
            profile = np.ascontiguousarray(source.profile, dtype=DTYPE)
            key = id(source)
            if key not in self._line_ids:
                lo, hi = source.span
                sid = ctypes.c_int32()
                _native.check(lib.os_fdtd2d_add_line_source(h, 0 if source.axis == 'x' else 1, source.position, lo,
                                                            hi, _native.fptr(profile), ctypes.byref(sid)))
                self._line_ids[key] = sid.value
            elif self._profiles_sent.get(key) is not source.profile:
                _native.check(lib.os_fdtd2d_set_line_profile(h, self._line_ids[key], _native.fptr(profile)))
            self._profiles_sent[key] = source.profile
        for monitor in self._monitors:
            if id(monitor) not in self._monitor_ids:
                mid = ctypes.c_int32()
                normal = 0 if monitor.axis == 'x' else 1
                _native.check(lib.os_fdtd2d_add_flux_line(h, normal, monitor.position, monitor.span[0],
                                                          monitor.span[1], monitor.n_freqs, ctypes.byref(mid)))
                self._monitor_ids[id(monitor)] = mid.value
        for entry in self._poles:
            if id(entry) not in self._monitor_ids:
                self._monitor_ids[id(entry)] = self._create_pole(lib, h, *entry)
        for source in self._tfsf:
            if id(source) not in self._monitor_ids:
                tid = ctypes.c_int32()
                coef_h = np.zeros(4, dtype=DTYPE)
                coef_e = np.zeros(4, dtype=DTYPE)
                coef_h[:len(source.coef_h)] = source.coef_h
                coef_e[:len(source.coef_e)] = source.coef_e
                _native.check(lib.os_fdtd2d_add_tfsf(
                    h, source.x0, source.x1, source.y0, source.y1, source.aux_cells, source.aux_x0,
                    source.AUX_SOURCE_INDEX, _native.fptr(coef_h), _native.fptr(coef_e), float(source.mur[0]),
                    float(source.mur[1]), _native.fptr(source.aux_coef_h), _native.fptr(source.aux_coef_e),
                    ctypes.byref(tid)))
                self._monitor_ids[id(source)] = tid.value
        for probe in self._probes:
            if id(probe) not in self._monitor_ids:
                pid = ctypes.c_int32()
                _native.check(lib.os_fdtd2d_add_probe(h, probe.ix, probe.iy, self.FIELDS[probe.field_component],
                                                      ctypes.byref(pid)))
                self._monitor_ids[id(probe)] = pid.value
                probe._first_step = self.n_step
        for monitor in self._maps:
            if id(monitor) not in self._monitor_ids:
                mid = ctypes.c_int32()
                xs, ys = monitor.x_slice, monitor.y_slice
                _native.check(lib.os_fdtd2d_add_dft_map(h, xs.start or 0, xs.stop, ys.start or 0, ys.stop,
                                                        monitor.downsample, monitor.n_freqs, ctypes.byref(mid)))
                self._monitor_ids[id(monitor)] = mid.value
        if self._sample_interval_sent != self.sample_interval:
            _native.check(lib.os_fdtd2d_set_sample_interval(h, self.sample_interval))
            self._sample_interval_sent = self.sample_interval
        config = (self.variant, self.steps_per_launch, self.tile_rows)
        if self._config_sent != config:
            _native.check(lib.os_fdtd2d_configure(h, *config))
            self._config_sent = config

    def _upload_materials(self, lib, h, materials):
        arrays = [materials.get(name) for name in ('eps_r', 'sigma_e', 'mu_r', 'sigma_m')]
        arrays = [None if a is None else np.ascontiguousarray(a, dtype=DTYPE) for a in arrays]
        _native.check(lib.os_fdtd2d_set_materials(h, *(_native.fptr(a) for a in arrays), float(self.dt),
                                                  float(DTYPE(EPS0)), float(DTYPE(MU0))))
        self.h2d_bytes += sum(a.nbytes for a in arrays if a is not None)

    def configure(self, variant=None, steps_per_launch=None, tile_rows=None):
        """Kernel choice (results are bit-identical for every choice): variant 1 = temporally blocked kernels
        advancing steps_per_launch (1..4, default 3) steps per launch with tile_rows rows per interior tile (0, the
        default: chosen from the grid), the frame one step per launch; variant 2 = the same with the blocked general
        kernel on the frame; variant 0 = one H and one E kernel per step."""
        if variant is not None:
            self.variant = int(variant)
        if steps_per_launch is not None:
            self.steps_per_launch = int(steps_per_launch)
        if tile_rows is not None:
            self.tile_rows = int(tile_rows)
        if self._handle is not None:
            self.sync_device()

    AUTOTUNE_ROWS = (32, 48, 64, 96, 128, 192, 256)

    def autotune(self, candidates=AUTOTUNE_ROWS, repeats=4):
        """Time the interior tile heights on this engine's fields and keep the fastest (the simulation state is not
        changed: trial launches write the idle buffer set).  Returns (rows, ms per launch)."""
        self.sync_device()
        arr = (ctypes.c_int32 * len(candidates))(*candidates)
        rows, ms = ctypes.c_int32(), ctypes.c_float()
        _native.check(_native.load().os_fdtd2d_autotune(self.handle, self.steps_per_launch, arr, len(candidates),
                                                        int(repeats), ctypes.byref(rows), ctypes.byref(ms)))
        self.tile_rows = int(rows.value)
        self._config_sent = (self.variant, self.steps_per_launch, self.tile_rows)
        return self.tile_rows, float(ms.value)

    def launch_count(self):
        """Kernels the last advance launched."""
        n = ctypes.c_int64()
        _native.check(_native.load().os_fdtd2d_launch_count(self.handle, ctypes.byref(n)))
        return int(n.value)

    def plan_info(self, steps_per_launch=None):
        """(interior cells, interior tiles, general tiles) of the blocked kernels' plan."""
        T = self.steps_per_launch if steps_per_launch is None else int(steps_per_launch)
        a, b, c = ctypes.c_int64(), ctypes.c_int64(), ctypes.c_int64()
        _native.check(_native.load().os_fdtd2d_plan_info(self.handle, T, ctypes.byref(a), ctypes.byref(b),
                                                         ctypes.byref(c)))
        return int(a.value), int(b.value), int(c.value)

    def set_profiling(self, on):
        _native.check(_native.load().os_fdtd2d_set_profiling(self.handle, int(bool(on))))

    def set_stall_probe(self, wait_ns):
        """Test hook of the bounded waits (0: off): one warp of the next blocked advances waits on a barrier nothing
        completes, at most wait_ns ns, and gives up; the next synchronising call raises RuntimeError."""
        _native.check(_native.load().os_fdtd2d_set_stall_probe(self.handle, int(wait_ns)))

    def kernel_times(self):
        """{kernel kind name: (total device ms, launches)} of the last advance (profiling on)."""
        out = {}
        for kind, name in self.KERNEL_KINDS.items():
            ms, n = ctypes.c_double(), ctypes.c_int64()
            _native.check(_native.load().os_fdtd2d_kernel_times(self.handle, kind, ctypes.byref(ms), ctypes.byref(n)))
            if n.value:
                out[name] = (float(ms.value), int(n.value))
        return out

    # ------------------------------------------------------------------------------------------- stepping
    def chunk_tables(self, n_steps):
        """(line values (n_lines, n_steps), first sample, n_samples, phase table, clock after the chunk): the host
        side of one device chunk.  Clock: t_half = t + dt/2, t_full = t + dt accumulated in float64
        (fdtd_ez_2d.py:76-79)."""
        dt = float(self.dt)
        t = self.time
        t_half = np.empty(n_steps)
        t_full = np.empty(n_steps)
        for k in range(n_steps):
            t_half[k] = t + 0.5 * dt
            t = t + dt
            t_full[k] = t
        rows = self._lines + self._tfsf   # line sources, then TFSF boxes (the device's value-table order)
        values = (np.stack([src.values(t_half) for src in rows]) if rows
                  else np.zeros((0, n_steps), dtype=np.float32))
        m = self.sample_interval
        first_q = self.n_step // m + 1
        last_q = (self.n_step + n_steps) // m
        n_q = max(0, last_q - first_q + 1)
        tables = []
        for monitor in self._monitors + self._maps:   # flux lines, then field maps (the device's table order)
            times = [t_full[q * m - self.n_step - 1] for q in range(first_q, first_q + n_q)]
            tables.append(dft_phase_table(2.0 * np.pi * monitor.frequencies, times, monitor.dt * m))
            if monitor in self._maps and self.polarization == 'hz':   # H_z holds t - dt/2 (monitors.py:283-284)
                tables.append(dft_phase_table(2.0 * np.pi * monitor.frequencies,
                                              [t - 0.5 * monitor.dt for t in times], monitor.dt * m))
        phases = np.concatenate([tb.reshape(-1) for tb in tables]) if tables else np.zeros(0, np.float32)
        return np.ascontiguousarray(values, dtype=np.float32), first_q, n_q, phases, t

    def advance(self, n_steps, tables=None):
        """Run n_steps full Yee steps on the device (asynchronous); `tables` = a chunk_tables(n_steps) result
        prepared earlier for the same clock and step count (a repeated run from reset reuses it)."""
        n_steps = int(n_steps)
        if n_steps <= 0:
            return
        self.sync_device()
        values, first_q, n_q, phases, t_end = tables if tables is not None else self.chunk_tables(n_steps)
        self.h2d_bytes += values.nbytes + phases.nbytes
        _native.check(_native.load().os_fdtd2d_advance(
            self.handle, n_steps, _native.fptr(values) if values.size else None, first_q, n_q,
            _native.fptr(phases) if phases.size else None))
        self._append_step_times(n_steps)
        self.n_step += n_steps
        self.time = t_end

    def _append_step_times(self, n_steps):
        """The clock after each of the next n_steps steps (t_full, accumulated as chunk_tables does): the field
        probes' sample times."""
        if not self._probes:
            self._step_times.extend([float('nan')] * n_steps)   # no probe reads these steps
            return
        dt, t = float(self.dt), self.time
        for _ in range(n_steps):
            t = t + dt
            self._step_times.append(t)

    def set_stream(self, cuda_stream):
        """Enqueue on the caller's CUDA stream (an int cudaStream_t, e.g. torch.cuda.current_stream().cuda_stream;
        None = the engine's own stream)."""
        _native.check(_native.load().os_fdtd2d_set_stream(self.handle, cuda_stream or None))

    def synchronize(self):
        _native.check(_native.load().os_fdtd2d_synchronize(self.handle))

    def last_advance_ms(self):
        ms = ctypes.c_float()
        _native.check(_native.load().os_fdtd2d_last_advance_ms(self.handle, ctypes.byref(ms)))
        return float(ms.value)

    def reset(self):
        """Zero fields, psi and spectra; clock and step count back to 0."""
        _native.check(_native.load().os_fdtd2d_reset(self.handle))
        self.n_step = 0
        self.time = 0.0
        self._step_times = []

    # ------------------------------------------------------------------------------------------- readout
    def read_field(self, name):
        comp = self.FIELDS[name]
        out = np.empty((self.nx, self.ny), dtype=DTYPE)
        _native.check(_native.load().os_fdtd2d_read_field(self.handle, comp, _native.fptr(out)))
        return out

    def write_field(self, name, values):
        comp = self.FIELDS[name]
        arr = np.ascontiguousarray(values, dtype=DTYPE)
        if arr.shape != (self.nx, self.ny):
            raise ValueError(f'{name} must have shape {(self.nx, self.ny)}, got {arr.shape}')
        _native.check(_native.load().os_fdtd2d_write_field(self.handle, comp, _native.fptr(arr)))

    def read_cb(self):
        out = np.empty((self.nx, self.ny), dtype=DTYPE)
        self.sync_device()
        _native.check(_native.load().os_fdtd2d_read_cb(self.handle, _native.fptr(out)))
        return out

    def read_flux_spectra(self, monitor):
        if id(monitor) not in self._monitor_ids:
            self.sync_device()
        mid = self._monitor_ids[id(monitor)]
        n = monitor.n_cells
        e = np.empty((monitor.n_freqs, n, 2), dtype=np.float64)
        h = np.empty((monitor.n_freqs, n, 2), dtype=np.float64)
        _native.check(_native.load().os_fdtd2d_read_flux_spectra(self.handle, mid, _native.dptr(e),
                                                                 _native.dptr(h)))
        return e[..., 0] + 1j * e[..., 1], h[..., 0] + 1j * h[..., 1]

    def read_probe(self, probe):
        """(times float64, values float32) of a FieldProbe since it was added or the last reset."""
        if id(probe) not in self._monitor_ids:
            self.sync_device()
        lib, pid = _native.load(), self._monitor_ids[id(probe)]
        n = ctypes.c_int64()
        _native.check(lib.os_fdtd2d_read_probe(self.handle, pid, None, 0, ctypes.byref(n)))
        values = np.empty(n.value, dtype=np.float32)
        if n.value:
            _native.check(lib.os_fdtd2d_read_probe(self.handle, pid, _native.fptr(values), n.value,
                                                   ctypes.byref(n)))
        first = self.n_step - n.value
        return np.array(self._step_times[first:self.n_step], dtype=np.float64), values

    def read_dft_map(self, monitor):
        """(nf, mx, my) complex64 running DFT of a field-map monitor (E_z); (3, nf, mx, my) = H_z, E_x, E_y on the
        H_z engine."""
        if id(monitor) not in self._monitor_ids:
            self.sync_device()
        parts = 3 if self.polarization == 'hz' else 1
        out = np.empty((parts, monitor.n_freqs, monitor.mx, monitor.my, 2), dtype=np.float32)
        _native.check(_native.load().os_fdtd2d_read_dft_map(self.handle, self._monitor_ids[id(monitor)],
                                                            _native.fptr(out)))
        maps = out.view(np.complex64)[..., 0]
        return maps if parts == 3 else maps[0]

    def state(self):
        """Host copies of the public fields (FDTDEngine2D_Ez.state, fdtd_ez_2d.py:56-67)."""
        materials = self.domain.materials
        return {'ez': self.read_field('ez'), 'hx': self.read_field('hx'), 'hy': self.read_field('hy'),
                'eps_r': materials.array('eps_r'), 'sigma_e': materials.array('sigma_e'), 'jz_total': None,
                'q_accum': None, 'q_accum_time': 0.0}


class FDTDEngine2D_Hz(FDTDEngine2D_Ez):
    """Device engine of one 2D H_z simulation (FDTDEngine2D_Hz, open_sol/physics/em/solvers/fdtd_hz_2d.py:12): H_z at
    the cell centres, E_x / E_y on the hi-y / hi-x faces, face-averaged eps_xx / eps_yy / sigma_e.  Per Yee step an
    interior kernel over the box of plain cells (tile_rows rows per CTA, 0 = chosen per grid) and a border kernel over
    the rest (variant 1), by default two steps per interior launch where the grid allows it, or the in-place
    per-half-step kernels (variant 0); every choice gives bit-identical fields."""

    polarization = 'hz'
    FIELDS = {'hz': _native.OS_HZ_HZ, 'ex': _native.OS_HZ_EX, 'ey': _native.OS_HZ_EY}
    _CREATE = 'os_fdtd2d_hz_create'
    KERNEL_KINDS = {0: 'hz2d_interior_kernel', 1: 'hz2d_border_kernel', 2: 'ez2d_flux_kernel (E_x|E_y, H_z)',
                    3: 'hz2d_h_kernel+hz2d_e_kernel'}

    def __init__(self, domain, boundary_config, device: int = 0):
        super().__init__(domain, boundary_config, device)
        self.variant, self.steps_per_launch, self.tile_rows = 1, 2, 0
        bc = boundary_config
        widths_x, widths_y = domain.kernel_widths()
        self.shares_x = face_shares(widths_x, bc.periodic_x)
        self.shares_y = face_shares(widths_y, bc.periodic_y)

    def _create_pole(self, lib, h, pole, box, cropped):
        """The pole on the device as one face set per E component it reaches (FDTDEngine2D_Hz.add_drude /
        add_lorentz, fdtd_hz_2d.py:441-472): drive = float32 drive coefficient x face weight on each face box."""
        kind, damping, restoring, drive = self._pole_coefficients(pole)
        full = np.zeros((self.nx, self.ny), dtype=bool)
        full[box] = cropped
        bc = self.boundary_config
        ids = []
        for component, fbox, weight in pole_face_sets(full, self.shares_x, self.shares_y, bc.periodic_x,
                                                      bc.periodic_y):
            drive_box = np.ascontiguousarray(DTYPE(drive) * weight)
            pid = ctypes.c_int32()
            _native.check(lib.os_fdtd2d_hz_add_pole(h, kind, component, fbox[0].start, fbox[0].stop, fbox[1].start,
                                                    fbox[1].stop, float(damping), float(restoring),
                                                    _native.fptr(drive_box), float(DTYPE(1.0 / float(self.dt))),
                                                    ctypes.byref(pid)))
            ids.append(pid.value)
        return tuple(ids)

    def _upload_materials(self, lib, h, materials):
        arrays = [materials.get(name) for name in ('eps_xx', 'eps_yy', 'sigma_e', 'mu_r', 'sigma_m')]
        for k in (0, 1):
            if arrays[k] is None:
                arrays[k] = materials.array('eps_xx' if k == 0 else 'eps_yy')
        arrays = [None if a is None else np.ascontiguousarray(a, dtype=DTYPE) for a in arrays]
        shares = [np.ascontiguousarray(a) for a in (*self.shares_x, *self.shares_y)]
        _native.check(lib.os_fdtd2d_hz_set_materials(h, *(_native.fptr(a) for a in arrays),
                                                     *(_native.fptr(a) for a in shares), float(self.dt),
                                                     float(DTYPE(EPS0)), float(DTYPE(MU0))))
        self.h2d_bytes += sum(a.nbytes for a in arrays if a is not None)

    def configure(self, variant=None, steps_per_launch=None, tile_rows=None):
        """variant 1 (default): interior + border kernel per step, tile_rows interior rows per CTA (0 = chosen per
        grid); variant 0: one H_z and one E kernel per step.  steps_per_launch 2 (default) or 1: with 2, where the grid
        has no conductivity, no magnetic cells and rows of a multiple of 4 cells, the interior box advances two steps
        per launch (the border two single steps through a scratch field set, made here) except where the next step is
        a sampled one; a TFSF box or poles keep one step per launch."""
        super().configure(variant, steps_per_launch, tile_rows)

    def autotune(self, candidates=None, repeats=4):
        raise NotImplementedError('the H_z engine chooses its rows per CTA from the grid (configure(tile_rows=...))')

    def plan_info(self, steps_per_launch=None):
        raise NotImplementedError('the H_z engine has no blocked-kernel plan (hz_plan gives its split)')

    def hz_plan(self):
        """(interior cells, border cells) of the variant-1 step (of the two-step launch's box with
        steps_per_launch 2, where it applies)."""
        self.sync_device()
        a, b = ctypes.c_int64(), ctypes.c_int64()
        _native.check(_native.load().os_fdtd2d_hz_plan(self.handle, ctypes.byref(a), ctypes.byref(b)))
        return int(a.value), int(b.value)

    def lossless_form(self):
        """True when the step kernel evaluates the face cb from eps_r (no coefficient arrays stored)."""
        self.sync_device()
        out = ctypes.c_int32()
        _native.check(_native.load().os_fdtd2d_hz_form(self.handle, ctypes.byref(out)))
        return bool(out.value)

    def read_cb(self):
        """(cb_x, cb_y) of the E_x / E_y faces (nx, ny) from the device."""
        self.sync_device()
        cb_x = np.empty((self.nx, self.ny), dtype=DTYPE)
        cb_y = np.empty((self.nx, self.ny), dtype=DTYPE)
        _native.check(_native.load().os_fdtd2d_hz_read_cb(self.handle, _native.fptr(cb_x), _native.fptr(cb_y)))
        return cb_x, cb_y

    def state(self):
        """Host copies of the public fields (FDTDEngine2D_Hz.state, fdtd_hz_2d.py:94-104)."""
        materials = self.domain.materials
        return {'hz': self.read_field('hz'), 'eps_xx': materials.array('eps_xx'),
                'eps_yy': materials.array('eps_yy'), 'sigma_e': materials.array('sigma_e'), 'q_accum': None,
                'q_accum_time': 0.0}
