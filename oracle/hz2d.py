"""ORACLE -- TEST INFRASTRUCTURE ONLY.

Nothing in the product (``opensol_b200``) imports this module.  Only ``tests/`` use it, as the reference the CUDA H_z
engine is compared with.

A CPU restatement of open_sol's 2D H_z-polarisation FDTD path (``Simulation(polarization='hz').run`` ->
``EMPhysics.step`` -> ``FDTDEngine2D_Hz.advance``): setup in numpy, the time step in C (``oracle/hz2d.c``).  The grid,
Courant step, CPML rows, Gaussian pulse, DFT sample interval / phases and the clocks are those of the E_z oracle
(oracle/fdtd2d.py); what differs:

* materials: the dielectric helpers write eps_xx and eps_yy (physics/em/__init__.py:154-156,317-327);
* E face coefficients: width-weighted hi-face means of eps_xx (E_x, along y) and eps_yy (E_y, along x) and sigma_e,
  the partner cell wrapping on a periodic axis and the cell itself on the last face of an open one (face_shares /
  face_partner, physics/em/yee_grid.py:76-84,119-125), then ca / cb as fdtd_hz_2d_kernels.py:254-274;
* H_z coefficients da / db at the cell centres: the E_z engine's (fdtd_2d_base.py:294-);
* the sheet source sits on the hi faces of its line cells (TangentialSheetCurrentSource, physics/em/sources.py:469-480)
  with w_perp = the dual spacing across that face (placement.py:254-265; a line on the last cell of an open axis is
  refused), line eps = width-weighted mean of the line row and the next row of eps_xx (axis 'x') / eps_yy (axis 'y'),
  sigma_e included, cb = cb_x / cb_y (sources.py:582-602);
* flux: E_y (normal x) / E_x (normal y) with H_z, S_x = +E_y H_z, S_y = -E_x H_z (monitors.py:350-362).

Pinned against fixtures generated from the reference itself (``tests/golden/make_golden_hz.py``).
"""
from __future__ import annotations

import ctypes
import os

import numpy as np

from oracle.fdtd2d import (DTYPE, EPS0, ETA0, LIB_DIR, MU0, OracleDrude, OracleEz2D, _make_structs, _ptr, build_cpml,
                           dft_phases, dft_sample_interval, h_coefficients, paint_circle, paint_rect, sheet_admittance,
                           yee_inverse_spacings)


def face_shares(widths, periodic, real):
    """(lower, upper) hi-face weights w_k / (w_k + w_k+1), w_k+1 / (w_k + w_k+1) (yee_grid.py:119-125)."""
    widths = np.asarray(widths, dtype=np.float64)
    partner = np.roll(widths, -1) if periodic else np.concatenate((widths[1:], widths[-1:]))
    return (widths / (widths + partner)).astype(real), (partner / (widths + partner)).astype(real)


def partner_index(n, periodic):
    """Upper partner cell of each hi face of an axis of n cells (yee_grid.face_partner of the indices)."""
    idx = np.arange(int(n))
    return np.roll(idx, -1) if periodic else np.concatenate((idx[1:], idx[-1:]))


def face_coefficient_pair(eps_rel, sigma, dt, real):
    """ca, cb of one face set from face eps_r / sigma (fdtd_hz_2d_kernels.py:254-260), T = real."""
    dt = real(dt)
    eps = eps_rel * real(EPS0)
    k = sigma * dt / (2.0 * eps)
    denom = 1.0 + k
    return ((1.0 - k) / denom).astype(real), ((dt / eps) / denom).astype(real)


def e_face_coefficients(eps_xx, eps_yy, sigma_e, kernel_widths, periodic_x, periodic_y, dt, real):
    """(ca_x, cb_x, ca_y, cb_y) of the E_x (hi-y) and E_y (hi-x) faces (fdtd_hz_2d_kernels.py:263-274)."""
    nx, ny = eps_xx.shape
    lo_y, up_y = face_shares(kernel_widths[1], periodic_y, real)
    lo_x, up_x = face_shares(kernel_widths[0], periodic_x, real)
    pj, pi = partner_index(ny, periodic_y), partner_index(nx, periodic_x)
    exx, eyy, sig = (a.astype(real, copy=False) for a in (eps_xx, eps_yy, sigma_e))
    ca_x, cb_x = face_coefficient_pair(exx * lo_y + exx[:, pj] * up_y, sig * lo_y + sig[:, pj] * up_y, dt, real)
    lx, ux = lo_x[:, None], up_x[:, None]
    ca_y, cb_y = face_coefficient_pair(eyy * lx + eyy[pi] * ux, sig * lx + sig[pi] * ux, dt, real)
    return ca_x, cb_x, ca_y, cb_y


def _make_hz_state(real):
    R = ctypes.c_float if real == np.float32 else ctypes.c_double
    P = ctypes.POINTER(R)

    class StateHz(ctypes.Structure):
        _fields_ = [('nx', ctypes.c_int32), ('ny', ctypes.c_int32), ('periodic_x', ctypes.c_int32),
                    ('periodic_y', ctypes.c_int32), ('hz', P), ('ex', P), ('ey', P), ('ca_x', P), ('cb_x', P),
                    ('ca_y', P), ('cb_y', P), ('da', P), ('db', P), ('inv_dx_e', P), ('inv_dx_h', P),
                    ('inv_dy_e', P), ('inv_dy_h', P), ('npml', ctypes.c_int32), ('cpml_active', ctypes.c_int32 * 4),
                    ('b_e', P * 4), ('a_e', P * 4), ('inv_e', P * 4), ('b_h', P * 4), ('a_h', P * 4),
                    ('inv_h', P * 4), ('psi_e', P * 4), ('psi_h', P * 4)]
    return StateHz


_LIBS = {}


def load_library(real=np.float32):
    """The float32 / float64 build of oracle/hz2d.c (oracle/Makefile, into oracle/_build)."""
    key = np.dtype(real).name
    if key not in _LIBS:
        name = 'libhz2d_oracle_f32.so' if real == np.float32 else 'libhz2d_oracle_f64.so'
        path = os.path.join(LIB_DIR, name)
        if not os.path.exists(path):
            raise RuntimeError(f'oracle library {path} is not built (run: make -C oracle)')
        lib = ctypes.CDLL(path)
        _, Line, Flux = _make_structs(real)
        State = _make_hz_state(real)
        lib.oracle_hz2d_advance.restype = ctypes.c_int
        lib.oracle_hz2d_advance.argtypes = [ctypes.POINTER(State), ctypes.c_int64, ctypes.c_int64, ctypes.c_int32,
                                            ctypes.POINTER(Line), ctypes.c_int32, ctypes.POINTER(Flux),
                                            ctypes.c_int64]
        _LIBS[key] = (lib, State, Line, Flux)
    return _LIBS[key]


def centre_pairs(samples, periodic, stride):
    """(face cells, partner face cells, box cells) slice triples pairing the hi faces of the sampled cells with their
    lo faces (cell - 1); cell 0 pairs with the wrapped last face on a periodic axis, else with its own face
    (monitors.py:156-167 with yee_grid.lower_face, :91-94).  samples: the dft_sample_slice of the box."""
    hi = samples.stop
    if samples.start >= 1:
        return ((samples, slice(samples.start - 1, hi - 1, stride), slice(None)),)
    partner = -1 if periodic else 0
    first = (slice(0, 1), slice(partner, partner + 1 or None), slice(0, 1))
    if hi == 1:
        return (first,)
    return (first, (slice(1, hi), slice(0, hi - 1), slice(1, hi)))


class OracleHz2D(OracleEz2D):
    """The whole 2D H_z path of one simulation on the CPU (same construction calls as OracleEz2D)."""

    def __init__(self, size_x, size_y, dx, npml=15, boundaries=None, courant=None, precision='single'):
        super().__init__(size_x, size_y, dx, npml, boundaries, courant, precision)
        shape = (self.domain.nx, self.domain.ny)
        self.eps_xx = self.eps_r
        self.eps_yy = np.full(shape, DTYPE(1.0), dtype=DTYPE)
        self.hz = np.zeros(shape, dtype=self.real)
        self.ex = np.zeros(shape, dtype=self.real)
        self.ey = np.zeros(shape, dtype=self.real)
        del self.ez, self.hx, self.hy
        self.pole_faces = []   # [pole, comp (0 E_x, 1 E_y), face box, weight on the box, + states] in add order

    def add_dielectric_rectangle(self, x0, y0, x1, y1, eps_r, sigma_e=0.0):
        for array in (self.eps_xx, self.eps_yy):
            paint_rect(self.domain, array, x0, y0, x1, y1, eps_r)
        if sigma_e is not None:
            paint_rect(self.domain, self.sigma_e, x0, y0, x1, y1, sigma_e)

    def add_dielectric_circle(self, cx, cy, radius, eps_r, sigma_e=0.0):
        for array in (self.eps_xx, self.eps_yy):
            paint_circle(self.domain, array, cx, cy, radius, eps_r)
        if sigma_e is not None:
            paint_circle(self.domain, self.sigma_e, cx, cy, radius, sigma_e)

    def add_line_source(self, axis, position, wavelength=None, frequency=None, bandwidth=0.5, amplitude=1.0,
                        span=None):
        """As the E_z line source, on the hi faces of the line cells: w_perp = 1 / inv_d*_h[line cell] of the kernel
        widths (placement.py:254-265)."""
        src = super().add_line_source(axis, position, wavelength, frequency, bandwidth, amplitude, span)
        d = self.domain
        normal = 1 if axis == 'x' else 0
        n_cells = d.ny if axis == 'x' else d.nx
        periodic = d.periodic_y if axis == 'x' else d.periodic_x
        if src.position == n_cells - 1 and not periodic:
            self.sources.pop()
            raise ValueError('the H_z sheet would sit on the outer grid wall')
        _, inv_face = yee_inverse_spacings(d.kernel_widths[normal])
        src.normal_width = 1.0 / float(inv_face[src.position])
        return src

    def add_flux_monitor(self, axis, position, span, wavelengths=None, frequencies=None):
        mon = super().add_flux_monitor(axis, position, span, wavelengths, frequencies)
        mon.flux_sign = 1.0 if mon.normal_axis == 'x' else -1.0
        return mon

    def finalize(self):
        d, real = self.domain, self.real
        self.ca_x, self.cb_x, self.ca_y, self.cb_y = e_face_coefficients(
            self.eps_xx, self.eps_yy, self.sigma_e, d.kernel_widths, d.periodic_x, d.periodic_y, d.dt, real)
        self.da, self.db = h_coefficients(self.sigma_m, self.mu_r, d.dt, real)
        self.cpml_sides, self.curl = build_cpml(d, real)
        for src in self.sources:
            normal = 1 if src.axis == 'x' else 0
            widths = d.kernel_widths[normal]
            lower_row, upper_row = src.position, (src.position + 1) % widths.size
            w_lo, w_hi = float(widths[lower_row]), float(widths[upper_row])
            cell_eps, cb_face = (self.eps_xx, self.cb_x) if src.axis == 'x' else (self.eps_yy, self.cb_y)
            omega = 2.0 * np.pi * float(src.temporal.f0)

            def row(array, r, src=src):
                return array[src.lo:src.hi, r] if src.axis == 'x' else array[r, src.lo:src.hi]

            def row_eps(r, src=src, cell_eps=cell_eps, omega=omega):
                eps = (np.asarray(row(cell_eps, r), dtype=np.complex128)
                       - 1j * np.asarray(row(self.sigma_e, r), dtype=np.float64) / (omega * EPS0))
                # the susceptibility of every pole region on the row's cells (sources.py:401-427)
                for pole, box, cropped in self.poles:
                    along_box, normal_box = (box[0], box[1]) if src.axis == 'x' else (box[1], box[0])
                    start, stop = max(src.lo, along_box.start), min(src.hi, along_box.stop)
                    if not (normal_box.start <= r < normal_box.stop and start < stop):
                        continue
                    along = slice(start - along_box.start, stop - along_box.start)
                    mask_line = cropped[along, r - normal_box.start] if src.axis == 'x' else \
                        cropped[r - normal_box.start, along]
                    eps[start - src.lo:stop - src.lo] += pole.susceptibility(omega) * mask_line
                return eps

            line_eps = (row_eps(lower_row) * w_lo + row_eps(upper_row) * w_hi) / (w_lo + w_hi)
            admittance = sheet_admittance(line_eps, row(self.mu_r, src.position), row(self.sigma_m, src.position),
                                          omega, src.normal_width, float(d.dt))
            weight = np.asarray(2.0 * np.ones(src.hi - src.lo) / (float(ETA0) * src.normal_width), dtype=DTYPE)
            src.profile = (row(cb_face, src.position) * admittance * weight).astype(DTYPE)
        self.sample_interval = dft_sample_interval(float(d.dt), self.sources + self.tfsf,
                                                   [m.frequencies for m in self.monitors + self.maps])
        for m in self.monitors + self.maps:
            m.sample_interval = self.sample_interval
        self.psi_e = {s.name: np.zeros(self._psi_shape(s.name), dtype=real) for s in self.cpml_sides}
        self.psi_h = {s.name: np.zeros(self._psi_shape(s.name), dtype=real) for s in self.cpml_sides}
        self._finalized = True

    def _add_pole(self, pole, mask, set_background):
        """FDTDEngine2D_Hz.add_drude / add_lorentz (fdtd_hz_2d.py:441-472) with _pole_faces (:547-570): the cell region
        (its bounding box and cropped mask, for the sheet calibration's susceptibility) and, per E face set, the face
        average of the float32 cell mask (width-weighted hi-face mean, yee_grid.py:128-142) on the bounding box of its
        positive faces (fdtd_2d_base.py:29-36); set_background writes eps_inf into eps_xx and eps_yy."""
        mask = np.asarray(mask, dtype=bool)
        d = self.domain
        rows = np.flatnonzero(mask.any(axis=1))
        if rows.size:
            cols = np.flatnonzero(mask.any(axis=0))
            box = (slice(int(rows[0]), int(rows[-1]) + 1), slice(int(cols[0]), int(cols[-1]) + 1))
            self.poles.append([pole, box, mask[box].copy()])
        cell = mask.astype(DTYPE)
        lo_y, up_y = face_shares(d.kernel_widths[1], d.periodic_y, DTYPE)
        lo_x, up_x = face_shares(d.kernel_widths[0], d.periodic_x, DTYPE)
        pj, pi = partner_index(d.ny, d.periodic_y), partner_index(d.nx, d.periodic_x)
        weights = (cell * lo_y + cell[:, pj] * up_y, cell * lo_x[:, None] + cell[pi] * up_x[:, None])
        for comp, weight in enumerate(weights):
            positive = weight > 0
            face_rows = np.flatnonzero(positive.any(axis=1))
            if face_rows.size == 0:
                continue
            face_cols = np.flatnonzero(positive.any(axis=0))
            fbox = (slice(int(face_rows[0]), int(face_rows[-1]) + 1), slice(int(face_cols[0]), int(face_cols[-1]) + 1))
            self.pole_faces.append([pole, comp, fbox, weight[fbox].copy()])
        if set_background:
            self.eps_xx[mask] = DTYPE(pole.eps_inf)
            self.eps_yy[mask] = DTYPE(pole.eps_inf)

    def _pole_face_structs(self, R):
        """ctypes records of the pole face sets (states kept across chunks) and float32 1 / dt."""
        P = ctypes.POINTER(R)

        class PoleHz(ctypes.Structure):
            _fields_ = [('kind', ctypes.c_int32), ('comp', ctypes.c_int32), ('i0', ctypes.c_int32),
                        ('i1', ctypes.c_int32), ('j0', ctypes.c_int32), ('j1', ctypes.c_int32), ('damping', R),
                        ('restoring', R), ('drive', P), ('a', P), ('b', P)]

        dt = float(self.domain.dt)
        records = (PoleHz * max(1, len(self.pole_faces)))()
        for q, entry in enumerate(self.pole_faces):
            pole, comp, box, weight = entry[:4]
            if len(entry) == 4:   # first chunk: drive x weight and zero states
                damping, restoring, drive = pole.coefficients(dt)
                entry.extend([DTYPE(drive) * weight, np.zeros(weight.shape, DTYPE), np.zeros(weight.shape, DTYPE),
                              damping, restoring])
            drive_box, a, b, damping, restoring = entry[4:]
            rec = records[q]
            rec.kind = 0 if isinstance(pole, OracleDrude) else 1
            rec.comp, rec.damping, rec.restoring = comp, float(damping), float(restoring)
            rec.i0, rec.i1, rec.j0, rec.j1 = box[0].start, box[0].stop, box[1].start, box[1].stop
            rec.drive, rec.a, rec.b = _ptr(drive_box, R), _ptr(a, R), _ptr(b, R)
        return records, PoleHz, float(DTYPE(1.0 / dt))

    def add_dft_monitor(self, x0, y0, x1, y1, wavelengths=None, frequencies=None, downsample=1):
        """DFTMonitor for 'hz' (physics/em/monitors.py:276-284): H_z, E_x and E_y maps of the sampled cells."""
        mon = super().add_dft_monitor(x0, y0, x1, y1, wavelengths, frequencies, downsample)
        shape = mon.ez_dft.shape
        del mon.ez_dft
        mon.hz_dft, mon.ex_dft, mon.ey_dft = (np.zeros(shape, dtype=np.complex64) for _ in range(3))
        return mon

    def add_field_probe(self, x, y, field_component=None):
        return super().add_field_probe(x, y, field_component or 'hz')

    def add_tfsf(self, x0, y0, x1, y1, wavelength=None, frequency=None, bandwidth=0.5, amplitude=1.0,
                 waveform='gaussian'):
        """TFSFSourceHz (physics/em/sources.py:352-366): the E_z box's cells, line and source scale, with the H_z
        side coefficients dt / (mu0 w) on rows x0 / x1 - 1, the E side ones dt / (eps0 s) on the scattered faces, and
        the incident pair's negated coefficients (H_z at the line's centres 1 .. n-1, E_y on its faces, the last
        face's spacing repeating the last width).  aux_ez holds the incident E_y, aux_hy the incident H_z."""
        box = super().add_tfsf(x0, y0, x1, y1, wavelength, frequency, bandwidth, amplitude, waveform)
        dt = box.dt
        box.coef_h = [DTYPE(dt / (MU0 * w)) for w in box.side_widths_x] + [DTYPE(0.0), DTYPE(0.0)]
        box.coef_e = [DTYPE(dt / (EPS0 * sp)) for sp in box.spacings]
        box.aux_coef_h = np.asarray(-dt / (MU0 * box.widths[1:]), dtype=DTYPE)
        box.aux_coef_e = np.asarray(-dt / (EPS0 * np.append(box.face_spacings, box.widths[-1])), dtype=DTYPE)
        return box

    def _tfsf_hz_structs(self, R, n_steps):
        P = ctypes.POINTER(R)

        class TfsfHz(ctypes.Structure):
            _fields_ = [('x0', ctypes.c_int32), ('x1', ctypes.c_int32), ('y0', ctypes.c_int32),
                        ('y1', ctypes.c_int32), ('aux_x0', ctypes.c_int32), ('aux_n', ctypes.c_int32),
                        ('source_index', ctypes.c_int32), ('coef_h', R * 4), ('coef_e', R * 4), ('mur_lo', R),
                        ('mur_hi', R), ('aux_ey', P), ('aux_hz', P), ('aux_coef_h', P), ('aux_coef_e', P),
                        ('values', ctypes.POINTER(ctypes.c_float))]

        boxes = (TfsfHz * max(1, len(self.tfsf)))()
        dt = float(self.domain.dt)
        for b, box in enumerate(self.tfsf):
            t, values = self.time, np.empty(n_steps, dtype=np.float32)
            for k in range(n_steps):
                values[k] = DTYPE(box.scale * box.temporal(t + 0.5 * dt))
                t = t + dt
            box.values = values
            rec = boxes[b]
            rec.x0, rec.x1, rec.y0, rec.y1 = box.cells
            rec.aux_x0, rec.aux_n, rec.source_index = box.aux_x0, box.aux_ez.size, box.source_index
            for i in range(4):
                rec.coef_h[i], rec.coef_e[i] = float(box.coef_h[i]), float(box.coef_e[i])
            rec.mur_lo, rec.mur_hi = float(box.mur[0]), float(box.mur[1])
            rec.aux_ey, rec.aux_hz = _ptr(box.aux_ez, R), _ptr(box.aux_hy, R)
            rec.aux_coef_h, rec.aux_coef_e = _ptr(box.aux_coef_h, R), _ptr(box.aux_coef_e, R)
            rec.values = _ptr(values, ctypes.c_float)
        return boxes, TfsfHz

    def _fold_maps(self):
        """DFTMonitor.update for 'hz' (monitors.py:281-322): H_z with the phases of t - dt/2, E_x / E_y as the
        float32 mean of a cell's hi face and its lo partner (_centre_pairs) with the phases of t, each added in numpy
        complex64 (_dft_accum_host / _dft_accum_pair_host, :36-41)."""
        d = self.domain
        m = self.sample_interval
        for mon in self.maps:
            omega = 2.0 * np.pi * mon.frequencies
            table_e = dft_phases(omega, self.time, mon.dt * m)
            table_h = dft_phases(omega, self.time - 0.5 * mon.dt, mon.dt * m)
            ph_e = (table_e[:, 0] + 1j * table_e[:, 1]).astype(np.complex64)[:, None, None]
            ph_h = (table_h[:, 0] + 1j * table_h[:, 1]).astype(np.complex64)[:, None, None]
            xs, ys = mon.x_samples, mon.y_samples
            mon.hz_dft += ph_h * np.asarray(self.hz[xs, ys], dtype=np.float32)[None, :, :]
            for faces, partners, box in centre_pairs(ys, d.periodic_y, mon.downsample):
                mean = np.float32(0.5) * (self.ex[xs, faces] + self.ex[xs, partners])
                mon.ex_dft[:, :, box] += ph_e * mean[None, :, :]
            for faces, partners, box in centre_pairs(xs, d.periodic_x, mon.downsample):
                mean = np.float32(0.5) * (self.ey[faces, ys] + self.ey[partners, ys])
                mon.ey_dft[:, box, :] += ph_e * mean[None, :, :]

    def _advance_chunk(self, n_steps):
        lib, State, Line, Flux = load_library(self.real)
        d, real = self.domain, self.real
        R = ctypes.c_float if real == np.float32 else ctypes.c_double
        values, times_full = self.source_values(n_steps)
        first_q, n_q, phase_tables = self._chunk_phase_tables(n_steps, times_full)
        st = State()
        st.nx, st.ny, st.periodic_x, st.periodic_y = d.nx, d.ny, int(d.periodic_x), int(d.periodic_y)
        st.hz, st.ex, st.ey = _ptr(self.hz, R), _ptr(self.ex, R), _ptr(self.ey, R)
        for name in ('ca_x', 'cb_x', 'ca_y', 'cb_y', 'da', 'db'):
            setattr(st, name, _ptr(getattr(self, name), R))
        for name in ('inv_dx_e', 'inv_dx_h', 'inv_dy_e', 'inv_dy_h'):
            setattr(st, name, _ptr(self.curl[name], R))
        keep = self._cpml_state(st, R)
        lines = self._line_structs(Line, values)
        fluxes = self._flux_structs(Flux, phase_tables, first_q, n_q)
        boxes, TfsfHz = self._tfsf_hz_structs(R, n_steps)
        poles, PoleHz, inv_dt = self._pole_face_structs(R)
        lib.oracle_hz2d_advance_full.restype = ctypes.c_int
        lib.oracle_hz2d_advance_full.argtypes = [ctypes.POINTER(State), ctypes.c_int64, ctypes.c_int64, ctypes.c_int32,
                                                 ctypes.POINTER(Line), ctypes.c_int32, ctypes.POINTER(Flux),
                                                 ctypes.c_int64, ctypes.c_int32, ctypes.POINTER(TfsfHz),
                                                 ctypes.c_int32, ctypes.POINTER(PoleHz), R]
        rc = lib.oracle_hz2d_advance_full(ctypes.byref(st), self.n_step, n_steps, len(self.sources), lines,
                                          len(self.monitors), fluxes, self.sample_interval, len(self.tfsf), boxes,
                                          len(self.pole_faces), poles, inv_dt)
        del keep
        if rc != 0:
            raise RuntimeError('oracle phase table does not cover a sample')
        self._clock_after(n_steps, times_full)
