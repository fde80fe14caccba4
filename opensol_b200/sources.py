"""Temporal waveforms and soft line sources of the B200 FDTD engines.

Waveforms are evaluated on the host in float64 with Python's math functions for a Python float time, exactly as
open_sol's per-step call does (open_sol/core/sources.py:13-100), and rounded once to float32: the device reads a
per-step table of amplitude * temporal(t + dt/2) instead of a per-step host scalar, so a whole chunk of steps runs
without the host.  The sheet-current calibration (profile = cb |sqrt(eps/mu) cos(kappa/2)| 2 / (eta0 w_perp)) is
computed on the host from the line cells' materials (open_sol/physics/em/sources.py:383-392,430-436,582-602).
"""
from __future__ import annotations

import math

import numpy as np

from .constants import C0, DTYPE, EPS0, ETA0, MU0


class GaussianPulse:
    """exp(-((t - t0)/tau)^2) sin(2 pi f0 (t - t0)), tau = 1/(pi bandwidth f0), t0 = 4.5 tau (core/sources.py:23-53)."""

    def __init__(self, f0: float, bandwidth: float = 0.5, t0_factor: float = 4.5):
        self.f0 = f0
        self.bandwidth = bandwidth
        self.tau = 1.0 / (bandwidth * f0 * np.pi)
        self.t0 = t0_factor * self.tau

    def __call__(self, t):
        if isinstance(t, (float, int)):
            delay = t - self.t0
            return math.exp(-(delay / self.tau) ** 2) * math.sin(2.0 * math.pi * self.f0 * delay)
        delay = np.asarray(t, dtype=np.float64) - self.t0
        return np.exp(-(delay / self.tau) ** 2) * np.sin(2.0 * np.pi * self.f0 * delay)

    @property
    def duration(self) -> float:
        return 2.0 * self.t0

    def spectral_limit(self) -> float:
        return self.f0 * (1.0 + 3.72 * self.bandwidth)


class ContinuousWave:
    """(1 - exp(-t / tau_ramp)) sin(2 pi f0 t), tau_ramp = ramp_periods / f0 (core/sources.py:56-78)."""

    def __init__(self, f0: float, ramp_periods: float = 3.0):
        self.f0 = f0
        self.tau_ramp = ramp_periods / f0

    def __call__(self, t):
        if isinstance(t, (float, int)):
            return (1.0 - math.exp(-t / self.tau_ramp)) * math.sin(2.0 * math.pi * self.f0 * t)
        times = np.asarray(t, dtype=np.float64)
        return (1.0 - np.exp(-times / self.tau_ramp)) * np.sin(2.0 * np.pi * self.f0 * times)

    def spectral_limit(self):
        return None


class RickerWavelet:
    """(1 - 2 a^2) exp(-a^2), a = pi f_peak (t - t0), t0 = 4 / f_peak (core/sources.py:81-100)."""

    def __init__(self, f_peak: float, t0_factor: float = 4.0):
        self.f_peak = f_peak
        self.t0 = t0_factor / f_peak

    def __call__(self, t):
        if isinstance(t, (float, int)):
            arg = math.pi * self.f_peak * (t - self.t0)
            return (1.0 - 2.0 * arg * arg) * math.exp(-arg * arg)
        arg = np.pi * self.f_peak * (np.asarray(t, dtype=np.float64) - self.t0)
        return (1.0 - 2.0 * arg ** 2) * np.exp(-arg ** 2)

    @property
    def duration(self) -> float:
        return 2.0 * self.t0

    def spectral_limit(self) -> float:
        return 4.2 * self.f_peak


def make_temporal(waveform, frequency, bandwidth):
    if waveform == 'gaussian':
        return GaussianPulse(frequency, bandwidth)
    if waveform == 'cw':
        return ContinuousWave(frequency)
    if waveform == 'ricker':
        return RickerWavelet(frequency)
    raise ValueError(f"unknown waveform {waveform!r}; valid: 'gaussian', 'cw', 'ricker'")


def carrier_angular_frequency(temporal) -> float:
    frequency = temporal.f_peak if isinstance(temporal, RickerWavelet) else temporal.f0
    return 2.0 * np.pi * float(frequency)


def resolve_frequency(wavelength, frequency) -> float:
    """Source frequency [Hz] from exactly one of wavelength [m] / frequency [Hz] (physics/em/__init__.py:560-568)."""
    if (wavelength is None) == (frequency is None):
        raise ValueError(f"pass exactly one of wavelength or frequency, got wavelength={wavelength}, "
                         f"frequency={frequency}")
    value = float(frequency if frequency is not None else wavelength)
    if not (np.isfinite(value) and value > 0):
        raise ValueError(f"source wavelength / frequency must be finite and > 0, got {value}")
    return value if frequency is not None else C0 / value


class LineSource:
    """Soft E_z sheet current on a grid line: axis 'x' = along x at y-cell `position`, 'y' = along y at x-cell
    `position`, over the half-open cell range `span` (core/sources.py:190-229).  `profile` is the calibrated float32
    injection per cell (set at finalize)."""

    def __init__(self, axis, position, temporal, amplitude=1.0, span=None, profile=None):
        if axis not in ('x', 'y'):
            raise ValueError(f"LineSource axis must be 'x' or 'y', got {axis!r}")
        if span is not None:
            span = (int(span[0]), int(span[1]))
            if not 0 <= span[0] < span[1]:
                raise ValueError(f"LineSource span must be a half-open cell range lo < hi, got {span}")
        self.axis = axis
        self.position = int(position)
        self.temporal = temporal
        self.amplitude = DTYPE(amplitude)
        self.span = span
        self.profile = profile

    def values(self, t_half_list):
        """float32 amplitude * temporal(t) per time (the per-step value of LineSource.inject)."""
        out = np.empty(len(t_half_list), dtype=np.float32)
        temporal, amplitude = self.temporal, self.amplitude
        for k, t in enumerate(t_half_list):
            out[k] = DTYPE(amplitude * temporal(float(t)))
        return out


def sheet_admittance(line_eps, mu_r, sigma_m, omega, normal_spacing, dt):
    """float32 |sqrt(eps/mu) cos(kappa/2)| of the line cells at omega (physics/em/sources.py:430-436 with
    yee_grid.sheet_launch_factor, yee_grid.py:58-65)."""
    permeability = np.asarray(mu_r).astype(np.complex128) - 1j * np.asarray(sigma_m).astype(np.float64) / (omega * MU0)
    vacuum_half_phase = float(normal_spacing) * math.sin(0.5 * float(omega) * float(dt)) / (C0 * float(dt))
    launch = np.sqrt(1.0 - np.asarray(line_eps * permeability, dtype=np.complex128) * vacuum_half_phase ** 2)
    return np.abs(np.sqrt(line_eps / permeability) * launch).astype(DTYPE)


def e_coefficients_host(eps_r, sigma_e, dt):
    """float32 (ca, cb) of cells (fdtd_ez_2d_kernels.py:314-319), used for the calibration line cells."""
    dt = DTYPE(dt)
    eps = np.asarray(eps_r, dtype=DTYPE) * DTYPE(EPS0)
    k = np.asarray(sigma_e, dtype=DTYPE) * dt / (2.0 * eps)
    denom = 1.0 + k
    return (1.0 - k) / denom, (dt / eps) / denom


def _add_pole_susceptibility(line_eps, axis, position, lo, hi, dispersive_regions, omega):
    """Add to the complex eps of the cells [lo, hi) of a grid line (axis 'x': along x at y-cell `position`) the
    susceptibility chi(omega) of every pole region on them, times the region's cell mask there
    (_line_cell_permittivity, physics/em/sources.py:401-427)."""
    for pole, box, cropped in dispersive_regions:
        chi = complex(pole.susceptibility(omega))
        along_box, normal_box = (box[0], box[1]) if axis == 'x' else (box[1], box[0])
        start, stop = max(lo, along_box.start), min(hi, along_box.stop)
        if not (normal_box.start <= position < normal_box.stop and start < stop):
            continue
        along, normal = slice(start - along_box.start, stop - along_box.start), position - normal_box.start
        mask_line = cropped[along, normal] if axis == 'x' else cropped[normal, along]
        line_eps[start - lo:stop - lo] += chi * mask_line


def calibrate_line_source(source, materials, omega, normal_width, dt, dispersive_regions=()):
    """float32 profile of an E_z sheet current (SheetCurrentCalibration.apply for a LineSource,
    physics/em/sources.py:582-602): cb * admittance * 2 / (eta0 w_perp) on the line cells; the line's eps(omega)
    includes the susceptibility of every pole region it crosses (_line_cell_permittivity, :401-427)."""
    lo, hi = source.span
    if source.axis == 'x':
        line = (slice(lo, hi), source.position)
    else:
        line = (source.position, slice(lo, hi))

    def cells(name):
        arr = materials.get(name)
        if arr is None:
            return np.full(hi - lo, DTYPE(materials.DEFAULTS[name]), dtype=DTYPE)
        return np.ascontiguousarray(arr[line])

    eps_line, sigma_line = cells('eps_r'), cells('sigma_e')
    _, cb_line = e_coefficients_host(eps_line, sigma_line, dt)
    line_eps = eps_line.astype(np.complex128) - 1j * sigma_line.astype(np.float64) / (omega * EPS0)
    _add_pole_susceptibility(line_eps, source.axis, source.position, lo, hi, dispersive_regions, omega)
    admittance = sheet_admittance(line_eps, cells('mu_r'), cells('sigma_m'), omega, normal_width, dt)
    weight = np.asarray(2.0 * np.ones(hi - lo) / (float(ETA0) * normal_width), dtype=DTYPE)
    return (cb_line * admittance * weight).astype(DTYPE)


def calibrate_tangential_sheet(source, materials, omega, normal_spacing, dt, shares, normal_widths,
                               dispersive_regions=()):
    """float32 profile of an H_z in-plane sheet current on the hi faces of its line cells (SheetCurrentCalibration.apply
    for a TangentialSheetCurrentSource, physics/em/sources.py:582-602): cb of the E_x (axis 'x') / E_y (axis 'y') faces
    * admittance of the width-weighted face permittivity * 2 / (eta0 w_perp).  `shares` = the (lower, upper) face
    weights and `normal_widths` the kernel cell widths of the axis across the line; each row's eps(omega) includes the
    susceptibility of the pole regions on its cells."""
    lo, hi = source.span
    n = len(normal_widths)
    lower_row, upper_row = source.position, (source.position + 1) % n
    eps_name = 'eps_xx' if source.axis == 'x' else 'eps_yy'

    def row(name, r):
        arr = materials.get(name)
        if arr is None:
            return np.full(hi - lo, DTYPE(materials.DEFAULTS[name]), dtype=DTYPE)
        return np.ascontiguousarray(arr[lo:hi, r] if source.axis == 'x' else arr[r, lo:hi])

    # the faces' ca / cb (fdtd_hz_2d_kernels.py:254-274): face value = lower cell * lower share + upper cell * upper
    lower, upper = shares[0][source.position], shares[1][source.position]
    eps_face = row(eps_name, lower_row) * lower + row(eps_name, upper_row) * upper
    sigma_face = row('sigma_e', lower_row) * lower + row('sigma_e', upper_row) * upper
    _, cb_line = e_coefficients_host(eps_face, sigma_face, dt)

    def row_permittivity(r):
        eps = (row(eps_name, r).astype(np.complex128)
               - 1j * row('sigma_e', r).astype(np.float64) / (omega * EPS0))
        _add_pole_susceptibility(eps, source.axis, r, lo, hi, dispersive_regions, omega)
        return eps

    w_lo, w_hi = float(normal_widths[lower_row]), float(normal_widths[upper_row])
    line_eps = (row_permittivity(lower_row) * w_lo + row_permittivity(upper_row) * w_hi) / (w_lo + w_hi)
    admittance = sheet_admittance(line_eps, row('mu_r', source.position), row('sigma_m', source.position), omega,
                                  normal_spacing, dt)
    weight = np.asarray(2.0 * np.ones(hi - lo) / (float(ETA0) * normal_spacing), dtype=DTYPE)
    return (cb_line * admittance * weight).astype(DTYPE)


class TFSFSource:
    """+x plane wave in vacuum on a total-field box of cells [x0, x1) x [y0, y1) (physics/em/sources.py:206-379,
    _PlaneWaveBox + TFSFSource, or TFSFSourceHz for polarization 'hz', whose corrections act on H_z rows x0 / x1 - 1
    and the scattered E_y / E_x faces around the box): a 1D incident line (20 margin cells at the widths of cells x0 - 1 / x1, the box
    columns between; soft source at aux cell 10 upstream of the box, Mur ends matched to the numerical phase velocity
    at the carrier) advanced on the device beside the grid, and the scattered / total-field corrections on the box
    sides: H_y on rows x0 - 1 and x1 - 1, H_x on columns y0 - 1 and y1 - 1 after the H update, E_z on rows x0 and
    x1 - 1 after the E update.  Incident E_z peak = amplitude [V/m].  The parameters here are host float64 rounded to
    float32 exactly as the reference rounds them."""

    AUX_MARGIN = 20
    AUX_SOURCE_INDEX = 10

    def __init__(self, x0, x1, y0, y1, temporal, dt, amplitude=1.0, cell_widths=None, polarization='ez'):
        x0, x1, y0, y1 = int(x0), int(x1), int(y0), int(y1)
        if not (1 <= x0 < x1 and 1 <= y0 < y1):
            raise ValueError(f"TFSF box [{x0}, {x1}) x [{y0}, {y1}) must be non-empty and keep one scattered-field "
                             f"cell on the lo sides (x0 >= 1, y0 >= 1)")
        dx_cells, dy_cells = (np.asarray(w, dtype=np.float64) for w in cell_widths)
        if x1 >= dx_cells.size or y1 >= dy_cells.size:
            raise ValueError(f"TFSF box [{x0}, {x1}) x [{y0}, {y1}) needs a scattered-field cell on the hi sides of a "
                             f"{dx_cells.size} x {dy_cells.size} grid")
        self.x0, self.x1, self.y0, self.y1 = x0, x1, y0, y1
        self.temporal = temporal
        self.amplitude = float(amplitude)
        dt = float(dt)
        m = self.AUX_MARGIN
        up, down = float(dx_cells[x0 - 1]), float(dx_cells[x1])
        widths = np.concatenate((np.full(m, up), dx_cells[x0:x1], np.full(m, down)))
        face_spacings = 0.5 * (widths[:-1] + widths[1:])
        half_omega_dt = 0.5 * carrier_angular_frequency(temporal) * dt
        courant, cos_half_kappa, mur_lo = _aux_line_terms(up, dt, half_omega_dt)
        _, _, mur_hi = _aux_line_terms(down, dt, half_omega_dt)
        self.source_scale = 2.0 * courant * cos_half_kappa * self.amplitude
        self.mur = (DTYPE(mur_lo), DTYPE(mur_hi))
        side_widths_x = (float(dx_cells[x0]), float(dx_cells[x1 - 1]))
        side_spacings = tuple(0.5 * float(w[i] + w[i + 1]) for w, i in ((dx_cells, x0 - 1), (dx_cells, x1 - 1),
                                                                       (dy_cells, y0 - 1), (dy_cells, y1 - 1)))
        self.polarization = polarization
        if polarization == 'ez':
            self.coef_h = tuple(DTYPE(dt / (MU0 * s)) for s in side_spacings)     # H_y x0-1, x1-1; H_x y0-1, y1-1
            self.coef_e = tuple(DTYPE(dt / (EPS0 * w)) for w in side_widths_x)    # E_z x0, x1-1
            self.aux_coef_h = np.asarray(dt / (MU0 * face_spacings), dtype=DTYPE)  # (n - 1,) hi faces
            self.aux_coef_e = np.asarray(dt / (EPS0 * widths), dtype=DTYPE)        # (n,) centres
        else:
            # TFSFSourceHz (sources.py:352-379): the vacuum pair mu dHz/dt = -dEy/dx, eps0 dEy/dt = -dHz/dx, H_z at
            # the line's centres, E_y on its hi faces (the last face's spacing repeats the last width)
            self.coef_h = tuple(DTYPE(dt / (MU0 * w)) for w in side_widths_x)     # H_z x0, x1-1
            self.coef_e = tuple(DTYPE(dt / (EPS0 * s)) for s in side_spacings)    # E_y x0-1, x1-1; E_x y0-1, y1-1
            self.aux_coef_h = np.asarray(-dt / (MU0 * widths[1:]), dtype=DTYPE)  # H_z centres 1 .. n-1
            self.aux_coef_e = np.asarray(-dt / (EPS0 * np.append(face_spacings, widths[-1])), dtype=DTYPE)
        self.aux_x0 = m
        self.aux_cells = int(widths.size)

    def values(self, t_half):
        """float32 soft-source value of each step: FP32(source_scale * temporal(t + dt/2))."""
        return np.array([DTYPE(self.source_scale * self.temporal(float(t))) for t in t_half], dtype=DTYPE)


def _aux_line_terms(width, dt, half_omega_dt, index=1.0):
    """(Courant number, cos(kappa0 / 2), Mur coefficient) of a uniform 1D line at the carrier
    (physics/em/sources.py:191-204); ValueError when the carrier does not propagate on it."""
    courant = C0 * float(dt) / (float(index) * float(width))
    sin_half_kappa = math.sin(half_omega_dt) / courant
    if sin_half_kappa >= 1.0:
        raise ValueError(f"TFSF: the centre frequency has no propagating wave on the 1D grid (sin(k dx/2) = "
                         f"{sin_half_kappa:.3g} >= 1, at most pi cells per wavelength in the medium); refine the mesh")
    cos_half_kappa = math.sqrt(1.0 - sin_half_kappa ** 2)
    mur_courant = courant * cos_half_kappa / math.cos(half_omega_dt)
    return courant, cos_half_kappa, (mur_courant - 1.0) / (mur_courant + 1.0)
