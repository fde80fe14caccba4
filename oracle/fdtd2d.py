"""ORACLE -- TEST INFRASTRUCTURE ONLY.

Nothing in the product (``opensol_b200``) imports this module.  Only ``tests/``, ``__graft_entry__.smoke()`` and the
CPU-baseline leg of ``bench.py`` use it, as the reference the CUDA engine is compared with.

A CPU restatement of open_sol's 2D E_z FDTD path (``Simulation.run`` -> ``EMPhysics.step`` ->
``FDTDEngine2D_Ez.advance``) in two parts:

* setup, in numpy, written from the reference's own numpy expressions so every float32 / float64 rounding matches:
  grid and Courant step (open_sol/core/grid.py:9-17,170-172,184-203), uniform domain with the PML padded outside the
  window (open_sol/core/domain.py:180-197), cell edges / centres / containing cell (core/domain.py:58-81,275-282,
  core/grid.py:175-181), rect / circle masks on float32 centres (core/domain.py:90-112,255-267), material writes
  (core/material_grid.py:56-91), ca/cb/da/db (physics/em/solvers/fdtd_ez_2d_kernels.py:314-340), Yee inverse
  spacings (physics/em/yee_grid.py:11-45), CPML grading and recursion (physics/em/boundaries.py:551-632,671-686) with
  kappa folded into the curl spacings (boundaries.py:778-799, fdtd_2d_base.py:76-84), sheet-current calibration
  (physics/em/sources.py:383-392,430-436,582-602, yee_grid.py:58-65, physics/em/__init__.py:459-473,
  placement.py:223-255), Gaussian pulse (core/sources.py:23-53,221-229), DFT sample interval and phases
  (physics/em/monitors.py:22-24,177-191,219-220), flux readout (monitors.py:240-245,371-379), the engine clock
  (fdtd_ez_2d.py:76-79, fdtd_2d_base.py:470-476) and the runner's stop rule (coupling/runner.py:174-204,
  simulation.py:272-318);
* the time step itself, in C (``oracle/ez2d.c``, float32 or float64 build), called through ctypes.

Pinned against fixtures generated from the reference itself (``tests/golden/make_golden.py``).
"""
from __future__ import annotations

import ctypes
import math
import os
from dataclasses import dataclass, field

import numpy as np

C0 = 299792458.0
EPS0 = 8.8541878128e-12
MU0 = 1.2566370614e-6
ETA0 = np.sqrt(MU0 / EPS0)
DTYPE = np.float32
FACES = ('x_lo', 'x_hi', 'y_lo', 'y_hi')

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_DIR = os.path.join(_HERE, '_build')


# ----------------------------------------------------------------------------------------------- grid and domain

def courant_time_step(dx_min, dy_min, courant_factor=None):
    """open_sol/core/grid.py:9-17."""
    if courant_factor is None:
        courant_factor = 0.99
    inverse_spacing_squared = 1.0 / float(dx_min) ** 2 + 1.0 / float(dy_min) ** 2
    return DTYPE(float(courant_factor) / (C0 * np.sqrt(inverse_spacing_squared)))


def uniform_cell_count(length, dx):
    """open_sol/core/grid.py:170-172."""
    return int(np.ceil(length / dx - 1e-9))


def boundary_preset(name, npml):
    """Face types and PML cells of open_sol's Simulation boundary presets (simulation.py:388-399,
    boundaries.py:293-321)."""
    presets = {'pml': ('cpml',) * 4, 'periodic_x': ('periodic', 'periodic', 'cpml', 'cpml'),
               'periodic_y': ('cpml', 'cpml', 'periodic', 'periodic'), 'periodic': ('periodic',) * 4}
    faces = dict(zip(FACES, presets[name or 'pml']))
    return faces, {face: (npml if kind == 'cpml' else 0) for face, kind in faces.items()}


def containing_cell(coord, edges, first, last):
    """open_sol/core/domain.py:275-282."""
    coord = float(coord)
    snap = 1e-9 * (edges[first + 1] - edges[first])
    index = int(np.searchsorted(edges, coord + snap, side='right')) - 1
    return min(max(index, first), last)


@dataclass
class Domain2D:
    size_x: float
    size_y: float
    dx: float
    npml: int = 15
    boundaries: str = 'pml'
    courant: float = None

    def __post_init__(self):
        self.faces, self.sides = boundary_preset(self.boundaries, self.npml)
        total_x = self.size_x + (self.sides['x_lo'] + self.sides['x_hi']) * self.dx
        total_y = self.size_y + (self.sides['y_lo'] + self.sides['y_hi']) * self.dx
        self.nx = uniform_cell_count(total_x, self.dx)
        self.ny = uniform_cell_count(total_y, self.dx)
        self.grid_dx = DTYPE(self.dx)                      # Grid2D.dx (float32)
        self.dt = courant_time_step(self.dx, self.dx, self.courant)
        self.periodic_x = self.faces['x_lo'] == 'periodic'
        self.periodic_y = self.faces['y_lo'] == 'periodic'
        self.window = (slice(self.sides['x_lo'], self.nx - self.sides['x_hi']),
                       slice(self.sides['y_lo'], self.ny - self.sides['y_hi']))
        self.edges = tuple((np.arange(n + 1) - origin) * float(self.dx)
                           for n, origin in ((self.nx, self.sides['x_lo']), (self.ny, self.sides['y_lo'])))
        self.centers = tuple(0.5 * (e[:-1] + e[1:]) for e in self.edges)
        self.centers_f32 = tuple(c.astype(DTYPE) for c in self.centers)
        self.cell_widths = (np.full(self.nx, float(self.dx)), np.full(self.ny, float(self.dx)))
        self.kernel_widths = (np.full(self.nx, float(self.grid_dx)), np.full(self.ny, float(self.grid_dx)))

    def pos_to_cell_x(self, x):
        return containing_cell(x, self.edges[0], self.window[0].start, self.window[0].stop - 1)

    def pos_to_cell_y(self, y):
        return containing_cell(y, self.edges[1], self.window[1].start, self.window[1].stop - 1)


# ----------------------------------------------------------------------------------------------- materials

def _bbox_slices(centres, lo, hi):
    """Cells whose float32 centre can fall in [lo, hi] with a two-cell margin (the masks are evaluated there with
    the reference's own float32 expression, so restricting the evaluation changes no cell)."""
    a = int(np.searchsorted(centres, lo, side='left')) - 2
    b = int(np.searchsorted(centres, hi, side='right')) + 2
    return slice(max(a, 0), min(b, centres.size))


def paint_rect(domain, array, x0, y0, x1, y1, value):
    """MaterialGrid.assign of Domain.rect_mask (core/domain.py:255-260, core/material_grid.py:56-66)."""
    X, Y = domain.centers_f32
    x_min, x_max = min(x0, x1), max(x0, x1)
    y_min, y_max = min(y0, y1), max(y0, y1)
    sx, sy = _bbox_slices(X, x_min, x_max), _bbox_slices(Y, y_min, y_max)
    Xb, Yb = X[sx][:, None], Y[sy][None, :]
    mask = (Xb >= x_min) & (Xb < x_max) & (Yb >= y_min) & (Yb < y_max)
    np.copyto(array[sx, sy], DTYPE(value), where=mask)


def paint_circle(domain, array, cx, cy, radius, value):
    """MaterialGrid.assign of Domain.circle_mask (core/domain.py:262-267)."""
    X, Y = domain.centers_f32
    sx, sy = _bbox_slices(X, cx - radius, cx + radius), _bbox_slices(Y, cy - radius, cy + radius)
    Xb, Yb = X[sx][:, None], Y[sy][None, :]
    mask = (Xb - cx) ** 2 + (Yb - cy) ** 2 <= radius ** 2
    np.copyto(array[sx, sy], DTYPE(value), where=mask)


def rect_mask(domain, x0, y0, x1, y1):
    """Full-grid bool Domain.rect_mask (core/domain.py:255-260)."""
    mask = np.zeros((domain.nx, domain.ny), dtype=bool)
    X, Y = domain.centers_f32
    x_min, x_max = min(x0, x1), max(x0, x1)
    y_min, y_max = min(y0, y1), max(y0, y1)
    sx, sy = _bbox_slices(X, x_min, x_max), _bbox_slices(Y, y_min, y_max)
    Xb, Yb = X[sx][:, None], Y[sy][None, :]
    mask[sx, sy] = (Xb >= x_min) & (Xb < x_max) & (Yb >= y_min) & (Yb < y_max)
    return mask


def circle_mask(domain, cx, cy, radius):
    """Full-grid bool Domain.circle_mask (core/domain.py:262-267)."""
    mask = np.zeros((domain.nx, domain.ny), dtype=bool)
    X, Y = domain.centers_f32
    sx, sy = _bbox_slices(X, cx - radius, cx + radius), _bbox_slices(Y, cy - radius, cy + radius)
    Xb, Yb = X[sx][:, None], Y[sy][None, :]
    mask[sx, sy] = (Xb - cx) ** 2 + (Yb - cy) ** 2 <= radius ** 2
    return mask


class OracleDrude:
    """DrudePole (physics/em/materials.py:132-157): float32 parameters, ADE coefficients, susceptibility."""

    def __init__(self, omega_p, gamma, eps_inf=1.0):
        self.omega_p, self.gamma, self.eps_inf = DTYPE(omega_p), DTYPE(gamma), DTYPE(eps_inf)

    def coefficients(self, dt):
        g, wp = float(self.gamma), float(self.omega_p)
        denom = 1.0 + g * dt / 2.0
        return DTYPE(-g * dt / denom), DTYPE(0.0), DTYPE((EPS0 * wp ** 2 * dt) / denom)

    def susceptibility(self, omega):
        wp, g = float(self.omega_p), float(self.gamma)
        return complex(-wp ** 2 / (omega ** 2 - 1j * g * omega))


class OracleLorentz:
    """LorentzPole (physics/em/materials.py:160-190)."""

    def __init__(self, delta_eps, omega_0, gamma):
        self.delta_eps, self.omega_0, self.gamma = DTYPE(delta_eps), DTYPE(omega_0), DTYPE(gamma)

    def coefficients(self, dt):
        w0, g, de = float(self.omega_0), float(self.gamma), float(self.delta_eps)
        denom = 1.0 + g * dt / 2.0
        return DTYPE(-g * dt / denom), DTYPE(w0 ** 2 * dt ** 2 / denom), DTYPE(EPS0 * de * w0 ** 2 * dt ** 2 / denom)

    def susceptibility(self, omega):
        w0, g, de = float(self.omega_0), float(self.gamma), float(self.delta_eps)
        return complex(de * w0 ** 2 / (w0 ** 2 - omega ** 2 + 1j * g * omega))


def e_coefficients(sigma, eps_r, dt, real):
    """fdtd_ez_2d_kernels.py:314-319 (numpy twin), T = real."""
    dt = real(dt)
    eps = eps_r.astype(real, copy=False) * real(EPS0)
    k = sigma.astype(real, copy=False) * dt / (2.0 * eps)
    denom = 1.0 + k
    return ((1.0 - k) / denom).astype(real), ((dt / eps) / denom).astype(real)


def h_coefficients(sigma_m, mu_r, dt, real):
    """fdtd_ez_2d_kernels.py:335-340."""
    dt = real(dt)
    mu = mu_r.astype(real, copy=False) * real(MU0)
    k = sigma_m.astype(real, copy=False) * dt / (2.0 * mu)
    denom = 1.0 + k
    return ((1.0 - k) / denom).astype(real), ((dt / mu) / denom).astype(real)


# ----------------------------------------------------------------------------------------------- spacings and CPML

def yee_inverse_spacings(widths):
    """(1/w, 1/hi-face spacing) of one axis, float64 (yee_grid.py:29-38)."""
    widths = np.asarray(widths, dtype=np.float64)
    face_spacing = 0.5 * (widths + np.roll(widths, -1))
    return 1.0 / widths, 1.0 / face_spacing


def cpml_side_rows(side, n, npml):
    """boundaries.py:570-576."""
    if side == 'lo':
        return slice(1, npml + 1), slice(0, npml)
    return slice(n - npml - 1, n - 1), slice(n - npml - 1, n - 1)


def cpml_axis_profile(faces, n, axis, npml, pml_dx, order=3, sigma_factor=1.0, kappa_max=15.0, alpha_max=0.0):
    """(sigma_e, kappa_e, alpha_e, sigma_h, kappa_h, alpha_h) float64 rows of one axis (boundaries.py:551-632)."""
    lo_active, hi_active = faces[f'{axis}_lo'] == 'cpml', faces[f'{axis}_hi'] == 'cpml'
    sigma_e, kappa_e, alpha_e = np.zeros(n), np.ones(n), np.zeros(n)
    sigma_h, kappa_h, alpha_h = np.zeros(n), np.ones(n), np.zeros(n)
    n_layers = int(lo_active) + int(hi_active)
    sigma_max = sigma_factor * (order + 1) / (150.0 * np.pi * float(pml_dx)) if n_layers else 0.0

    def graded(depth):
        return (sigma_max * depth ** order, 1.0 + (kappa_max - 1.0) * depth ** order, alpha_max * (1.0 - depth))

    if lo_active:
        e_rows, h_rows = cpml_side_rows('lo', n, npml)
        sigma_e[e_rows], kappa_e[e_rows], alpha_e[e_rows] = graded(np.arange(npml - 1, -1, -1, dtype=np.float64) / npml)
        sigma_h[h_rows], kappa_h[h_rows], alpha_h[h_rows] = graded((np.arange(npml, 0, -1, dtype=np.float64) - 0.5) / npml)
    if hi_active:
        e_rows, h_rows = cpml_side_rows('hi', n, npml)
        sigma_e[e_rows], kappa_e[e_rows], alpha_e[e_rows] = graded(np.arange(0, npml, dtype=np.float64) / npml)
        sigma_h[h_rows], kappa_h[h_rows], alpha_h[h_rows] = graded((np.arange(1, npml + 1, dtype=np.float64) - 0.5) / npml)
    return sigma_e, kappa_e, alpha_e, sigma_h, kappa_h, alpha_h


def cpml_recursion(sigma, kappa, alpha, dt, real):
    """(a, b) in `real` (boundaries.py:560-567; note a uses the already-rounded b)."""
    b = np.exp(-(sigma / kappa + alpha) * float(dt) / EPS0).astype(real)
    denom = sigma * kappa + kappa ** 2 * alpha
    a = np.divide(sigma * (b - 1.0), denom, out=np.zeros_like(denom), where=denom > 1e-30).astype(real)
    return a, b


@dataclass
class CPMLSide:
    name: str
    b_e: np.ndarray
    a_e: np.ndarray
    inv_e: np.ndarray
    b_h: np.ndarray
    a_h: np.ndarray
    inv_h: np.ndarray
    e_rows: slice
    h_rows: slice
    kappa_e: np.ndarray
    kappa_h: np.ndarray


def build_cpml(domain, real):
    """Per active side the recursion rows and the bulk curl spacings (CPMLSided.__init__, boundaries.py:694-730), plus
    the kappa-folded curl spacings of the Yee kernels (boundaries.py:778-799)."""
    dt = float(domain.dt)
    pml_dx = float(domain.grid_dx)
    n_axis = {'x': domain.nx, 'y': domain.ny}
    profiles = {axis: cpml_axis_profile(domain.faces, n_axis[axis], axis, domain.npml, pml_dx) for axis in 'xy'}
    bulk = {'x': yee_inverse_spacings(np.full(domain.nx, pml_dx)), 'y': yee_inverse_spacings(np.full(domain.ny, pml_dx))}
    sides = []
    for face in FACES:
        if domain.faces[face] != 'cpml':
            continue
        axis = face[0]
        e_rows, h_rows = cpml_side_rows(face[2:], n_axis[axis], domain.npml)
        se, ke, ae, sh, kh, ah = profiles[axis]
        a_e, b_e = cpml_recursion(se[e_rows], ke[e_rows], ae[e_rows], dt, real)
        a_h, b_h = cpml_recursion(sh[h_rows], kh[h_rows], ah[h_rows], dt, real)
        inv_e_bulk, inv_h_bulk = bulk[axis]
        sides.append(CPMLSide(face, b_e, a_e, inv_e_bulk[e_rows].astype(real), b_h, a_h,
                              inv_h_bulk[h_rows].astype(real), e_rows, h_rows,
                              ke[e_rows].astype(real), kh[h_rows].astype(real)))
    # Curl spacings: grid_cell_widths(grid) (float32 dx as float64), cast to real, kappa divided in per side.
    curl = {}
    for axis, n in (('x', domain.nx), ('y', domain.ny)):
        inv_e, inv_h = yee_inverse_spacings(domain.kernel_widths[0 if axis == 'x' else 1])
        for kind, values in (('e', inv_e), ('h', inv_h)):
            folded = np.array(values.astype(real), dtype=real, copy=True)
            for side in sides:
                if side.name[0] == axis:
                    rows, kappa = (side.e_rows, side.kappa_e) if kind == 'e' else (side.h_rows, side.kappa_h)
                    folded[rows] /= kappa
            curl[f'inv_d{axis}_{kind}'] = folded
    return sides, curl


# ----------------------------------------------------------------------------------------------- sources, monitors

class GaussianPulse:
    """open_sol/core/sources.py:23-53 (scalar math path of a Python float time)."""

    def __init__(self, f0, bandwidth=0.5, t0_factor=4.5):
        self.f0 = f0
        self.bandwidth = bandwidth
        self.tau = 1.0 / (bandwidth * f0 * np.pi)
        self.t0 = t0_factor * self.tau

    def __call__(self, t):
        delay = t - self.t0
        return math.exp(-(delay / self.tau) ** 2) * math.sin(2.0 * math.pi * self.f0 * delay)

    def spectral_limit(self):
        return self.f0 * (1.0 + 3.72 * self.bandwidth)


@dataclass
class LineSource:
    axis: str
    position: int
    lo: int
    hi: int
    temporal: GaussianPulse
    amplitude: np.float32
    profile: np.ndarray = None


@dataclass
class FluxMonitor:
    """physics/em/monitors.py:325-379 for polarization 'ez'."""
    normal_axis: str          # 'x' or 'y' (the monitor's own axis)
    position: int
    lo: int
    hi: int
    frequencies: np.ndarray
    dt: float
    widths: np.ndarray
    e_acc: np.ndarray = None
    h_acc: np.ndarray = None
    sample_interval: int = 1
    flux_sign: float = None   # None: the E_z sign (S_x = -E_z H_y, S_y = +E_z H_x)

    def flux(self):
        e = self.e_acc
        h = self.h_acc * np.exp(1j * np.pi * self.frequencies * self.dt)[:, None]
        sign = self.flux_sign if self.flux_sign is not None else (-1.0 if self.normal_axis == 'x' else 1.0)
        e_time_average = np.cos(np.pi * self.frequencies * self.dt)
        integrand = sign * e_time_average[:, None] * np.real(e * np.conj(h))
        return integrand @ self.widths


def sheet_admittance(line_eps, mu_r, sigma_m, omega, normal_spacing, dt):
    """physics/em/sources.py:430-436 with yee_grid.sheet_launch_factor (yee_grid.py:58-65)."""
    permeability = mu_r.astype(np.complex128) - 1j * sigma_m.astype(np.float64) / (omega * MU0)
    vacuum_half_phase = float(normal_spacing) * math.sin(0.5 * float(omega) * float(dt)) / (C0 * float(dt))
    launch = np.sqrt(1.0 - np.asarray(line_eps * permeability, dtype=np.complex128) * vacuum_half_phase ** 2)
    return np.abs(np.sqrt(line_eps / permeability) * launch).astype(DTYPE)


def dft_sample_interval(dt, sources, monitor_frequencies):
    """physics/em/monitors.py:177-191 (harmonic order 1)."""
    if not sources or not monitor_frequencies:
        return 1
    limits = [float(s.temporal.spectral_limit()) for s in sources]
    sample_rate = max(limits) + max(float(np.max(f)) for f in monitor_frequencies)
    return max(1, int(np.floor(1.0 / (sample_rate * float(dt)))))


def dft_phases(omega, t, dt_m):
    """complex64 phases as float32 (nf, 2) (monitors.py:22-24)."""
    phase = -omega * float(t)
    out = np.empty((omega.size, 2), dtype=np.float32)
    out[:, 0] = (np.cos(phase) * float(dt_m)).astype(np.float32)
    out[:, 1] = (np.sin(phase) * float(dt_m)).astype(np.float32)
    return out


# ----------------------------------------------------------------------------------------------- ctypes binding

def _real_ptr(real):
    return ctypes.POINTER(ctypes.c_float if real == np.float32 else ctypes.c_double)


def _make_structs(real):
    R = ctypes.c_float if real == np.float32 else ctypes.c_double
    P = ctypes.POINTER(R)

    class State(ctypes.Structure):
        _fields_ = [('nx', ctypes.c_int32), ('ny', ctypes.c_int32), ('periodic_x', ctypes.c_int32),
                    ('periodic_y', ctypes.c_int32), ('ez', P), ('hx', P), ('hy', P), ('ca', P), ('cb', P),
                    ('da', P), ('db', P), ('da_uniform', R), ('db_uniform', R), ('inv_dx_e', P), ('inv_dx_h', P),
                    ('inv_dy_e', P), ('inv_dy_h', P), ('npml', ctypes.c_int32), ('cpml_active', ctypes.c_int32 * 4),
                    ('b_e', P * 4), ('a_e', P * 4), ('inv_e', P * 4), ('b_h', P * 4), ('a_h', P * 4),
                    ('inv_h', P * 4), ('psi_e', P * 4), ('psi_h', P * 4)]

    class Line(ctypes.Structure):
        _fields_ = [('axis', ctypes.c_int32), ('position', ctypes.c_int32), ('lo', ctypes.c_int32),
                    ('hi', ctypes.c_int32), ('profile', ctypes.POINTER(ctypes.c_float)),
                    ('values', ctypes.POINTER(ctypes.c_float))]

    class Flux(ctypes.Structure):
        _fields_ = [('normal_axis', ctypes.c_int32), ('position', ctypes.c_int32), ('lo', ctypes.c_int32),
                    ('hi', ctypes.c_int32), ('nf', ctypes.c_int32), ('e_acc', ctypes.POINTER(ctypes.c_double)),
                    ('h_acc', ctypes.POINTER(ctypes.c_double)), ('phases', ctypes.POINTER(ctypes.c_float)),
                    ('first_sample', ctypes.c_int64), ('n_samples', ctypes.c_int64)]
    return State, Line, Flux


def _make_tfsf_struct(real):
    R = ctypes.c_float if real == np.float32 else ctypes.c_double
    P = ctypes.POINTER(R)

    class Tfsf(ctypes.Structure):
        _fields_ = [('x0', ctypes.c_int32), ('x1', ctypes.c_int32), ('y0', ctypes.c_int32), ('y1', ctypes.c_int32),
                    ('aux_x0', ctypes.c_int32), ('aux_n', ctypes.c_int32), ('source_index', ctypes.c_int32),
                    ('coef_h', R * 4), ('coef_e', R * 2), ('mur_lo', R), ('mur_hi', R), ('aux_ez', P), ('aux_hy', P),
                    ('aux_coef_h', P), ('aux_coef_e', P), ('values', ctypes.POINTER(ctypes.c_float))]
    return Tfsf


def _make_pole_struct(real):
    R = ctypes.c_float if real == np.float32 else ctypes.c_double
    P = ctypes.POINTER(R)

    class Pole(ctypes.Structure):
        _fields_ = [('kind', ctypes.c_int32), ('i0', ctypes.c_int32), ('i1', ctypes.c_int32), ('j0', ctypes.c_int32),
                    ('j1', ctypes.c_int32), ('damping', R), ('restoring', R), ('drive', P), ('a', P), ('b', P)]
    return Pole


_LIBS = {}


def load_library(real=np.float32):
    """The float32 / float64 build of oracle/ez2d.c (built by oracle/Makefile into oracle/_build)."""
    key = np.dtype(real).name
    if key not in _LIBS:
        name = 'libez2d_oracle_f32.so' if real == np.float32 else 'libez2d_oracle_f64.so'
        path = os.path.join(LIB_DIR, name)
        if not os.path.exists(path):
            raise RuntimeError(f'oracle library {path} is not built (run: make -C oracle)')
        lib = ctypes.CDLL(path)
        State, Line, Flux = _make_structs(real)
        P = ctypes.POINTER(ctypes.c_float if real == np.float32 else ctypes.c_double)
        R = ctypes.c_float if real == np.float32 else ctypes.c_double
        lib.oracle_ez2d_advance.restype = ctypes.c_int
        lib.oracle_ez2d_advance.argtypes = [ctypes.POINTER(State), ctypes.c_int64, ctypes.c_int64, ctypes.c_int32,
                                            ctypes.POINTER(Line), ctypes.c_int32, ctypes.POINTER(Flux),
                                            ctypes.c_int64]
        Tfsf = _make_tfsf_struct(real)
        lib.oracle_ez2d_advance_tfsf.restype = ctypes.c_int
        lib.oracle_ez2d_advance_tfsf.argtypes = [ctypes.POINTER(State), ctypes.c_int64, ctypes.c_int64,
                                                 ctypes.c_int32, ctypes.POINTER(Line), ctypes.c_int32,
                                                 ctypes.POINTER(Flux), ctypes.c_int64, ctypes.c_int32,
                                                 ctypes.POINTER(Tfsf)]
        lib.tfsf_struct = Tfsf
        Pole = _make_pole_struct(real)
        lib.oracle_ez2d_advance_full.restype = ctypes.c_int
        lib.oracle_ez2d_advance_full.argtypes = [ctypes.POINTER(State), ctypes.c_int64, ctypes.c_int64,
                                                 ctypes.c_int32, ctypes.POINTER(Line), ctypes.c_int32,
                                                 ctypes.POINTER(Flux), ctypes.c_int64, ctypes.c_int32,
                                                 ctypes.POINTER(Tfsf), ctypes.c_int32, ctypes.POINTER(Pole), P,
                                                 ctypes.c_int32 * 4, R]
        lib.pole_struct = Pole
        _LIBS[key] = (lib, State, Line, Flux)
    return _LIBS[key]


def _ptr(array, ctype):
    return array.ctypes.data_as(ctypes.POINTER(ctype)) if array is not None else None


# ----------------------------------------------------------------------------------------------- the oracle run

class TfsfBox:
    """A TFSF plane-wave box of OracleEz2D.add_tfsf: cells, incident line, coefficients, temporal."""


class OracleEz2D:
    """The whole 2D E_z path of one simulation on the CPU: geometry, sources and flux monitors as the reference's
    Simulation / EMPhysics methods take them, then ``run(duration=...)`` or ``run(n_steps=...)``."""

    def __init__(self, size_x, size_y, dx, npml=15, boundaries=None, courant=None, precision='single'):
        self.domain = Domain2D(size_x, size_y, dx, npml, boundaries or 'pml', courant)
        self.real = np.float32 if precision == 'single' else np.float64
        d = self.domain
        shape = (d.nx, d.ny)
        self.eps_r = np.full(shape, DTYPE(1.0), dtype=DTYPE)
        self.sigma_e = np.zeros(shape, dtype=DTYPE)
        self.mu_r = np.full(shape, DTYPE(1.0), dtype=DTYPE)
        self.sigma_m = np.zeros(shape, dtype=DTYPE)
        self.ez = np.zeros(shape, dtype=self.real)
        self.hx = np.zeros(shape, dtype=self.real)
        self.hy = np.zeros(shape, dtype=self.real)
        self.sources, self.monitors = [], []
        self.maps = []           # field-map DFT monitors (add_dft_monitor)
        self.tfsf = []           # TFSF plane-wave boxes (add_tfsf)
        self.poles = []          # [pole, (slice, slice) box, cropped bool mask, state arrays] (add order)
        self.probes = []         # field probes (add_field_probe): [ix, iy, component, times, values]
        self.n_step = 0
        self.time = 0.0          # engine clock (host float64 accumulation)
        self.runner_t = 0.0      # runner clock
        self.sample_interval = None
        self._finalized = False

    # -- geometry
    def add_dielectric_rectangle(self, x0, y0, x1, y1, eps_r, sigma_e=0.0):
        paint_rect(self.domain, self.eps_r, x0, y0, x1, y1, eps_r)
        if sigma_e is not None:
            paint_rect(self.domain, self.sigma_e, x0, y0, x1, y1, sigma_e)

    def add_dielectric_circle(self, cx, cy, radius, eps_r, sigma_e=0.0):
        paint_circle(self.domain, self.eps_r, cx, cy, radius, eps_r)
        if sigma_e is not None:
            paint_circle(self.domain, self.sigma_e, cx, cy, radius, sigma_e)

    # -- sources and monitors
    def add_line_source(self, axis, position, wavelength=None, frequency=None, bandwidth=0.5, amplitude=1.0,
                        span=None):
        """physics/em/__init__.py:442-473 with placement.sheet_line (span None: the whole grid line)."""
        d = self.domain
        f0 = frequency if frequency is not None else C0 / wavelength
        if axis == 'x':
            line_cell, along = d.pos_to_cell_y(position), d.pos_to_cell_x
            n_along = d.nx
        else:
            line_cell, along = d.pos_to_cell_x(position), d.pos_to_cell_y
            n_along = d.ny
        if span is None:
            lo, hi = 0, n_along
        else:
            start, end = sorted((float(span[0]), float(span[1])))
            lo, hi = along(start), along(end) + 1
            window = d.window[0 if axis == 'x' else 1]
            if lo == window.start and d.faces[f'{axis}_lo'] == 'cpml':
                lo = 0
            if hi == window.stop and d.faces[f'{axis}_hi'] == 'cpml':
                hi = n_along
        src = LineSource(axis, line_cell, lo, hi, GaussianPulse(f0, bandwidth), DTYPE(amplitude))
        src.normal_width = float(d.cell_widths[1 if axis == 'x' else 0][line_cell])
        self.sources.append(src)
        return src

    def add_flux_monitor(self, axis, position, span, wavelengths=None, frequencies=None):
        """physics/em/__init__.py:511-518, placement.flux_line_cells (placement.py:55-71)."""
        d = self.domain
        freqs = (np.atleast_1d(np.array(frequencies, dtype=np.float64)) if frequencies is not None
                 else C0 / np.atleast_1d(np.array(wavelengths, dtype=np.float64)))
        lo_c, hi_c = sorted((float(span[0]), float(span[1])))
        if axis == 'x':
            normal, line_cell, lo, hi, widths = 'y', d.pos_to_cell_y(position), d.pos_to_cell_x(lo_c), \
                d.pos_to_cell_x(hi_c) + 1, d.cell_widths[0]
        else:
            normal, line_cell, lo, hi, widths = 'x', d.pos_to_cell_x(position), d.pos_to_cell_y(lo_c), \
                d.pos_to_cell_y(hi_c) + 1, d.cell_widths[1]
        mon = FluxMonitor(normal, line_cell, lo, hi, freqs, float(d.dt), widths[lo:hi].copy())
        mon.e_acc = np.zeros((freqs.size, hi - lo), dtype=np.complex128)
        mon.h_acc = np.zeros((freqs.size, hi - lo), dtype=np.complex128)
        self.monitors.append(mon)
        return mon

    def add_dft_monitor(self, x0, y0, x1, y1, wavelengths=None, frequencies=None, downsample=1):
        """physics/em/__init__.py:500-509 with placement.box_cells (placement.py:97-105) and DFTMonitor
        (monitors.py:248-289, polarization 'ez'): the cell box of the physical box, sampled every `downsample`-th cell
        from the middle of the first block (dft_sample_slice, monitors.py:152-155); complex64 sums (nf, mx, my)."""
        d = self.domain
        freqs = (np.atleast_1d(np.array(frequencies, dtype=np.float64)) if frequencies is not None
                 else C0 / np.atleast_1d(np.array(wavelengths, dtype=np.float64)))
        x_lo, x_hi = sorted((x0, x1))
        y_lo, y_hi = sorted((y0, y1))
        ix0, ix1 = d.pos_to_cell_x(x_lo), d.pos_to_cell_x(x_hi) + 1
        iy0, iy1 = d.pos_to_cell_y(y_lo), d.pos_to_cell_y(y_hi) + 1
        ds = int(downsample)
        xs = slice(ix0 + min(ds, ix1 - ix0) // 2, ix1, ds)
        ys = slice(iy0 + min(ds, iy1 - iy0) // 2, iy1, ds)
        mon = FluxMonitor.__new__(FluxMonitor)   # a plain record: frequencies, dt, sample boxes, sums
        mon.frequencies, mon.dt, mon.x_samples, mon.y_samples, mon.downsample = freqs, float(d.dt), xs, ys, ds
        mon.ez_dft = np.zeros((freqs.size, len(range(xs.start, xs.stop, ds)), len(range(ys.start, ys.stop, ds))),
                              dtype=np.complex64)
        self.maps.append(mon)
        return mon

    def add_drude_rectangle(self, x0, y0, x1, y1, drude):
        """physics/em/__init__.py:329-340: the pole on the mask, eps_r = eps_inf under it."""
        self._add_pole(drude, rect_mask(self.domain, x0, y0, x1, y1), True)

    def add_drude_circle(self, cx, cy, radius, drude):
        self._add_pole(drude, circle_mask(self.domain, cx, cy, radius), True)

    def add_dispersive(self, pole, mask):
        self._add_pole(pole, np.asarray(mask, dtype=bool), False)

    def _add_pole(self, pole, mask, set_background):
        """fdtd_ez_2d.py:123-163 with _bounding_box (fdtd_2d_base.py:29-36): the pole on the bounding box of its
        mask, drive = mask x drive there."""
        rows = np.flatnonzero(mask.any(axis=1))
        if rows.size:
            cols = np.flatnonzero(mask.any(axis=0))
            box = (slice(int(rows[0]), int(rows[-1]) + 1), slice(int(cols[0]), int(cols[-1]) + 1))
            self.poles.append([pole, box, mask[box].copy()])
        if set_background:
            self.eps_r[mask] = DTYPE(pole.eps_inf)

    def add_tfsf(self, x0, y0, x1, y1, wavelength=None, frequency=None, bandwidth=0.5, amplitude=1.0,
                 waveform='gaussian'):
        """physics/em/__init__.py:475-490 with placement.tfsf_box_cells (placement.py:108-128) and the +x plane-wave box
        of physics/em/sources.py:206-332 (_PlaneWaveBox, TFSFSource): 20 margin cells at the widths of cells x0 - 1 /
        x1 around the box columns, soft source at aux cell 10 scaled by 2 S cos(kappa0/2) amplitude, Mur ends at the
        numerical phase velocity of the carrier, side coefficients dt / (mu0 or eps0 x spacing) in float32."""
        if waveform != 'gaussian':
            raise ValueError('the oracle restates the Gaussian waveform only')
        d = self.domain
        f0 = float(frequency) if frequency is not None else C0 / float(wavelength)
        x_lo, x_hi = sorted((x0, x1))
        y_lo, y_hi = sorted((y0, y1))
        ix0, ix1 = d.pos_to_cell_x(x_lo), d.pos_to_cell_x(x_hi) + 1
        iy0, iy1 = d.pos_to_cell_y(y_lo), d.pos_to_cell_y(y_hi) + 1
        dt = float(d.dt)
        dx_cells = np.full(d.nx, float(DTYPE(d.dx)))
        dy_cells = np.full(d.ny, float(DTYPE(d.dx)))
        margin, source_index = 20, 10
        up, down = float(dx_cells[ix0 - 1]), float(dx_cells[ix1])
        widths = np.concatenate((np.full(margin, up), dx_cells[ix0:ix1], np.full(margin, down)))
        face_spacings = 0.5 * (widths[:-1] + widths[1:])
        half = 0.5 * (2.0 * np.pi * float(f0)) * dt

        def line_terms(width):   # _aux_line_terms (sources.py:191-204)
            courant = C0 * dt / width
            sin_half_kappa = math.sin(half) / courant
            cos_half_kappa = math.sqrt(1.0 - sin_half_kappa ** 2)
            mur_courant = courant * cos_half_kappa / math.cos(half)
            return courant, cos_half_kappa, (mur_courant - 1.0) / (mur_courant + 1.0)

        courant, cos_half_kappa, mur_lo = line_terms(up)
        _, _, mur_hi = line_terms(down)
        spacings = [0.5 * float(w[i] + w[i + 1]) for w, i in ((dx_cells, ix0 - 1), (dx_cells, ix1 - 1),
                                                              (dy_cells, iy0 - 1), (dy_cells, iy1 - 1))]
        box = TfsfBox()
        box.__dict__.update({'cells': (ix0, ix1, iy0, iy1), 'aux_x0': margin, 'source_index': source_index,
               'temporal': GaussianPulse(f0, bandwidth), 'scale': 2.0 * courant * cos_half_kappa * float(amplitude),
               'coef_h': [DTYPE(dt / (MU0 * sp)) for sp in spacings],
               'coef_e': [DTYPE(dt / (EPS0 * float(dx_cells[ix0]))), DTYPE(dt / (EPS0 * float(dx_cells[ix1 - 1])))],
               'mur': (DTYPE(mur_lo), DTYPE(mur_hi)),
               'aux_coef_h': np.asarray(dt / (MU0 * face_spacings), dtype=DTYPE),
               'aux_coef_e': np.asarray(dt / (EPS0 * widths), dtype=DTYPE),
               'aux_ez': np.zeros(widths.size, dtype=DTYPE), 'aux_hy': np.zeros(widths.size, dtype=DTYPE),
               'widths': widths, 'face_spacings': face_spacings, 'spacings': spacings,
               'side_widths_x': (float(dx_cells[ix0]), float(dx_cells[ix1 - 1])), 'dt': dt})
        self.tfsf.append(box)
        return box

    def add_field_probe(self, x, y, field_component=None):
        """physics/em/__init__.py:492-498 with placement.probe_cell (placement.py:29-45) and FieldProbe.record at
        t_full after every step (core/monitors.py:226-236, fdtd_2d_base.py:481-487): (times, values) lists."""
        d = self.domain
        component = field_component or 'ez'
        probe = [d.pos_to_cell_x(x), d.pos_to_cell_y(y), component, [], []]
        self.probes.append(probe)
        return probe

    def _record_probes(self):
        for ix, iy, component, times, values in self.probes:
            times.append(self.time)
            values.append(np.float32(getattr(self, component)[ix, iy]))

    def _fold_maps(self):
        """DFTMonitor.update at a sample step (monitors.py:281-311) with _dft_accum_host (:36-37): the complex64
        phase exp(-j omega t) m dt at the engine clock, then acc += phase * E_z[box] in numpy complex64."""
        m = self.sample_interval
        for mon in self.maps:
            table = dft_phases(2.0 * np.pi * mon.frequencies, self.time, mon.dt * m)
            ph = (table[:, 0] + 1j * table[:, 1]).astype(np.complex64)
            f = np.asarray(self.ez[mon.x_samples, mon.y_samples], dtype=np.float32)
            mon.ez_dft += ph[:, None, None] * f[None, :, :]

    # -- finalize: coefficients, CPML, calibration, sample interval
    def finalize(self):
        d, real = self.domain, self.real
        self.ca, self.cb = e_coefficients(self.sigma_e, self.eps_r, d.dt, real)
        self.da, self.db = h_coefficients(self.sigma_m, self.mu_r, d.dt, real)
        self.cpml_sides, self.curl = build_cpml(d, real)
        for src in self.sources:
            if src.axis == 'x':
                line = (slice(src.lo, src.hi), src.position)
            else:
                line = (src.position, slice(src.lo, src.hi))
            omega = 2.0 * np.pi * float(src.temporal.f0)
            line_eps = (np.asarray(self.eps_r[line], dtype=np.complex128)
                        - 1j * np.asarray(self.sigma_e[line], dtype=np.float64) / (omega * EPS0))
            # the susceptibility of every pole region the line crosses (sources.py:401-427)
            for pole, box, cropped in self.poles:
                chi = pole.susceptibility(omega)
                along_box, normal_box = (box[0], box[1]) if src.axis == 'x' else (box[1], box[0])
                start, stop = max(src.lo, along_box.start), min(src.hi, along_box.stop)
                if not (normal_box.start <= src.position < normal_box.stop and start < stop):
                    continue
                along = slice(start - along_box.start, stop - along_box.start)
                normal = src.position - normal_box.start
                mask_line = cropped[along, normal] if src.axis == 'x' else cropped[normal, along]
                line_eps[start - src.lo:stop - src.lo] += chi * mask_line
            admittance = sheet_admittance(line_eps, self.mu_r[line], self.sigma_m[line], omega, src.normal_width,
                                          float(d.dt))
            weight = np.asarray(2.0 * np.ones(src.hi - src.lo) / (float(ETA0) * src.normal_width), dtype=DTYPE)
            src.profile = (self.cb[line] * admittance * weight).astype(DTYPE)
        self.sample_interval = dft_sample_interval(float(d.dt), self.sources + self.tfsf,
                                                   [m.frequencies for m in self.monitors + self.maps])
        for m in self.monitors + self.maps:
            m.sample_interval = self.sample_interval
        self.psi_e = {s.name: np.zeros(self._psi_shape(s.name), dtype=real) for s in self.cpml_sides}
        self.psi_h = {s.name: np.zeros(self._psi_shape(s.name), dtype=real) for s in self.cpml_sides}
        self._finalized = True

    def _psi_shape(self, face):
        d = self.domain
        return (d.npml, d.ny) if face[0] == 'x' else (d.nx, d.npml)

    # -- stepping
    def steps_for_duration(self, duration):
        """Ticks MultiphysicsRunner.advance runs until t >= t_end - dt/2 (runner.py:182,191-203)."""
        dt = float(self.domain.dt)
        t_end = self.runner_t + float(duration)
        stop = t_end - 0.5 * dt
        t, n = self.runner_t, 0
        while t < stop:
            t = t + dt
            n += 1
        return n

    def run(self, duration=None, n_steps=None):
        if not self._finalized:
            self.finalize()
        if n_steps is None:
            n_steps = self.steps_for_duration(duration)
        self.advance(n_steps)

    def source_values(self, n_steps):
        """Per line source, float32 amplitude * temporal(t + dt/2) of the next n_steps steps, and the engine clock
        after them (fdtd_ez_2d.py:76-79,96-102; core/sources.py:221-229)."""
        dt = float(self.domain.dt)
        values = [np.empty(n_steps, dtype=np.float32) for _ in self.sources]
        t = self.time
        times_full = np.empty(n_steps)
        for k in range(n_steps):
            t_half = t + 0.5 * dt
            for src, v in zip(self.sources, values):
                v[k] = DTYPE(src.amplitude * src.temporal(t_half))
            t = t + dt
            times_full[k] = t
        return values, times_full

    def _chunk_phase_tables(self, n_steps, times_full):
        """(first sample, sample count, per-monitor float32 (n_q, nf, 2) phase tables) of the DFT samples the next
        n_steps steps take (monitors.py:22-24,219-220)."""
        m = self.sample_interval
        first_q = self.n_step // m + 1
        last_q = (self.n_step + n_steps) // m
        n_q = max(0, last_q - first_q + 1)
        phase_tables = []
        for mon in self.monitors:
            omega = 2.0 * np.pi * mon.frequencies
            table = np.empty((max(n_q, 1), mon.frequencies.size, 2), dtype=np.float32)
            for qi in range(n_q):
                step = (first_q + qi) * m
                table[qi] = dft_phases(omega, times_full[step - self.n_step - 1], mon.dt * m)
            phase_tables.append(table)
        return first_q, n_q, phase_tables

    def _cpml_state(self, st, R):
        """Fill the CPML members of a ctypes state; returns the arrays the pointers refer to."""
        st.npml = self.domain.npml
        keep = []
        for side in self.cpml_sides:
            k = FACES.index(side.name)
            st.cpml_active[k] = 1
            for attr in ('b_e', 'a_e', 'inv_e', 'b_h', 'a_h', 'inv_h'):
                arr = np.ascontiguousarray(getattr(side, attr), dtype=self.real)
                keep.append(arr)
                getattr(st, attr)[k] = _ptr(arr, R)
            st.psi_e[k] = _ptr(self.psi_e[side.name], R)
            st.psi_h[k] = _ptr(self.psi_h[side.name], R)
        return keep

    def _line_structs(self, Line, values):
        lines = (Line * max(1, len(self.sources)))()
        for i, (src, v) in enumerate(zip(self.sources, values)):
            lines[i].axis, lines[i].position = (0 if src.axis == 'x' else 1), src.position
            lines[i].lo, lines[i].hi = src.lo, src.hi
            lines[i].profile = _ptr(src.profile, ctypes.c_float)
            lines[i].values = _ptr(v, ctypes.c_float)
        return lines

    def _flux_structs(self, Flux, phase_tables, first_q, n_q):
        fluxes = (Flux * max(1, len(self.monitors)))()
        for i, (mon, table) in enumerate(zip(self.monitors, phase_tables)):
            fluxes[i].normal_axis = 0 if mon.normal_axis == 'x' else 1
            fluxes[i].position, fluxes[i].lo, fluxes[i].hi = mon.position, mon.lo, mon.hi
            fluxes[i].nf = mon.frequencies.size
            fluxes[i].e_acc = mon.e_acc.ctypes.data_as(ctypes.POINTER(ctypes.c_double))
            fluxes[i].h_acc = mon.h_acc.ctypes.data_as(ctypes.POINTER(ctypes.c_double))
            fluxes[i].phases = _ptr(table, ctypes.c_float)
            fluxes[i].first_sample, fluxes[i].n_samples = first_q, n_q
        return fluxes

    def _pole_structs(self, Pole, R):
        """ctypes records of the poles (states kept across chunks), the Drude total, its union box, float32 1 / dt."""
        dt = float(self.domain.dt)
        records = (Pole * max(1, len(self.poles)))()
        union = None
        for q, entry in enumerate(self.poles):
            pole, box, cropped = entry[:3]
            if len(entry) == 3:   # first chunk: drive and zero states
                damping, restoring, drive = pole.coefficients(dt)
                shape = cropped.shape
                entry.extend([cropped.astype(DTYPE) * drive, np.zeros(shape, DTYPE), np.zeros(shape, DTYPE),
                              damping, restoring])
            drive_box, a, b, damping, restoring = entry[3:]
            kind = 0 if isinstance(pole, OracleDrude) else 1
            rec = records[q]
            rec.kind, rec.damping, rec.restoring = kind, float(damping), float(restoring)
            rec.i0, rec.i1, rec.j0, rec.j1 = box[0].start, box[0].stop, box[1].start, box[1].stop
            rec.drive, rec.a, rec.b = _ptr(drive_box, R), _ptr(a, R), _ptr(b, R)
            if kind == 0:
                union = (box if union is None else (slice(min(union[0].start, box[0].start),
                                                          max(union[0].stop, box[0].stop)),
                                                    slice(min(union[1].start, box[1].start),
                                                          max(union[1].stop, box[1].stop))))
        if getattr(self, 'jz_total', None) is None:
            self.jz_total = np.zeros((self.domain.nx, self.domain.ny), dtype=DTYPE)
        box4 = (ctypes.c_int32 * 4)(*((union[0].start, union[0].stop, union[1].start, union[1].stop) if union
                                      else (0, 0, 0, 0)))
        return records, self.jz_total, box4, float(DTYPE(1.0 / dt))

    def _tfsf_structs(self, Tfsf, R, n_steps):
        """ctypes records of the TFSF boxes with this chunk's soft-source values FP32(scale * temporal(t + dt/2))."""
        boxes = (Tfsf * max(1, len(self.tfsf)))()
        dt = float(self.domain.dt)
        for b, box in enumerate(self.tfsf):
            t, values = self.time, np.empty(n_steps, dtype=np.float32)
            for k in range(n_steps):
                values[k] = DTYPE(box.scale * box.temporal(t + 0.5 * dt))
                t = t + dt
            box.values = values   # kept alive for the call
            rec = boxes[b]
            rec.x0, rec.x1, rec.y0, rec.y1 = box.cells
            rec.aux_x0, rec.aux_n, rec.source_index = box.aux_x0, box.aux_ez.size, box.source_index
            for i in range(4):
                rec.coef_h[i] = float(box.coef_h[i])
            rec.coef_e[0], rec.coef_e[1] = float(box.coef_e[0]), float(box.coef_e[1])
            rec.mur_lo, rec.mur_hi = float(box.mur[0]), float(box.mur[1])
            rec.aux_ez, rec.aux_hy = _ptr(box.aux_ez, R), _ptr(box.aux_hy, R)
            rec.aux_coef_h, rec.aux_coef_e = _ptr(box.aux_coef_h, R), _ptr(box.aux_coef_e, R)
            rec.values = _ptr(values, ctypes.c_float)
        return boxes

    def _clock_after(self, n_steps, times_full):
        self.n_step += n_steps
        if n_steps:
            self.time = float(times_full[-1])
        dt = float(self.domain.dt)
        for _ in range(n_steps):
            self.runner_t = self.runner_t + dt

    def advance(self, n_steps):
        """n_steps steps; with field maps, in pieces that end on the DFT sample steps, each followed by the maps'
        update (the reference updates its monitors after every sampled step)."""
        if not self.maps and not self.probes:
            self._advance_chunk(n_steps)
            return
        m = self.sample_interval
        while n_steps > 0:
            piece = 1 if self.probes else min(n_steps, m - self.n_step % m)
            self._advance_chunk(piece)
            n_steps -= piece
            if self.maps and self.n_step % m == 0:
                self._fold_maps()
            self._record_probes()

    def _advance_chunk(self, n_steps):
        lib, State, Line, Flux = load_library(self.real)
        d, real = self.domain, self.real
        R = ctypes.c_float if real == np.float32 else ctypes.c_double
        values, times_full = self.source_values(n_steps)
        first_q, n_q, phase_tables = self._chunk_phase_tables(n_steps, times_full)
        st = State()
        st.nx, st.ny, st.periodic_x, st.periodic_y = d.nx, d.ny, int(d.periodic_x), int(d.periodic_y)
        st.ez, st.hx, st.hy = _ptr(self.ez, R), _ptr(self.hx, R), _ptr(self.hy, R)
        ca_unit = bool(np.all(self.ca == 1))
        st.ca = None if ca_unit else _ptr(self.ca, R)
        st.cb = _ptr(self.cb, R)
        st.da, st.db = _ptr(self.da, R), _ptr(self.db, R)
        st.da_uniform, st.db_uniform = 1.0, 0.0
        for name in ('inv_dx_e', 'inv_dx_h', 'inv_dy_e', 'inv_dy_h'):
            setattr(st, name, _ptr(self.curl[name], R))
        keep = self._cpml_state(st, R)
        lines = self._line_structs(Line, values)
        fluxes = self._flux_structs(Flux, phase_tables, first_q, n_q)
        boxes = self._tfsf_structs(lib.tfsf_struct, R, n_steps)
        poles, jz_total, drude_box, inv_dt = self._pole_structs(lib.pole_struct, R)
        rc = lib.oracle_ez2d_advance_full(ctypes.byref(st), self.n_step, n_steps, len(self.sources), lines,
                                          len(self.monitors), fluxes, self.sample_interval, len(self.tfsf), boxes,
                                          len(self.poles), poles, _ptr(jz_total, R), drude_box, inv_dt)
        del keep
        if rc != 0:
            raise RuntimeError('oracle phase table does not cover a sample')
        self._clock_after(n_steps, times_full)
