"""Boundary types of the 2D / 3D FDTD engines and the CPML rows they upload.

BCType / BoundaryConfig keep open_sol's names, presets and validation messages (open_sol/physics/em/boundaries.py:42-
356).  The CPML grading (sigma, kappa, alpha per row), the psi recursion (a, b) and the kappa fold into the curl
spacings are computed on the host in float64 and rounded once to the field type, exactly as open_sol does
(boundaries.py:541-632, 671-686, 774-799), and handed to the device engine as per-side rows.
"""
from __future__ import annotations

import math
from dataclasses import dataclass
from enum import Enum

import numpy as np

from .constants import DTYPE, EPS0, FACES, FACES_3D


class BCType(Enum):
    CPML = 'cpml'
    PEC = 'pec'
    PMC = 'pmc'
    PERIODIC = 'periodic'
    BLOCH = 'bloch'
    SYMMETRIC = 'symmetric'
    ANTISYMMETRIC = 'antisymmetric'


MIRROR_TYPES = frozenset({BCType.SYMMETRIC, BCType.ANTISYMMETRIC})
MIRROR_GHOST_CELLS = 1
# Face types the B200 engines step: CPML and periodic (k = 0).  The wall / mirror rows and Bloch k != 0 are not built.
SUPPORTED_TYPES = frozenset({BCType.CPML, BCType.PERIODIC, BCType.BLOCH})


def _face_property(face):
    stored_name = '_' + face

    def get_face(self):
        return getattr(self, stored_name)

    def set_face(self, value):
        try:
            bc_type = BCType(value.value if isinstance(value, BCType) else value)
        except ValueError:
            raise ValueError(f"{face} must be one of {[t.value for t in BCType]}, got {value!r}") from None
        setattr(self, stored_name, bc_type)

    return property(get_face, set_face)


class BoundaryConfig:
    """Per-face boundary types plus CPML settings (boundaries.py:194-356); z faces exist for 3D domains."""
    x_lo = _face_property('x_lo')
    x_hi = _face_property('x_hi')
    y_lo = _face_property('y_lo')
    y_hi = _face_property('y_hi')
    z_lo = _face_property('z_lo')
    z_hi = _face_property('z_hi')

    def __init__(self, x_lo='cpml', x_hi='cpml', y_lo='cpml', y_hi='cpml', z_lo=None, z_hi=None):
        self.x_lo = x_lo
        self.x_hi = x_hi
        self.y_lo = y_lo
        self.y_hi = y_hi
        self.dimensions = 2 if z_lo is None and z_hi is None else 3
        if self.dimensions == 3:
            self.z_lo = z_lo or 'cpml'
            self.z_hi = z_hi or 'cpml'
        self.cpml_npml: int = 15
        self.cpml_order: int = 3
        self.cpml_sigma_factor: float = 1.0
        self.cpml_kappa_max: float = 15.0
        self.cpml_alpha_max: float = 0.0
        self.bloch_kx: float = 0.0
        self.bloch_ky: float = 0.0
        self._validate()

    @property
    def faces(self):
        return FACES if self.dimensions == 2 else FACES_3D

    def _validate(self):
        if not (math.isfinite(self.bloch_kx) and math.isfinite(self.bloch_ky)):
            raise ValueError(f"bloch_kx / bloch_ky must be finite [rad/m], got {self.bloch_kx!r}, {self.bloch_ky!r}")
        periodic_types = {BCType.PERIODIC, BCType.BLOCH}
        axes = [('x', self.x_lo, self.x_hi), ('y', self.y_lo, self.y_hi)]
        if self.dimensions == 3:
            axes.append(('z', self.z_lo, self.z_hi))
        for axis_name, lo, hi in axes:
            if (lo in periodic_types or hi in periodic_types) and lo != hi:
                raise ValueError(f"{axis_name}: periodic/bloch BCs must be paired. Got {lo.value}/{hi.value}")
        if self.needs_cpml:
            if int(self.cpml_npml) != self.cpml_npml or self.cpml_npml < 1:
                raise ValueError(f"cpml_npml must be an integer >= 1 with a cpml face, got {self.cpml_npml!r}")
            if int(self.cpml_order) != self.cpml_order or self.cpml_order < 1:
                raise ValueError(f"cpml_order must be an integer >= 1, got {self.cpml_order!r}")
            if not self.cpml_sigma_factor > 0.0:
                raise ValueError(f"cpml_sigma_factor must be > 0, got {self.cpml_sigma_factor!r}")
            if not self.cpml_kappa_max >= 1.0:
                raise ValueError(f"cpml_kappa_max must be >= 1, got {self.cpml_kappa_max!r}")
            if not self.cpml_alpha_max >= 0.0:
                raise ValueError(f"cpml_alpha_max must be >= 0 S/m, got {self.cpml_alpha_max!r}")

    def require_supported(self, engine_label):
        """NotImplementedError for a face type the B200 engines do not step (walls, mirrors, Bloch k != 0)."""
        for face in self.faces:
            kind = getattr(self, face)
            if kind not in SUPPORTED_TYPES:
                raise NotImplementedError(f"{engine_label}: the B200 engine steps cpml and periodic faces; {face} is "
                                          f"{kind.value}")
        if self.has_bloch_phase:
            raise NotImplementedError(f"{engine_label}: Bloch k != 0 (a complex field set) is not built")

    @property
    def needs_cpml(self) -> bool:
        return any(getattr(self, face) == BCType.CPML for face in self.faces)

    @property
    def cpml_sides(self):
        return {face: getattr(self, face) == BCType.CPML for face in self.faces}

    def _periodic(self, face):
        return getattr(self, face) in (BCType.PERIODIC, BCType.BLOCH)

    @property
    def periodic_x(self) -> bool:
        return self._periodic('x_lo')

    @property
    def periodic_y(self) -> bool:
        return self._periodic('y_lo')

    @property
    def periodic_z(self) -> bool:
        return self.dimensions == 3 and self._periodic('z_lo')

    @property
    def has_bloch_phase(self) -> bool:
        return ((self.x_lo == BCType.BLOCH and self.bloch_kx != 0.0)
                or (self.y_lo == BCType.BLOCH and self.bloch_ky != 0.0))

    @property
    def npml_sides(self):
        return {face: (self.cpml_npml if getattr(self, face) == BCType.CPML
                       else MIRROR_GHOST_CELLS if getattr(self, face) in MIRROR_TYPES else 0) for face in self.faces}

    @classmethod
    def all_pml(cls, npml: int = 15):
        bc = cls('cpml', 'cpml', 'cpml', 'cpml')
        bc.cpml_npml = npml
        return bc

    @classmethod
    def all_pec(cls):
        return cls('pec', 'pec', 'pec', 'pec')

    @classmethod
    def all_pmc(cls):
        return cls('pmc', 'pmc', 'pmc', 'pmc')

    @classmethod
    def with_periodic_x(cls, npml_y: int = 15):
        bc = cls('periodic', 'periodic', 'cpml', 'cpml')
        bc.cpml_npml = npml_y
        return bc

    @classmethod
    def with_periodic_y(cls, npml_x: int = 15):
        bc = cls('cpml', 'cpml', 'periodic', 'periodic')
        bc.cpml_npml = npml_x
        return bc

    @classmethod
    def periodic_xy(cls):
        return cls('periodic', 'periodic', 'periodic', 'periodic')

    @classmethod
    def all_pml_3d(cls, npml: int = 12):
        bc = cls('cpml', 'cpml', 'cpml', 'cpml', 'cpml', 'cpml')
        bc.cpml_npml = npml
        return bc

    def __repr__(self):
        faces = ', '.join(f"{face}='{getattr(self, face).value}'" for face in self.faces)
        return f"BoundaryConfig({faces})"


def resolve_boundary(boundaries, npml):
    """Simulation's boundary presets (open_sol/simulation.py:388-399)."""
    if boundaries is None:
        return BoundaryConfig.all_pml(npml)
    if isinstance(boundaries, str):
        presets = {'pml': BoundaryConfig.all_pml(npml), 'pec': BoundaryConfig.all_pec(),
                   'pmc': BoundaryConfig.all_pmc(), 'periodic_x': BoundaryConfig.with_periodic_x(npml),
                   'periodic_y': BoundaryConfig.with_periodic_y(npml), 'periodic': BoundaryConfig.periodic_xy()}
        bc = presets.get(boundaries)
        if bc is None:
            raise ValueError(f"Unknown boundary preset: '{boundaries}'. Options: {list(presets.keys())}")
        return bc
    return boundaries


# ---- CPML rows ------------------------------------------------------------------------------------------------
# Along an axis of n cells (npml cells per layer): lo E rows 1..npml at depths (npml-1 .. 0)/npml, lo H rows
# 0..npml-1 at (npml-1/2 .. 1/2)/npml, hi E and H rows n-npml-1..n-2 at (0 .. npml-1)/npml and (1/2 .. npml-1/2)/npml.

def cpml_side_rows(side: str, n_cells: int, npml: int):
    """(E rows, H rows) of one side 'lo' / 'hi' (boundaries.py:570-576)."""
    n, npml = int(n_cells), int(npml)
    if side == 'lo':
        return slice(1, npml + 1), slice(0, npml)
    return slice(n - npml - 1, n - 1), slice(n - npml - 1, n - 1)


def cpml_sigma_max(config, pml_dx):
    return config.cpml_sigma_factor * (config.cpml_order + 1) / (150.0 * np.pi * float(pml_dx))


def cpml_axis_profiles(config, n_cells, axis, pml_dx):
    """float64 (sigma_e, kappa_e, alpha_e, sigma_h, kappa_h, alpha_h) rows of one axis (boundaries.py:551-632)."""
    sides = config.cpml_sides
    lo_active, hi_active = sides[f'{axis}_lo'], sides[f'{axis}_hi']
    npml, n = int(config.cpml_npml), int(n_cells)
    n_layers = int(lo_active) + int(hi_active)
    if n_layers and n < n_layers * npml + 2:
        raise ValueError(f"{axis} axis: {n} cells cannot hold {n_layers} CPML layer(s) of {npml} cells plus the 2 "
                         f"unstretched rows; it needs at least {n_layers * npml + 2} cells")
    sigma_e, kappa_e, alpha_e = np.zeros(n), np.ones(n), np.zeros(n)
    sigma_h, kappa_h, alpha_h = np.zeros(n), np.ones(n), np.zeros(n)
    sigma_max = cpml_sigma_max(config, pml_dx) if n_layers else 0.0
    order, kappa_max, alpha_max = config.cpml_order, config.cpml_kappa_max, config.cpml_alpha_max

    def graded(depth):
        return (sigma_max * depth ** order, 1.0 + (kappa_max - 1.0) * depth ** order, alpha_max * (1.0 - depth))

    if lo_active:
        e_rows, h_rows = cpml_side_rows('lo', n, npml)
        sigma_e[e_rows], kappa_e[e_rows], alpha_e[e_rows] = graded(np.arange(npml - 1, -1, -1, dtype=np.float64) / npml)
        sigma_h[h_rows], kappa_h[h_rows], alpha_h[h_rows] = graded(
            (np.arange(npml, 0, -1, dtype=np.float64) - 0.5) / npml)
    if hi_active:
        e_rows, h_rows = cpml_side_rows('hi', n, npml)
        sigma_e[e_rows], kappa_e[e_rows], alpha_e[e_rows] = graded(np.arange(0, npml, dtype=np.float64) / npml)
        sigma_h[h_rows], kappa_h[h_rows], alpha_h[h_rows] = graded(
            (np.arange(1, npml + 1, dtype=np.float64) - 0.5) / npml)
    return sigma_e, kappa_e, alpha_e, sigma_h, kappa_h, alpha_h


def cpml_recursion(sigma, kappa, alpha, dt, dtype=np.float32):
    """(a, b) rows in `dtype`: b = exp(-(sigma/kappa + alpha) dt / eps0), a = sigma (b - 1) / (sigma kappa + kappa^2
    alpha) with b already rounded to `dtype` (boundaries.py:560-567)."""
    b = np.exp(-(sigma / kappa + alpha) * float(dt) / EPS0).astype(dtype)
    denom = sigma * kappa + kappa ** 2 * alpha
    a = np.divide(sigma * (b - 1.0), denom, out=np.zeros_like(denom), where=denom > 1e-30).astype(dtype)
    return a, b


def inverse_spacings(widths):
    """float64 (1/w_i, 1/mean(w_i, w_(i+1) mod n)) of one axis (physics/em/yee_grid.py:29-38)."""
    widths = np.asarray(widths, dtype=np.float64)
    if widths.ndim != 1 or widths.size == 0:
        raise ValueError(f"cell widths must be a non-empty 1D array, got shape {widths.shape}")
    face_spacing = 0.5 * (widths + np.roll(widths, -1))
    return 1.0 / widths, 1.0 / face_spacing


def face_shares(widths, periodic):
    """float32 (lower, upper) hi-face weights w_k / (w_k + w_k+1), w_k+1 / (w_k + w_k+1); the last partner is the
    first cell (periodic) or the cell itself (yee_grid.py:76-84,119-125)."""
    widths = np.asarray(widths, dtype=np.float64)
    partner = np.roll(widths, -1) if periodic else np.concatenate((widths[1:], widths[-1:]))
    return (widths / (widths + partner)).astype(DTYPE), (partner / (widths + partner)).astype(DTYPE)


@dataclass(frozen=True)
class CPMLSideRows:
    """float32 rows of one active side: recursion b / a and bulk curl spacing of its E (cell-centre) and H (hi-face)
    rows, plus the kappa rows folded into the curl spacings."""
    face: str
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


@dataclass(frozen=True)
class YeeRows:
    """What an engine uploads for its boundaries: kappa-folded curl spacings per axis (inv_d<axis>_e / _h) and the
    rows of every active CPML side (FACES order)."""
    curl: dict
    sides: tuple


def build_yee_rows(config, shape, pml_dx, kernel_dx, dt, dtype=np.float32):
    """Curl spacings and CPML rows of a uniform grid `shape` (2 or 3 axes): the per-side rows of CPMLSided
    (boundaries.py:694-730) / cpml_slabs and the kappa fold of _curl_spacings (fdtd_2d_base.py:76-84)."""
    axes = 'xyz'[:len(shape)]
    pml_dx = float(pml_dx)
    profiles = {axis: cpml_axis_profiles(config, n, axis, pml_dx) for axis, n in zip(axes, shape)}
    sides = []
    faces = tuple(f'{axis}_{side}' for axis in axes for side in ('lo', 'hi'))
    for face in faces:
        if not config.cpml_sides[face]:
            continue
        axis = face[0]
        n = shape[axes.index(axis)]
        e_rows, h_rows = cpml_side_rows(face[2:], n, config.cpml_npml)
        se, ke, ae, sh, kh, ah = profiles[axis]
        a_e, b_e = cpml_recursion(se[e_rows], ke[e_rows], ae[e_rows], dt, dtype)
        a_h, b_h = cpml_recursion(sh[h_rows], kh[h_rows], ah[h_rows], dt, dtype)
        bulk_e, bulk_h = inverse_spacings(np.full(n, pml_dx))
        sides.append(CPMLSideRows(face, b_e, a_e, bulk_e[e_rows].astype(dtype), b_h, a_h,
                                  bulk_h[h_rows].astype(dtype), e_rows, h_rows, ke[e_rows].astype(dtype),
                                  kh[h_rows].astype(dtype)))
    curl = {}
    for axis, n in zip(axes, shape):
        inv_e, inv_h = inverse_spacings(np.full(n, float(kernel_dx)))
        for kind, values in (('e', inv_e), ('h', inv_h)):
            folded = np.array(values.astype(dtype), dtype=dtype, copy=True)
            for side in sides:
                if side.face[0] == axis:
                    rows, kappa = (side.e_rows, side.kappa_e) if kind == 'e' else (side.h_rows, side.kappa_h)
                    folded[rows] /= kappa
            curl[f'inv_d{axis}_{kind}'] = folded
    return YeeRows(curl=curl, sides=tuple(sides))
