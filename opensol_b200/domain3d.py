"""Uniform 3D domain of the B200 engine: cubic cells, CPML padded outside the physical window on every cpml face, the
float32 material arrays, and the 3D boundary configuration.

Geometry follows open_sol (open_sol/core/domain3d.py:12-140, core/grid3d.py:8-68): totals = window + padding per
axis, uniform_cell_count cells of width dx, float32 widths, dt = DTYPE(courant / (C0 sqrt(sum 1 / dx_min^2))) of the
float32 widths; cell edges (k - origin) dx in float64, containing cell with the 1e-9-cell snap.  BoundaryConfig3D
keeps open_sol's face types, CPML settings and validation messages (physics/em3d/boundaries3d.py:17-158).
"""
from __future__ import annotations

import math

import numpy as np

from .constants import DTYPE
from .domain import BoxMask, MaterialGrid, containing_cell
from .grid import uniform_cell_count, yee_time_step

FACES_3D = ('x_lo', 'x_hi', 'y_lo', 'y_hi', 'z_lo', 'z_hi')
AXES = ('x', 'y', 'z')
MIRROR_TYPES_3D = ('symmetric', 'antisymmetric')
FACE_TYPES_3D = ('cpml', 'pec', 'pmc', 'periodic', *MIRROR_TYPES_3D)
MIRROR_GHOST_CELLS = 1


def courant_time_step_3d(dx_min, dy_min, dz_min, courant_factor=None):
    """float32 EM time step of the 3D CFL limit of the finest cells (core/grid3d.py:8-17)."""
    return yee_time_step(dx_min, dy_min, dz_min, courant=courant_factor)


class BoundaryConfig3D:
    """Per-face type over FACES_3D plus the CPML settings (boundaries3d.py:17-140)."""

    def __init__(self, faces: dict = None, npml: int = 15, order: int = 3, sigma_factor: float = 1.0,
                 kappa_max: float = 15.0, alpha_max: float = 0.0, bloch_k=(0.0, 0.0, 0.0)):
        faces = dict(faces or {})
        unknown = sorted(set(faces) - set(FACES_3D))
        if unknown:
            raise ValueError(f'BoundaryConfig3D: unknown faces {unknown}; valid: {", ".join(FACES_3D)}')
        for face in FACES_3D:
            setattr(self, face, faces.get(face, 'cpml'))
        self.cpml_npml = npml
        self.cpml_order = order
        self.cpml_sigma_factor = sigma_factor
        self.cpml_kappa_max = kappa_max
        self.cpml_alpha_max = alpha_max
        self.bloch_kx, self.bloch_ky, self.bloch_kz = (float(value) for value in bloch_k)
        self.validate()

    def validate(self):
        for face in FACES_3D:
            if getattr(self, face) not in FACE_TYPES_3D:
                raise ValueError(f'{face} must be one of {", ".join(FACE_TYPES_3D)}, got {getattr(self, face)!r}')
        if not all(math.isfinite(value) for value in self.bloch_k):
            raise ValueError(f'bloch_kx / bloch_ky / bloch_kz must be finite [rad/m], got {self.bloch_k}')
        for axis in AXES:
            lo, hi = getattr(self, f'{axis}_lo'), getattr(self, f'{axis}_hi')
            if (lo == 'periodic') != (hi == 'periodic'):
                raise ValueError(f'{axis}: periodic faces must be paired, got {lo} / {hi}')
        if self.needs_cpml:
            if int(self.cpml_npml) != self.cpml_npml or self.cpml_npml < 1:
                raise ValueError(f'cpml_npml must be an integer >= 1 with a cpml face, got {self.cpml_npml!r}')
            if int(self.cpml_order) != self.cpml_order or self.cpml_order < 1:
                raise ValueError(f'cpml_order must be an integer >= 1, got {self.cpml_order!r}')
            if not self.cpml_sigma_factor > 0.0 or not self.cpml_kappa_max >= 1.0 or not self.cpml_alpha_max >= 0.0:
                raise ValueError('CPML needs sigma_factor > 0, kappa_max >= 1 and alpha_max >= 0, got '
                                 f'{self.cpml_sigma_factor!r}, {self.cpml_kappa_max!r}, {self.cpml_alpha_max!r}')

    def require_supported(self):
        """NotImplementedError for the face kinds the B200 3D engine does not step (mirrors, Bloch phases)."""
        mirrors = [face for face in FACES_3D if getattr(self, face) in MIRROR_TYPES_3D]
        if mirrors:
            raise NotImplementedError(f'the B200 3D engine has no mirror faces yet ({", ".join(mirrors)})')
        if self.has_bloch_phase:
            raise NotImplementedError('the B200 3D engine steps one real field set: no Bloch phase')

    @property
    def needs_cpml(self) -> bool:
        return any(getattr(self, face) == 'cpml' for face in FACES_3D)

    @property
    def cpml_sides(self) -> dict:
        return {face: getattr(self, face) == 'cpml' for face in FACES_3D}

    @property
    def npml_sides(self) -> dict:
        return {face: int(self.cpml_npml) if getattr(self, face) == 'cpml'
                else MIRROR_GHOST_CELLS if getattr(self, face) in MIRROR_TYPES_3D else 0 for face in FACES_3D}

    def periodic(self, axis) -> bool:
        return getattr(self, f'{axis}_lo') == 'periodic'

    @property
    def bloch_k(self) -> tuple:
        return (self.bloch_kx, self.bloch_ky, self.bloch_kz)

    @property
    def has_bloch_phase(self) -> bool:
        return any(self.periodic(axis) and k != 0.0 for axis, k in zip(AXES, self.bloch_k))

    def __eq__(self, other):
        if not isinstance(other, BoundaryConfig3D):
            return NotImplemented
        names = list(FACES_3D) + ['cpml_npml', 'cpml_order', 'cpml_sigma_factor', 'cpml_kappa_max',
                                  'cpml_alpha_max', 'bloch_kx', 'bloch_ky', 'bloch_kz']
        return all(getattr(self, n) == getattr(other, n) for n in names)

    __hash__ = None

    def __repr__(self):
        return f"BoundaryConfig3D({', '.join(f'{face}={getattr(self, face)!r}' for face in FACES_3D)})"


class Domain3D:
    """Grid shape, float32 widths and dt, padding per face, float32 MaterialGrid (nx, ny, nz); physical origin at the
    window's lower corner."""

    dimensions = 3

    def __init__(self, shape, dx, npml_sides, boundary_config, sizes, courant=None, pinned_host=False):
        self.shape = tuple(int(n) for n in shape)
        self.nx, self.ny, self.nz = self.shape
        self.dx = float(dx)
        self.npml_sides = {face: int(npml_sides.get(face, 0)) for face in FACES_3D}
        self.boundary_config = boundary_config
        self.size_x, self.size_y, self.size_z = (float(s) for s in sizes)
        for axis, count in zip(AXES, self.shape):
            if count - self.npml_sides[f'{axis}_lo'] - self.npml_sides[f'{axis}_hi'] < 1:
                raise ValueError(f"Domain3D has no physical cells along {axis}: grid {self.shape}, "
                                 f"PML sides {self.npml_sides}")
        dx32 = float(DTYPE(self.dx))
        self.grid_widths = tuple(np.full(n, dx32) for n in self.shape)   # float32 widths as float64
        self.dt = courant_time_step_3d(dx32, dx32, dx32, courant)
        self.courant = DTYPE(0.99 if courant is None else courant)
        self.origins = tuple(self.npml_sides[f'{axis}_lo'] for axis in AXES)
        self._edges = tuple((np.arange(n + 1) - o) * self.dx for n, o in zip(self.shape, self.origins))
        self.materials = MaterialGrid(self.shape, pinned=pinned_host)

    @classmethod
    def uniform(cls, size_x: float, size_y: float, size_z: float, dx: float, npml_sides: dict = None,
                courant: float = None, boundary_config=None, pinned_host=False):
        """Cubic cells of width dx; npml_sides (FACES_3D keys, missing = 0) pad the window with dx cells
        (core/domain3d.py:55-65)."""
        if not dx > 0:
            raise ValueError(f"Grid3D needs dx > 0, got {dx}")
        sides = {face: int((npml_sides or {}).get(face, 0)) for face in FACES_3D}
        totals = [size + (sides[f'{axis}_lo'] + sides[f'{axis}_hi']) * dx
                  for axis, size in zip(AXES, (size_x, size_y, size_z))]
        shape = [uniform_cell_count(total, dx) for total in totals]
        return cls(shape, dx, sides, boundary_config, (size_x, size_y, size_z), courant, pinned_host)

    def physical_window(self):
        return tuple(slice(self.npml_sides[f'{axis}_lo'], n - self.npml_sides[f'{axis}_hi'])
                     for axis, n in zip(AXES, self.shape))

    def cell_edges(self):
        return self._edges

    def cell_centers(self):
        return tuple(0.5 * (e[:-1] + e[1:]) for e in self._edges)

    def validate_physical_pos(self, x, y, z, label=''):
        sizes = (self.size_x, self.size_y, self.size_z)
        tolerance = 1e-9 * max(sizes)
        if not all(-tolerance <= v <= s + tolerance for v, s in zip((x, y, z), sizes)):
            coordinates = ', '.join(f'{value*1e6:.10g}' for value in (x, y, z))
            extents = ' x '.join(f'{size*1e6:.10g}' for size in sizes)
            raise ValueError(f"{label} position ({coordinates}) µm outside physical domain ({extents}) µm")

    def pos_to_cell(self, x, y, z):
        window = self.physical_window()
        return tuple(containing_cell(c, self._edges[a], window[a].start, window[a].stop - 1)
                     for a, c in enumerate((x, y, z)))

    def sphere_mask(self, cx, cy, cz, radius):
        """Cells whose centre lies within radius of (cx, cy, cz), as a BoxMask over their bounding box."""
        centres = self.cell_centers()
        box = []
        for a, c in enumerate((cx, cy, cz)):
            lo = int(np.searchsorted(centres[a], c - radius, side='left'))
            hi = int(np.searchsorted(centres[a], c + radius, side='right'))
            box.append(slice(max(lo, 0), min(max(hi, 0), self.shape[a])))
        x, y, z = (centres[a][box[a]] for a in range(3))
        block = ((x[:, None, None] - cx) ** 2 + (y[None, :, None] - cy) ** 2
                 + (z[None, None, :] - cz) ** 2) <= radius * radius
        return BoxMask(tuple(box), block)
