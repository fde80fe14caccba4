"""Dispersive poles of the 2D engines: Drude and Lorentz media (physics/em/materials.py:132-190).

The auxiliary-differential-equation coefficients are computed in float64 and rounded to float32 as open_sol rounds
them; the device steps them in velocity form (J += damping J + drive E, or dP += damping dP - restoring P + drive E,
P += dP).  susceptibility() gives the continuous-time chi(omega) the sheet-source calibration adds on pole cells.
The E_z engine steps a pole on its cells, the H_z engine on the E_x / E_y face sets of pole_face_sets().
"""
from __future__ import annotations

import math

import numpy as np

from .constants import DTYPE, EPS0


def _scalar_or_array(value):
    return complex(value) if np.ndim(value) == 0 else value


class DrudePole:
    """dJ/dt + gamma J = eps0 omega_p^2 E, above a background eps_inf (materials.py:132-157)."""

    def __init__(self, omega_p: float, gamma: float, eps_inf: float = 1.0):
        self.omega_p = DTYPE(omega_p)
        self.gamma = DTYPE(gamma)
        self.eps_inf = DTYPE(eps_inf)

    def ade_coefficients(self, dt):
        """(damping, drive) float32: damping = -gamma dt / (1 + gamma dt / 2), drive = eps0 wp^2 dt / (1 + gamma dt /
        2)."""
        dt = float(dt)
        gamma, wp = float(self.gamma), float(self.omega_p)
        denom = 1.0 + gamma * dt / 2.0
        return DTYPE(-gamma * dt / denom), DTYPE((EPS0 * wp ** 2 * dt) / denom)

    def susceptibility(self, omega):
        omega = np.asarray(omega, dtype=np.float64)
        wp, gamma = float(self.omega_p), float(self.gamma)
        return _scalar_or_array(-wp ** 2 / (omega ** 2 - 1j * gamma * omega))

    def step_term(self, dt):
        """Leap-frog stability term (omega_p dt)^2 / 4 (materials.py:199-211)."""
        return (float(self.omega_p) * dt) ** 2 / 4.0


class LorentzPole:
    """P'' + gamma P' + omega_0^2 P = eps0 delta_eps omega_0^2 E (materials.py:160-190)."""

    def __init__(self, delta_eps: float, omega_0: float, gamma: float):
        self.delta_eps = DTYPE(delta_eps)
        self.omega_0 = DTYPE(omega_0)
        self.gamma = DTYPE(gamma)

    def ade_coefficients(self, dt):
        """(damping, restoring, drive) float32 of the velocity-form step."""
        dt = float(dt)
        w0, g, de = float(self.omega_0), float(self.gamma), float(self.delta_eps)
        denom = 1.0 + g * dt / 2.0
        return (DTYPE(-g * dt / denom), DTYPE(w0 ** 2 * dt ** 2 / denom),
                DTYPE(EPS0 * de * w0 ** 2 * dt ** 2 / denom))

    def susceptibility(self, omega):
        omega = np.asarray(omega, dtype=np.float64)
        w0, gamma, de = float(self.omega_0), float(self.gamma), float(self.delta_eps)
        return _scalar_or_array(de * w0 ** 2 / (w0 ** 2 - omega ** 2 + 1j * gamma * omega))

    def step_term(self, dt):
        """delta_eps (omega_0 dt)^2 / (4 - (omega_0 dt)^2); ValueError when omega_0 dt >= 2."""
        r2 = (float(self.omega_0) * dt) ** 2
        if r2 >= 4.0:
            raise ValueError(f'Lorentz pole: omega_0 dt = {math.sqrt(r2):.4g} >= 2, so the Lorentz update is unstable; '
                             f'lower courant_factor or refine the mesh')
        return float(self.delta_eps) * r2 / (4.0 - r2)


def bounding_box(mask):
    """(slice, slice) bounding the set cells of a full-grid bool mask, None when none is set."""
    rows = np.flatnonzero(mask.any(axis=1))
    if rows.size == 0:
        return None
    cols = np.flatnonzero(mask.any(axis=0))
    return slice(int(rows[0]), int(rows[-1]) + 1), slice(int(cols[0]), int(cols[-1]) + 1)


def pole_face_sets(full_mask, shares_x, shares_y, periodic_x, periodic_y):
    """[(component, face box, float32 face weights on the box)] of a pole's cell mask on the H_z engine's E face sets
    (_pole_faces, fdtd_hz_2d.py:547-570): component 0 = E_x (hi-y faces), 1 = E_y (hi-x faces); weight = the
    width-weighted face average of the float32 mask, cell x lower share + partner x upper share (the partner wraps on
    a periodic axis and is the cell itself on the last face of an open one, yee_grid.py:119-142), boxed on the faces
    whose weight is > 0; a set without such faces is left out."""
    cell = np.asarray(full_mask, dtype=bool).astype(DTYPE)
    nx, ny = cell.shape

    def partners(n, periodic):
        idx = np.arange(n)
        return np.roll(idx, -1) if periodic else np.concatenate((idx[1:], idx[-1:]))

    lo_y, up_y = (np.asarray(a, dtype=DTYPE) for a in shares_y)
    lo_x, up_x = (np.asarray(a, dtype=DTYPE) for a in shares_x)
    weights = (cell * lo_y + cell[:, partners(ny, periodic_y)] * up_y,
               cell * lo_x[:, None] + cell[partners(nx, periodic_x)] * up_x[:, None])
    sets = []
    for component, weight in enumerate(weights):
        box = bounding_box(weight > 0)
        if box is not None:
            sets.append((component, box, np.ascontiguousarray(weight[box])))
    return sets
