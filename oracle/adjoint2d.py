"""ORACLE -- TEST INFRASTRUCTURE ONLY.

Nothing in the product (``opensol_b200``) imports this module.  Only ``tests/`` use it, as the reference the device
adjoint is compared with.

The discrete adjoint of the 2D E_z time step in float64 numpy, for small grids: the forward step of oracle/ez2d.c
(the reference's update order: H Yee, H-row CPML per side, E Yee, E-row CPML per side, line injection, DFT sample;
open_sol/physics/em/solvers/fdtd_ez_2d.py:71-119) written out vectorised with its E history kept, and its exact
transpose run backward in time.  open_sol has no FDTD adjoint; the gradient this module computes is checked in the
tests against central finite differences of the float64 oracle stepper (itself pinned to the reference's float64
stepper), and the device adjoint is checked against both.

Objective: J = flux of one monitor at one frequency after n steps (FluxMonitor.flux, monitors.py:371-379).  The
parameter is eps_r on the cells of a design box away from CPML, sources and monitors, where E^{n+1} = E^n + cb curl,
cb = dt / (eps_r eps0), so dJ/deps_r = -(1 / eps_r) sum_n lambda_E^{n+1} (E^{n+1} - E^n), lambda_E^{n+1} being the
adjoint of E right after the E update of step n.
"""
from __future__ import annotations

import numpy as np

from oracle.fdtd2d import FACES, dft_phases


def _wrap(v):
    return v * 1.0 + v * 0.0


class _Ops:
    """The float64 coefficient arrays and CPML rows of a finalized OracleEz2D (precision 'double')."""

    def __init__(self, o):
        d = o.domain
        self.nx, self.ny, self.px, self.py, self.npml = d.nx, d.ny, d.periodic_x, d.periodic_y, d.npml
        self.ca, self.cb, self.da, self.db = (np.asarray(a, np.float64) for a in (o.ca, o.cb, o.da, o.db))
        self.ixe = np.asarray(o.curl['inv_dx_e'], np.float64)
        self.ixh = np.asarray(o.curl['inv_dx_h'], np.float64)
        self.iye = np.asarray(o.curl['inv_dy_e'], np.float64)
        self.iyh = np.asarray(o.curl['inv_dy_h'], np.float64)
        self.sides = []
        for side in o.cpml_sides:
            n = self.nx if side.name[0] == 'x' else self.ny
            lo = side.name.endswith('lo')
            first_e = 1 if lo else n - self.npml - 1
            first_h = 0 if lo else n - self.npml - 1
            self.sides.append({'name': side.name, 'x': side.name[0] == 'x',
                               'rows_e': np.arange(first_e, first_e + self.npml),
                               'rows_h': np.arange(first_h, first_h + self.npml),
                               'b_e': np.asarray(side.b_e, np.float64), 'a_e': np.asarray(side.a_e, np.float64),
                               'inv_e': np.asarray(side.inv_e, np.float64),
                               'b_h': np.asarray(side.b_h, np.float64), 'a_h': np.asarray(side.a_h, np.float64),
                               'inv_h': np.asarray(side.inv_h, np.float64)})
        self.hx_rows = np.arange(self.ny) if self.py else np.arange(self.ny - 1)   # updated H_x columns
        self.hy_rows = np.arange(self.nx) if self.px else np.arange(self.nx - 1)   # updated H_y rows

    # ---- forward half steps (oracle/ez2d.c update_h / cpml_side / update_e)
    def h_half(self, E, Hx, Hy, psi_h):
        ny, nx = self.ny, self.nx
        j = self.hx_rows
        jp = (j + 1) % ny
        e_up_j = np.where((j + 1 < ny)[None, :], E[:, jp], _wrap(E[:, jp]))
        Hx[:, j] = self.da[:, j] * Hx[:, j] - self.db[:, j] * (e_up_j - E[:, j]) * self.iyh[j][None, :]
        i = self.hy_rows
        ip = (i + 1) % nx
        e_up_i = np.where((i + 1 < nx)[:, None], E[ip, :], _wrap(E[ip, :]))
        Hy[i, :] = self.da[i, :] * Hy[i, :] + self.db[i, :] * (e_up_i - E[i, :]) * self.ixh[i][:, None]
        for s in self.sides:
            r = s['rows_h']
            if s['x']:
                q = psi_h[s['name']] * s['b_h'][:, None]
                q = q + s['a_h'][:, None] * (E[r + 1, :] - E[r, :]) * s['inv_h'][:, None]
                psi_h[s['name']] = q
                Hy[r, :] = Hy[r, :] + 1.0 * self.db[r, :] * q
            else:
                q = psi_h[s['name']] * s['b_h'][None, :]
                q = q + s['a_h'][None, :] * (E[:, r + 1] - E[:, r]) * s['inv_h'][None, :]
                psi_h[s['name']] = q
                Hx[:, r] = Hx[:, r] + (-1.0) * self.db[:, r] * q

    def e_half(self, E, Hx, Hy, psi_e):
        nx, ny = self.nx, self.ny
        curl = np.empty_like(E)
        curl[1:, :] = (Hy[1:, :] - Hy[:-1, :]) * self.ixe[1:, None]
        curl[0, :] = ((Hy[0, :] - _wrap(Hy[nx - 1, :])) if self.px else Hy[0, :]) * self.ixe[0]
        curl[:, 1:] -= (Hx[:, 1:] - Hx[:, :-1]) * self.iye[None, 1:]
        curl[:, 0] -= ((Hx[:, 0] - _wrap(Hx[:, ny - 1])) if self.py else Hx[:, 0]) * self.iye[0]
        E[...] = self.ca * E + self.cb * curl
        for s in self.sides:
            r = s['rows_e']
            if s['x']:
                q = psi_e[s['name']] * s['b_e'][:, None]
                q = q + s['a_e'][:, None] * (Hy[r, :] - Hy[r - 1, :]) * s['inv_e'][:, None]
                psi_e[s['name']] = q
                E[r, :] = E[r, :] + 1.0 * self.cb[r, :] * q
            else:
                q = psi_e[s['name']] * s['b_e'][None, :]
                q = q + s['a_e'][None, :] * (Hx[:, r] - Hx[:, r - 1]) * s['inv_e'][None, :]
                psi_e[s['name']] = q
                E[:, r] = E[:, r] + (-1.0) * self.cb[:, r] * q

    # ---- transposed half steps
    def e_half_T(self, lE, lHx, lHy, lpsi_e):
        """Adjoint of the E half step: lE is the adjoint of E after it; updates lHx / lHy (adjoints of the H it read),
        lpsi_e, and turns lE into the adjoint of E before it."""
        nx, ny = self.nx, self.ny
        u = self.cb * lE
        for s in self.sides:
            r = s['rows_e']
            if s['x']:
                w = lpsi_e[s['name']] + 1.0 * u[r, :]
                g = s['a_e'][:, None] * s['inv_e'][:, None] * w
                np.add.at(lHy, (r,), g)
                np.add.at(lHy, (r - 1,), -g)
                lpsi_e[s['name']] = s['b_e'][:, None] * w
            else:
                w = lpsi_e[s['name']] + (-1.0) * u[:, r]
                g = s['a_e'][None, :] * s['inv_e'][None, :] * w
                lHx[:, r] += g
                lHx[:, r - 1] -= g
                lpsi_e[s['name']] = s['b_e'][None, :] * w
        a = u * self.ixe[:, None]
        lHy += a
        lHy[:-1, :] -= a[1:, :]
        if self.px:
            lHy[nx - 1, :] -= a[0, :]
        c = u * self.iye[None, :]
        lHx -= c
        lHx[:, :-1] += c[:, 1:]
        if self.py:
            lHx[:, ny - 1] += c[:, 0]
        lE *= self.ca

    def h_half_T(self, lE, lHx, lHy, lpsi_h):
        """Adjoint of the H half step: lHx / lHy are the adjoints of H after it; updates lE (adjoint of the E it read)
        and lpsi_h, and turns lHx / lHy into the adjoints of H before it."""
        nx, ny = self.nx, self.ny
        for s in self.sides:
            r = s['rows_h']
            if s['x']:
                w = lpsi_h[s['name']] + 1.0 * self.db[r, :] * lHy[r, :]
                g = s['a_h'][:, None] * s['inv_h'][:, None] * w
                np.add.at(lE, (r + 1,), g)
                np.add.at(lE, (r,), -g)
                lpsi_h[s['name']] = s['b_h'][:, None] * w
            else:
                w = lpsi_h[s['name']] + (-1.0) * self.db[:, r] * lHx[:, r]
                g = s['a_h'][None, :] * s['inv_h'][None, :] * w
                lE[:, r + 1] += g
                lE[:, r] -= g
                lpsi_h[s['name']] = s['b_h'][None, :] * w
        j = self.hx_rows
        v = self.db[:, j] * lHx[:, j] * self.iyh[j][None, :]
        np.add.at(lE, (slice(None), (j + 1) % ny), -v)
        lE[:, j] += v
        lHx[:, j] = self.da[:, j] * lHx[:, j]
        i = self.hy_rows
        v = self.db[i, :] * lHy[i, :] * self.ixh[i][:, None]
        np.add.at(lE, ((i + 1) % nx,), v)
        lE[i, :] -= v
        lHy[i, :] = self.da[i, :] * lHy[i, :]


def _line_cells(mon):
    if mon.normal_axis == 'x':
        return (mon.position, slice(mon.lo, mon.hi)), 'hy'
    return (slice(mon.lo, mon.hi), mon.position), 'hx'


def forward(o, n_steps, box=None):
    """Run a fresh finalized float64 OracleEz2D for n_steps in numpy; returns (E history over `box` (n_steps + 1,
    ...) or None, {'samples': [(q, phases, e, h) per sample of monitor 0]}) and leaves the oracle's fields, spectra
    and clock as its own stepper would."""
    ops = _Ops(o)
    E, Hx, Hy = o.ez, o.hx, o.hy
    psi_h = {k: np.asarray(v, np.float64).copy() for k, v in o.psi_h.items()}
    psi_e = {k: np.asarray(v, np.float64).copy() for k, v in o.psi_e.items()}
    m = o.sample_interval
    values, times_full = o.source_values(n_steps)
    history = None if box is None else np.empty((n_steps + 1,) + E[box].shape)
    if history is not None:
        history[0] = E[box]
    samples = []
    for k in range(n_steps):
        ops.h_half(E, Hx, Hy, psi_h)
        ops.e_half(E, Hx, Hy, psi_e)
        for src, v in zip(o.sources, values):
            if v[k] == 0.0:
                continue
            line = (slice(src.lo, src.hi), src.position) if src.axis == 'x' else (src.position,
                                                                                 slice(src.lo, src.hi))
            E[line] += (np.float32(v[k]) * src.profile).astype(np.float32)
        n = o.n_step + k + 1
        if history is not None:
            history[k + 1] = E[box]
        if o.monitors and n % m == 0:
            q = n // m
            for mi, mon in enumerate(o.monitors):
                ph = dft_phases(2.0 * np.pi * mon.frequencies, times_full[k], mon.dt * m)
                cells, hname = _line_cells(mon)
                e = E[cells].astype(np.float64)
                h = (Hx if hname == 'hx' else Hy)[cells].astype(np.float64)
                phc = ph[:, 0].astype(np.float64) + 1j * ph[:, 1].astype(np.float64)
                mon.e_acc += phc[:, None] * e[None, :]
                mon.h_acc += phc[:, None] * h[None, :]
                if mi == 0:
                    samples.append((k, phc, e, h))
    for name in psi_h:
        o.psi_h[name][...] = psi_h[name]
        o.psi_e[name][...] = psi_e[name]
    o.n_step += n_steps
    o.time = float(times_full[-1]) if n_steps else o.time
    return history, samples


def flux_adjoint_sources(mon, freq_index, samples):
    """Per sample, (dJ/de, dJ/dh) on the monitor's line cells of J = mon.flux()[freq_index]."""
    f = mon.frequencies[freq_index]
    r = np.exp(1j * np.pi * f * mon.dt)
    E_c = mon.e_acc[freq_index]
    H_c = mon.h_acc[freq_index]
    sign = -1.0 if mon.normal_axis == 'x' else 1.0
    scale = np.cos(np.pi * f * mon.dt) * sign * mon.widths
    out = {}
    for k, phc, _, _ in samples:
        ph = phc[freq_index]
        de = scale * np.real(ph * np.conj(H_c * r))
        dh = scale * np.real(E_c * np.conj(ph * r))
        out[k] = (de, dh)
    return out


def gradient(o_builder, n_steps, box, freq_index=0):
    """(J, dJ/deps_r over box) of a float64 oracle built by o_builder() (fresh, finalized), by the adjoint."""
    o = o_builder()
    history, samples = forward(o, n_steps, box)
    mon = o.monitors[0]
    J = float(mon.flux()[freq_index])
    sources = flux_adjoint_sources(mon, freq_index, samples)
    ops = _Ops(o)
    lE = np.zeros((ops.nx, ops.ny))
    lHx, lHy = np.zeros_like(lE), np.zeros_like(lE)
    lpsi_e = {s['name']: np.zeros_like(o.psi_e[s['name']], dtype=np.float64) for s in ops.sides}
    lpsi_h = {s['name']: np.zeros_like(o.psi_h[s['name']], dtype=np.float64) for s in ops.sides}
    cells, hname = _line_cells(mon)
    grad = np.zeros(history.shape[1:])
    for k in range(n_steps - 1, -1, -1):
        if k in sources:
            de, dh = sources[k]
            lE[cells] += de
            (lHx if hname == 'hx' else lHy)[cells] += dh
        grad += lE[box] * (history[k + 1] - history[k])
        ops.e_half_T(lE, lHx, lHy, lpsi_e)
        ops.h_half_T(lE, lHx, lHy, lpsi_h)
    eps = np.asarray(o.eps_r[box], np.float64)
    return J, -grad / eps
