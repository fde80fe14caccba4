"""ORACLE -- TEST INFRASTRUCTURE ONLY.

Nothing in the product (``opensol_b200``) imports this module.  Only ``tests/``, ``__graft_entry__.smoke()`` and the
CPU-baseline leg of ``bench.py`` use it, as the reference the CUDA engine is compared with.

A CPU restatement of open_sol's 3D FDTD path (``EMPhysics3D.step`` -> ``FDTDEngine3D.advance``) for a Cartesian
uniform grid with one real field set and single-precision fields:

* setup, in numpy, written from the reference's own expressions so every float32 / float64 rounding matches: grid
  and 3D Courant step (open_sol/core/grid3d.py:8-17,62-68), cell edges and containing cell (core/grid.py:20-31,
  core/domain.py:275-282), curl spacings with the kappa fold (physics/em3d/engine3d.py:191-203), CPML layer rows
  (physics/em3d/boundaries3d.py:207-243 over physics/em/boundaries.py:560-632), hi-face shares
  (physics/em/yee_grid.py:76-84,119-125), the uint16 material index and its per-id tables
  (physics/em3d/material_index3d.py:131-179, engine3d.py:337-369) with the PEC wall layers
  (boundaries3d.py:147-158), the dipole placement, dual volume and calibration (physics3d.py:403-423,
  sources3d.py:31-75, engine3d.py:299-312), flux planes and boxes (physics3d.py:434-497, monitors3d.py:23-162) with
  the DFT phases and sample interval (physics/em/monitors.py:22-24,177-191) and the engine clock (engine3d.py:
  497-554);
* the two fused field updates in C (``oracle/em3d.c``), called through ctypes.

Pinned against fixtures generated from the reference itself (``tests/golden/make_golden3d.py``): bit for bit against
the reference's numpy twins, within float32 rounding against its numba twins.
"""
from __future__ import annotations

import ctypes
import math
import os

import numpy as np

from oracle.fdtd2d import (C0, DTYPE, EPS0, GaussianPulse, containing_cell, cpml_axis_profile, cpml_recursion,
                           dft_phases, dft_sample_interval, uniform_cell_count)

AXES = ('x', 'y', 'z')
FACES_3D = ('x_lo', 'x_hi', 'y_lo', 'y_hi', 'z_lo', 'z_hi')
MAX_MATERIAL_IDS = 65535
_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, '_build', 'libem3d_oracle.so')


# ----------------------------------------------------------------------------------------------- grid

def courant_time_step_3d(dx_min, dy_min, dz_min, courant_factor=None):
    """core/grid3d.py:8-17."""
    courant_factor = 0.99 if courant_factor is None else courant_factor
    inverse_spacing_squared = 1.0 / float(dx_min) ** 2 + 1.0 / float(dy_min) ** 2 + 1.0 / float(dz_min) ** 2
    return DTYPE(float(courant_factor) / (C0 * np.sqrt(inverse_spacing_squared)))


def face_shares(widths, periodic):
    """(lower, upper) float32 hi-face weights (yee_grid.py:76-84,119-125)."""
    widths = np.asarray(widths, dtype=np.float64)
    partner = np.roll(widths, -1) if periodic else np.concatenate((widths[1:], widths[-1:]))
    return (widths / (widths + partner)).astype(DTYPE), (partner / (widths + partner)).astype(DTYPE)


# ----------------------------------------------------------------------------------------------- material index

def material_index(arrays, limit=MAX_MATERIAL_IDS - 1):
    """(uint16 id per cell, float32 table per array name): the id of a cell is the rank of its tuple of value levels
    (arrays in the given order, those with a single value left out) among the occurring tuples in lexicographic order,
    which is what the reference's stage-by-stage ranking computes (material_index3d.py:110-179).  Exact levels only:
    an array or a joint count above `limit` raises (the reference re-quantises those; no oracle case needs it)."""
    levels, names = {}, list(arrays)
    for name in names:
        values = np.unique(arrays[name])
        if values.size > limit:
            raise ValueError(f'{name}: {values.size} distinct values exceed the exact index of the oracle')
        levels[name] = values.astype(DTYPE)
    order = [name for name in names if levels[name].size > 1]
    shape = next(iter(arrays.values())).shape
    if not order:
        return np.zeros(shape, np.uint16), {name: levels[name][:1].copy() for name in names}
    codes = np.stack([np.searchsorted(levels[name], arrays[name].ravel()) for name in order], axis=1)
    if len(order) == 1:   # one varying array: its level codes are already the ranks
        tuples, ids = np.arange(levels[order[0]].size)[:, None], codes[:, 0]
    else:
        tuples, ids = np.unique(codes, axis=0, return_inverse=True)
    if tuples.shape[0] > limit:
        raise ValueError('joint material count exceeds the exact index of the oracle')
    tables = {}
    for name in names:
        if name in order:
            tables[name] = levels[name][tuples[:, order.index(name)]].astype(DTYPE)
        else:
            tables[name] = np.repeat(levels[name][:1], tuples.shape[0]).astype(DTYPE)
    return ids.reshape(shape).astype(np.uint16), tables


# ----------------------------------------------------------------------------------------------- monitors

def face_samples(widths, first_edge, last_edge, wrap=False):
    """monitors3d.py:23-36."""
    if wrap:
        widths = np.asarray(widths, dtype=np.float64)
        return slice(0, widths.size), 0.5 * (widths + np.roll(widths, -1))
    edges = np.arange(max(first_edge, 1), last_edge + 1)
    weights = np.empty(edges.size)
    for position, edge in enumerate(edges):
        below = widths[edge - 1] if edge > first_edge else 0.0
        above = widths[edge] if edge < last_edge else 0.0
        weights[position] = 0.5 * (below + above)
    return slice(int(edges[0]) - 1, int(edges[-1])), weights


class PlaneFlux:
    """PlaneFlux3D (monitors3d.py:42-134): two (E, H) pairs on a cell-edge plane, complex128 running DFTs."""

    def __init__(self, normal_axis, edge, bounds, frequencies, dt, widths, shape, periodic):
        self.normal_axis, self.edge = normal_axis, int(edge)
        self.bounds = tuple(tuple(int(v) for v in b) for b in bounds)
        self.frequencies = np.atleast_1d(np.asarray(frequencies, dtype=np.float64))
        self.dt = float(dt)
        self.sample_interval = 1
        first_axis, second_axis = (normal_axis + 1) % 3, (normal_axis + 2) % 3
        self.pairs = []
        for e_axis, h_axis, face_axis, cell_axis, sign in ((first_axis, second_axis, first_axis, second_axis, 1.0),
                                                           (second_axis, first_axis, second_axis, first_axis, -1.0)):
            wrap = bool(periodic[face_axis]) and tuple(self.bounds[face_axis]) == (0, shape[face_axis])
            face_slice, face_weights = face_samples(widths[face_axis], *self.bounds[face_axis], wrap=wrap)
            cell_slice = slice(*self.bounds[cell_axis])
            cell_weights = np.asarray(widths[cell_axis][cell_slice], dtype=np.float64)
            lower, upper, h_index = [None] * 3, [None] * 3, [None] * 3
            for index in (lower, upper, h_index):
                index[face_axis], index[cell_axis] = face_slice, cell_slice
            lower[normal_axis], upper[normal_axis], h_index[normal_axis] = edge - 1, edge, edge - 1
            by_axis = {face_axis: face_weights, cell_axis: cell_weights}
            low_axis, high_axis = sorted((face_axis, cell_axis))
            area = np.outer(by_axis[low_axis], by_axis[high_axis])
            self.pairs.append({'e': 'e' + 'xyz'[e_axis], 'h': 'h' + 'xyz'[h_axis], 'sign': sign, 'area': area,
                               'lower': tuple(lower), 'upper': tuple(upper), 'h_index': tuple(h_index),
                               'e_dft': np.zeros((self.frequencies.size,) + area.shape, np.complex128),
                               'h_dft': np.zeros((self.frequencies.size,) + area.shape, np.complex128)})

    def update(self, fields, phases):
        """E = mean of the two layers across the plane, H on the plane; complex128 sums (monitors.py:84-96)."""
        ph = (phases[:, 0].astype(np.float64) + 1j * phases[:, 1].astype(np.float64))[:, None, None]
        for pair in self.pairs:
            e = fields[pair['e']]
            mean = 0.5 * (e[pair['lower']].astype(np.float64) + e[pair['upper']].astype(np.float64))
            pair['e_dft'] += ph * mean[None]
            pair['h_dft'] += ph * fields[pair['h']][pair['h_index']].astype(np.float64)[None]

    def spectra(self):
        return [pair[key] for pair in self.pairs for key in ('e_dft', 'h_dft')]

    def flux(self):
        """monitors3d.py:116-134: cos(omega dt / 2) Re(E H*) over the plane, H re-timed to the E time."""
        retime = np.exp(1j * np.pi * self.frequencies * self.dt)[:, None, None]
        total = np.zeros(self.frequencies.size)
        for pair in self.pairs:
            total += pair['sign'] * np.einsum('fij,ij->f', np.real(pair['e_dft'] * np.conj(pair['h_dft'] * retime)),
                                              pair['area'])
        return np.cos(np.pi * self.frequencies * self.dt) * total


class FluxBox:
    """FluxBox3D (monitors3d.py:137-162): six planes, net outward flux."""

    def __init__(self, edge_bounds, frequencies, dt, widths, shape, periodic):
        self.frequencies = np.atleast_1d(np.asarray(frequencies, dtype=np.float64))
        self.faces = [(sign, PlaneFlux(axis, edge_bounds[axis][side], edge_bounds, self.frequencies, dt, widths, shape,
                                       periodic))
                      for axis in range(3) for side, sign in ((0, -1.0), (1, 1.0))]
        self.sample_interval = 1

    def planes(self):
        return [plane for _, plane in self.faces]

    def update(self, fields, phases):
        for _, plane in self.faces:
            plane.update(fields, phases)

    def spectra(self):
        return [s for plane in self.planes() for s in plane.spectra()]

    def flux(self):
        return sum(sign * plane.flux() for sign, plane in self.faces)


# ----------------------------------------------------------------------------------------------- ctypes binding

_I = ctypes.POINTER(ctypes.c_int32)
_REALS = {'single': (np.float32, ctypes.c_float, 'libem3d_oracle.so'),
          'double': (np.float64, ctypes.c_double, 'libem3d_oracle_f64.so')}


def _state_type(ctype):
    """The C struct OracleEM3D for arithmetic type ctype (float or double build of oracle/em3d.c)."""
    P = ctypes.POINTER(ctype)

    class State(ctypes.Structure):
        _fields_ = [('nx', ctypes.c_int32), ('ny', ctypes.c_int32), ('nz', ctypes.c_int32),
                    ('px', ctypes.c_int32), ('py', ctypes.c_int32), ('pz', ctypes.c_int32)] + \
                   [(name, P) for name in ('ex', 'ey', 'ez', 'hx', 'hy', 'hz')] + \
                   [('mat', ctypes.POINTER(ctypes.c_uint16))] + \
                   [(name, P) for name in ('t_ex', 't_ey', 't_ez', 't_sig', 't_mu', 't_sm', 'iex', 'iey', 'iez',
                                            'ihx', 'ihy', 'ihz', 'wlx', 'wux', 'wly', 'wuy', 'wlz', 'wuz')] + \
                   [('dt', ctype), ('nr', ctypes.c_int32 * 3), ('rm_h', _I * 3), ('rm_e', _I * 3),
                    ('b_h', P * 3), ('g_h', P * 3), ('b_e', P * 3), ('g_e', P * 3),
                    ('ph_first', P * 3), ('ph_second', P * 3), ('pe_first', P * 3), ('pe_second', P * 3)]
    return State


_LIB = {}


def load_library(precision='single'):
    """(library, State struct type) of the float ('single') or double build."""
    if precision not in _LIB:
        _, ctype, name = _REALS[precision]
        path = os.path.join(_HERE, '_build', name)
        if not os.path.exists(path):
            raise RuntimeError(f'oracle library {path} is not built (run: make -C oracle)')
        lib = ctypes.CDLL(path)
        State = _state_type(ctype)
        lib.oracle_em3d_update_h.argtypes = [ctypes.POINTER(State)]
        lib.oracle_em3d_update_e.argtypes = [ctypes.POINTER(State)]
        lib.oracle_em3d_face_cb.argtypes = [ctypes.POINTER(State), ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                            ctypes.c_int]
        lib.oracle_em3d_face_cb.restype = ctype
        _LIB[precision] = (lib, State)
    return _LIB[precision]


def _fp(a):
    if a is None:
        return None
    ctype = ctypes.c_double if a.dtype == np.float64 else ctypes.c_float
    return a.ctypes.data_as(ctypes.POINTER(ctype))


# ----------------------------------------------------------------------------------------------- the oracle run

class OracleEM3D:
    """The 3D FDTD path on the CPU for a uniform grid: Domain3D.uniform(size_x, size_y, size_z, dx, npml_sides,
    boundary_config) with face types over FACES_3D (cpml / pec / pmc / periodic), float32 material arrays written by
    the caller (eps_r, sigma_e, mu_r, optional sigma_m), then add_dipole / add_flux_box / add_flux_plane, finalize(),
    run(n_steps).  precision='double' steps float64 fields with float64 coefficient and CPML rows (the float32
    materials, dt and face shares promoted): the run the float32 results' error is stated against."""

    def __init__(self, size_x, size_y, size_z, dx, faces=None, npml=15, courant=None, precision='single'):
        if precision not in _REALS:
            raise ValueError(f"precision must be 'single' or 'double', got {precision!r}")
        self.precision = precision
        self.real = _REALS[precision][0]
        self.faces = {face: (faces or {}).get(face, 'cpml') for face in FACES_3D}
        self.npml = int(npml)
        self.sides = {face: self.npml if kind == 'cpml' else 0 for face, kind in self.faces.items()}
        sizes = (size_x, size_y, size_z)
        self.sizes = tuple(float(s) for s in sizes)
        self.dx = float(dx)
        self.shape = tuple(uniform_cell_count(size + (self.sides[f'{a}_lo'] + self.sides[f'{a}_hi']) * dx, dx)
                           for a, size in zip(AXES, sizes))
        self.nx, self.ny, self.nz = self.shape
        dx32 = float(DTYPE(dx))
        self.dt = float(courant_time_step_3d(dx32, dx32, dx32, courant))
        self.periodic = tuple(self.faces[f'{a}_lo'] == 'periodic' for a in AXES)
        self.widths = tuple(np.full(n, dx32) for n in self.shape)           # engine widths (float32 dx as float64)
        self.origins = tuple(self.sides[f'{a}_lo'] for a in AXES)
        self.window = tuple(slice(o, n - self.sides[f'{a}_hi']) for a, o, n in zip(AXES, self.origins, self.shape))
        self.edges = tuple((np.arange(n + 1) - o) * self.dx for n, o in zip(self.shape, self.origins))
        self.materials = {'eps_r': np.ones(self.shape, DTYPE), 'sigma_e': np.zeros(self.shape, DTYPE),
                          'mu_r': np.ones(self.shape, DTYPE)}
        self.fields = {name: np.zeros(self.shape, self.real) for name in ('ex', 'ey', 'ez', 'hx', 'hy', 'hz')}
        self.sources, self.monitors = [], []
        self.time, self.n_step = 0.0, 0
        self._build_rows()

    # ---- rows: spacings, CPML, shares (engine3d.py:189-205, boundaries3d.py:207-243)
    def _build_rows(self):
        bulk = []
        for widths, periodic in zip(self.widths, self.periodic):
            inverse_h = 1.0 / (0.5 * (widths + np.roll(widths, -1)))
            if not periodic:
                inverse_h[-1] = 0.0
            bulk.append((1.0 / widths, inverse_h))
        pml_sizes = tuple(float(max(w[0], w[-1])) for w in self.widths)
        self.inv_e, self.inv_h, self.layers = [], [], {}
        for axis_index, axis in enumerate(AXES):
            n = self.shape[axis_index]
            se, ke, ae, sh, kh, ah = cpml_axis_profile(self.faces, n, axis, self.npml, pml_sizes[axis_index])
            inverse_e, inverse_h = bulk[axis_index]
            self.inv_e.append((inverse_e / ke).astype(self.real))
            self.inv_h.append((inverse_h / kh).astype(self.real))
            sides = []
            for side in ('lo', 'hi'):
                if self.faces[f'{axis}_{side}'] == 'cpml':
                    sides.append((slice(1, self.npml + 1), slice(0, self.npml)) if side == 'lo' else
                                 (slice(n - self.npml - 1, n - 1), slice(n - self.npml - 1, n - 1)))
            if not sides:
                continue
            for kind_index, kind in enumerate(('e', 'h')):
                row_map = np.full(n, -1, dtype=np.int32)
                decays, gains = [], []
                sigma, kappa, alpha = (se, ke, ae) if kind == 'e' else (sh, kh, ah)
                for rows in sides:
                    selected = rows[kind_index]
                    row_map[selected] = np.arange(len(decays) * self.npml, (len(decays) + 1) * self.npml,
                                                  dtype=np.int32)
                    a, b = cpml_recursion(sigma[selected], kappa[selected], alpha[selected], self.dt, self.real)
                    inverse = (inverse_e if kind == 'e' else inverse_h)[selected].astype(self.real)
                    decays.append(b)
                    gains.append(a * inverse)
                n_rows = self.npml * len(sides)
                psi_shape = list(self.shape)
                psi_shape[axis_index] = n_rows
                self.layers[(axis_index, kind)] = {
                    'row_map': row_map, 'b': np.concatenate(decays).astype(self.real),
                    'gain': np.concatenate(gains).astype(self.real), 'n_rows': n_rows,
                    'first': np.zeros(psi_shape, self.real), 'second': np.zeros(psi_shape, self.real)}
        self.shares = [tuple(np.asarray(w, self.real) for w in face_shares(widths, p))
                       for widths, p in zip(self.widths, self.periodic)]

    # ---- placement (domain3d.py:123-140, physics3d.py:403-497)
    def pos_to_cell(self, position):
        return [containing_cell(c, self.edges[a], self.window[a].start, self.window[a].stop - 1)
                for a, c in enumerate(position)]

    def nearest_edge(self, axis, coordinate):
        first, last = self.window[axis].start, self.window[axis].stop
        edges = self.edges[axis]
        return first + int(np.argmin(np.abs(edges[first:last + 1] - float(coordinate))))

    def add_dipole(self, x, y, z, orientation='z', dipole_moment=1e-12, wavelength=None, bandwidth=0.5):
        axis = AXES.index(orientation)
        cell = self.pos_to_cell((x, y, z))
        first, last = self.window[axis].start, self.window[axis].stop - 2
        cell[axis] = min(range(first, last + 1),
                         key=lambda f: abs(float(self.edges[axis][f + 1]) - (x, y, z)[axis]))
        lengths = []
        for other, widths in enumerate(self.widths):
            index = cell[other]
            partner = (index + 1) % widths.size if self.periodic[other] else min(index + 1, widths.size - 1)
            lengths.append(0.5 * (widths[index] + widths[partner]) if other == axis else widths[index])
        source = {'axis': axis, 'cell': tuple(cell), 'temporal': GaussianPulse(C0 / wavelength, bandwidth),
                  'moment': float(dipole_moment), 'volume': float(math.prod(lengths)), 'weight': None}
        self.sources.append(source)
        return source

    def add_flux_box(self, lo, hi, wavelengths=None, frequencies=None):
        bounds = []
        for axis in range(3):
            first = self.nearest_edge(axis, min(lo[axis], hi[axis]))
            last = self.nearest_edge(axis, max(lo[axis], hi[axis]))
            bounds.append((first, last))
        freqs = (np.asarray(frequencies, dtype=np.float64) if frequencies is not None
                 else C0 / np.asarray(wavelengths, dtype=np.float64))
        box = FluxBox(bounds, freqs, self.dt, self.widths, self.shape, self.periodic)
        self.monitors.append(box)
        return box

    def add_flux_plane(self, normal, position, wavelengths):
        axis = AXES.index(normal)
        bounds = [(w.start, w.stop) for w in self.window]
        bounds[axis] = (self.nearest_edge(axis, position),) * 2
        plane = PlaneFlux(axis, bounds[axis][0], bounds, C0 / np.asarray(wavelengths, dtype=np.float64), self.dt,
                          self.widths, self.shape, self.periodic)
        self.monitors.append(plane)
        return plane

    # ---- finalize (physics3d.py:192-217, engine3d.py:337-369)
    def finalize(self):
        names = ['eps_r', 'sigma_e', 'mu_r'] + [n for n in ('eps_xx', 'eps_yy', 'sigma_m') if n in self.materials]
        self.material_id, tables = material_index({n: self.materials[n] for n in names})
        pec_id = np.uint16(tables['eps_r'].size)

        def with_pec(values, pec_value):
            return np.concatenate((values, np.full(1, pec_value, DTYPE))).astype(self.real)
        self.t_ez = with_pec(tables['eps_r'], -1.0)
        self.t_ex = with_pec(tables.get('eps_xx', tables['eps_r']), -1.0)
        self.t_ey = with_pec(tables.get('eps_yy', tables['eps_r']), -1.0)
        self.t_sig = with_pec(tables['sigma_e'], 0.0)
        self.t_mu = with_pec(tables['mu_r'], 1.0)
        self.t_sm = with_pec(tables.get('sigma_m', np.zeros(tables['eps_r'].size, DTYPE)), 0.0)
        for axis, name in enumerate(AXES):
            for side in ('lo', 'hi'):
                if self.faces[f'{name}_{side}'] == 'pec':
                    layer = self.window[axis].start if side == 'lo' else self.window[axis].stop - 1
                    key = [slice(None)] * 3
                    key[axis] = slice(layer, layer + 1)
                    self.material_id[tuple(key)] = pec_id
        self._state = self._make_state()
        lib, _ = load_library(self.precision)
        for source in self.sources:
            cb = lib.oracle_em3d_face_cb(ctypes.byref(self._state), source['axis'], *source['cell'])
            source['weight'] = self.real(self.real(cb) * self.real(source['moment'] / source['volume']))
        interval = dft_sample_interval(self.dt, [_SourceView(s) for s in self.sources],
                                       [m.frequencies for m in self.monitors])
        for monitor in self.monitors:
            monitor.sample_interval = interval
            for plane in (monitor.planes() if isinstance(monitor, FluxBox) else [monitor]):
                plane.sample_interval = interval

    def _make_state(self):
        st = load_library(self.precision)[1]()
        st.nx, st.ny, st.nz = self.shape
        st.px, st.py, st.pz = (int(p) for p in self.periodic)
        for name, arr in self.fields.items():
            setattr(st, name, _fp(arr))
        self._keep = [self.material_id, self.t_ex, self.t_ey, self.t_ez, self.t_sig, self.t_mu, self.t_sm]
        st.mat = self.material_id.ctypes.data_as(ctypes.POINTER(ctypes.c_uint16))
        for name in ('t_ex', 't_ey', 't_ez', 't_sig', 't_mu', 't_sm'):
            setattr(st, name, _fp(getattr(self, name)))
        for axis, a in enumerate('xyz'):
            setattr(st, f'ie{a}', _fp(self.inv_e[axis]))
            setattr(st, f'ih{a}', _fp(self.inv_h[axis]))
            setattr(st, f'wl{a}', _fp(self.shares[axis][0]))
            setattr(st, f'wu{a}', _fp(self.shares[axis][1]))
        st.dt = self.real(DTYPE(self.dt))
        for axis in range(3):
            h, e = self.layers.get((axis, 'h')), self.layers.get((axis, 'e'))
            st.nr[axis] = h['n_rows'] if h else 0
            if h:
                st.rm_h[axis] = h['row_map'].ctypes.data_as(ctypes.POINTER(ctypes.c_int32))
                st.rm_e[axis] = e['row_map'].ctypes.data_as(ctypes.POINTER(ctypes.c_int32))
                st.b_h[axis], st.g_h[axis] = _fp(h['b']), _fp(h['gain'])
                st.b_e[axis], st.g_e[axis] = _fp(e['b']), _fp(e['gain'])
                st.ph_first[axis], st.ph_second[axis] = _fp(h['first']), _fp(h['second'])
                st.pe_first[axis], st.pe_second[axis] = _fp(e['first']), _fp(e['second'])
        return st

    # ---- stepping (engine3d.py:497-554)
    def source_value(self, source, t_half):
        return self.real(source['temporal'](t_half))

    def run(self, n_steps):
        lib, _ = load_library(self.precision)
        for _ in range(int(n_steps)):
            t = self.time
            lib.oracle_em3d_update_h(ctypes.byref(self._state))
            lib.oracle_em3d_update_e(ctypes.byref(self._state))
            t_half = t + 0.5 * self.dt
            for source in self.sources:
                value = self.source_value(source, t_half)
                field = self.fields['e' + 'xyz'[source['axis']]]
                i, j, k = source['cell']
                field[i, j, k] = self.real(field[i, j, k] + self.real(value * source['weight']))
            self.time = t + self.dt
            self.n_step += 1
            for monitor in self.monitors:
                if self.n_step % monitor.sample_interval == 0:
                    omega = 2.0 * np.pi * monitor.frequencies
                    monitor.update(self.fields, dft_phases(omega, self.time, self.dt * monitor.sample_interval))


class _SourceView:
    """The temporal of an oracle dipole as dft_sample_interval reads it."""

    def __init__(self, source):
        self.temporal = source['temporal']
