"""Pin the H_z oracle to open_sol itself: every H_z golden fixture (generated by running the reference's CPU backend,
tests/golden/make_golden_hz.py) must be reproduced bit for bit -- H_z / E_x / E_y at every checkpoint (SHA-256 and
stored arrays), complex128 line spectra, fluxes and the setup rows (face coefficients, curl spacings, CPML rows,
calibrated sheet profiles)."""
import hashlib
import os

import numpy as np
import pytest

from cases import apply_ops
from cases_hz import HZ_CASES
from oracle.hz2d import OracleHz2D, e_face_coefficients, face_shares

GOLDEN = os.path.join(os.path.dirname(__file__), 'golden')


def _digest(a):
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


def _oracle_kwargs(spec):
    return {k: v for k, v in spec['sim'].items() if k != 'polarization'}


def _run_oracle(spec):
    o = OracleHz2D(**_oracle_kwargs(spec))
    mons = apply_ops(o, spec)
    snaps = {}
    done = 0
    for cp in spec['checkpoints']:
        o.run(n_steps=cp - done)
        done = cp
        snaps[cp] = ({n: getattr(o, n).copy() for n in ('hz', 'ex', 'ey')},
                     [(m.e_acc.copy(), m.h_acc.copy(), m.flux()) for m in mons])
    return o, mons, snaps


@pytest.mark.parametrize('spec', HZ_CASES, ids=[c['name'] for c in HZ_CASES])
def test_hz_oracle_matches_reference_fields_and_spectra(spec):
    g = np.load(os.path.join(GOLDEN, f"{spec['name']}.npz"))
    o, mons, snaps = _run_oracle(spec)
    assert int(g['n_step']) == o.n_step
    assert int(g['sample_interval']) == o.sample_interval
    for cp, (fields, spectra) in snaps.items():
        for name, arr in fields.items():
            assert _digest(arr) == str(g[f'sha_{name}_{cp}']), f'{name} at step {cp}'
            if f'{name}_{cp}' in g:
                np.testing.assert_array_equal(arr, g[f'{name}_{cp}'])
        for k, (e, h, flux) in enumerate(spectra):
            np.testing.assert_array_equal(e, g[f'spec_e{k}_{cp}'])
            np.testing.assert_array_equal(h, g[f'spec_h{k}_{cp}'])
            np.testing.assert_array_equal(flux, g[f'flux{k}_{cp}'])


@pytest.mark.parametrize('spec', HZ_CASES, ids=[c['name'] for c in HZ_CASES])
def test_hz_oracle_matches_reference_setup(spec):
    g = np.load(os.path.join(GOLDEN, f"{spec['name']}.npz"))
    o = OracleHz2D(**_oracle_kwargs(spec))
    mons = apply_ops(o, spec)
    o.finalize()
    assert (o.domain.nx, o.domain.ny) == (int(g['nx']), int(g['ny']))
    assert o.domain.dt == g['dt']
    for name in ('ca_x', 'cb_x', 'ca_y', 'cb_y', 'da', 'db'):
        np.testing.assert_array_equal(getattr(o, name), g[name], err_msg=name)
    for name in ('inv_dx_e', 'inv_dx_h', 'inv_dy_e', 'inv_dy_h'):
        np.testing.assert_array_equal(o.curl[name], g[name], err_msg=name)
    for k, src in enumerate(o.sources):
        np.testing.assert_array_equal(src.profile, g[f'profile{k}'])
        line = g[f'source_line{k}']
        assert (0 if src.axis == 'x' else 1, src.position) == (int(line[0]), int(line[1]))
    for side_index, side in enumerate(o.cpml_sides):
        for kind in ('e', 'h'):
            np.testing.assert_array_equal(getattr(side, f'b_{kind}'), g[f'cpml{side_index}_{kind}_b'])
            np.testing.assert_array_equal(getattr(side, f'a_{kind}'), g[f'cpml{side_index}_{kind}_a'])
            np.testing.assert_array_equal(getattr(side, f'inv_{kind}'), g[f'cpml{side_index}_{kind}_inv'])
    for k, mon in enumerate(mons):
        info = g[f'monitor{k}']
        assert (0 if mon.normal_axis == 'x' else 1, mon.position, mon.lo, mon.hi) == tuple(int(v) for v in info)


def test_face_shares_uniform_is_exact_half():
    lo, up = face_shares(np.full(7, 2.5e-8), False, np.float32)
    assert np.all(lo == np.float32(0.5)) and np.all(up == np.float32(0.5))


def test_face_coefficients_open_axis_last_face_uses_own_cell():
    """On an open axis the last face pairs a cell with itself; on a periodic one with row 0."""
    eps = np.ones((4, 5), np.float32)
    eps[:, -1] = 4.0
    eps[-1, :] = 9.0
    widths = (np.full(4, 1e-8), np.full(5, 1e-8))
    zero = np.zeros_like(eps)
    dt = np.float32(1e-17)
    _, cb_x_open, _, cb_y_open = e_face_coefficients(eps, eps, zero, widths, False, False, dt, np.float32)
    _, cb_x_per, _, cb_y_per = e_face_coefficients(eps, eps, zero, widths, True, True, dt, np.float32)
    assert cb_x_open[0, -1] == cb_x_open[1, -1] and cb_x_open[0, -1] < cb_x_per[0, -1]   # 4 vs mean(4, 1)
    assert cb_y_open[-1, 0] < cb_y_per[-1, 0]                                            # 9 vs mean(9, 1)


def test_sheet_on_outer_wall_is_refused():
    o = OracleHz2D(1.0e-6, 1.0e-6, 25e-9, npml=0, boundaries='periodic_x')
    with pytest.raises(ValueError):
        o.add_line_source('x', 0.999e-6, wavelength=700e-9)   # y is open: its last cell's hi face is the wall
    o.add_line_source('y', 0.999e-6, wavelength=700e-9)       # x is periodic: the face wraps to row 0
    assert len(o.sources) == 1
