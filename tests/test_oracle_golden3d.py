"""Pin the 3D oracle to open_sol's em_fdtd_3d engine: against the fixtures of tests/golden/make_golden3d.py the
oracle must reproduce the setup rows exactly and the reference's numpy twins bit for bit (SHA-256 of all six fields at
every checkpoint, of every monitor's complex128 spectra, and the fluxes), and its default numba twins within float32
rounding (they evaluate the coefficients in float64)."""
import hashlib
import os

import numpy as np
import pytest

from cases3d import CASES3D, DX, boundary_faces, paint, window_size
from oracle.fdtd3d import OracleEM3D

GOLDEN = os.path.join(os.path.dirname(__file__), 'golden')
FIELDS = ('ex', 'ey', 'ez', 'hx', 'hy', 'hz')
# numba twins vs float32 arithmetic: fields relative to the run's peak |E| (or |H|), fluxes relative
NUMBA_FIELD_RTOL = 1e-5
NUMBA_FLUX_RTOL = 1e-5


def _digest(a):
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


def build_oracle(spec):
    sx, sy, sz = window_size(spec)
    o = OracleEM3D(sx, sy, sz, DX, faces=boundary_faces(spec), npml=spec['npml'])
    for name, values in paint(spec).items():
        o.materials[name] = values.copy()
    d = spec['dipole']
    o.add_dipole(*(f * s for f, s in zip(d['at'], (sx, sy, sz))), orientation=d['orientation'],
                 dipole_moment=d['moment'], wavelength=d['wavelength'], bandwidth=d['bandwidth'])
    if spec['flux_box'] is not None:
        b = spec['flux_box']
        o.add_flux_box(tuple(f * s for f, s in zip(b['lo'], (sx, sy, sz))),
                       tuple(f * s for f, s in zip(b['hi'], (sx, sy, sz))), b['wavelengths'])
    for p in spec['flux_planes']:
        size = {'x': sx, 'y': sy, 'z': sz}[p['normal']]
        o.add_flux_plane(p['normal'], p['at'] * size, p['wavelengths'])
    o.finalize()
    return o


def _planes(monitor):
    return monitor.planes() if hasattr(monitor, 'planes') else [monitor]


@pytest.fixture(scope='module', params=[c['name'] for c in CASES3D])
def case(request):
    spec = next(c for c in CASES3D if c['name'] == request.param)
    return spec, np.load(os.path.join(GOLDEN, f"{spec['name']}.npz"))


def test_setup_rows(case):
    spec, g = case
    o = build_oracle(spec)
    assert tuple(o.shape) == tuple(g['shape'])
    assert np.float32(o.dt) == g['dt']
    assert int(o.monitors[0].sample_interval) == int(g['sample_interval'])
    assert _digest(o.material_id) == str(g['sha_material_id'])
    for name in ('table_eps_z', 'table_sigma', 'table_mu', 'table_sigma_m'):
        mine = {'table_eps_z': o.t_ez, 'table_sigma': o.t_sig, 'table_mu': o.t_mu, 'table_sigma_m': o.t_sm}[name]
        np.testing.assert_array_equal(mine, g[name])
    for axis in range(3):
        np.testing.assert_array_equal(o.inv_e[axis], g[f'inv_e{axis}'])
        np.testing.assert_array_equal(o.inv_h[axis], g[f'inv_h{axis}'])
    keys = sorted(k[:-8] for k in g.files if k.startswith('cpml_') and k.endswith('_row_map'))
    assert keys == sorted(f'cpml_{axis}{kind}' for axis, kind in o.layers)
    for (axis, kind), layer in o.layers.items():
        key = f'cpml_{axis}{kind}'
        np.testing.assert_array_equal(layer['row_map'], g[key + '_row_map'])
        np.testing.assert_array_equal(layer['b'], g[key + '_b'])
        np.testing.assert_array_equal(layer['gain'], g[key + '_gain'])
    src = o.sources[0]
    assert tuple(src['cell']) == tuple(g['dipole_cell'])
    assert src['volume'] == float(g['dipole_volume'])
    assert np.float32(src['weight']) == g['dipole_weight'][0]
    for k, monitor in enumerate(o.monitors):
        np.testing.assert_array_equal(monitor.frequencies, g[f'monitor{k}_frequencies'])
        planes = np.asarray([(p.normal_axis, p.edge, *sum(p.bounds, ())) for p in _planes(monitor)])
        np.testing.assert_array_equal(planes, g[f'monitor{k}_planes'])


def test_fields_spectra_fluxes(case):
    spec, g = case
    o = build_oracle(spec)
    done = 0
    peak = {'e': 0.0, 'h': 0.0}
    for cp in spec['checkpoints']:
        for _ in range(cp - done):
            o.run(1)
            for name in FIELDS:
                peak[name[0]] = max(peak[name[0]], float(np.abs(o.fields[name]).max()))
        done = cp
        for name in FIELDS:
            arr = o.fields[name]
            # bit for bit against the numpy twins
            assert _digest(arr) == str(g[f'numpy_sha_{name}_{cp}']), (name, cp)
            # the numba twins (float64 coefficients) within 1e-5 of the run's peak field of the same kind
            for plane in ('xmid', 'zmid'):
                ref = g[f'numba_{name}_{plane}_{cp}']
                mine = arr[arr.shape[0] // 2] if plane == 'xmid' else arr[:, :, arr.shape[2] // 2]
                assert np.abs(mine - ref).max() <= NUMBA_FIELD_RTOL * peak[name[0]], (name, plane, cp)
        for k, monitor in enumerate(o.monitors):
            flux = monitor.flux()
            np.testing.assert_array_equal(flux, g[f'numpy_flux{k}_{cp}'])
            spectra = np.concatenate([s.reshape(-1) for s in monitor.spectra()])
            assert _digest(spectra) == str(g[f'numpy_sha_spectra{k}_{cp}'])
            np.testing.assert_allclose(flux, g[f'numba_flux{k}_{cp}'], rtol=NUMBA_FLUX_RTOL, atol=0)
    assert o.n_step == int(g['numpy_n_step'])
    assert o.time == float(g['numpy_time'])
