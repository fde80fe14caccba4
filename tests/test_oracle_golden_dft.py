"""Pin the oracle's field-map (running DFT) monitors, field probes, TFSF boxes and dispersive poles to open_sol itself: the fixtures of
tests/golden/dft_*.npz (generated by running the reference's CPU backend, see tests/golden/make_golden_dft.py) must be
reproduced bit for bit -- the complex64 maps at every checkpoint (E_z; H_z with E_x / E_y at the cell centres), the
sample boxes, the flux line spectra, the fields' digests and the probes' times and values."""
import hashlib
import os

import numpy as np
import pytest

from cases import apply_ops
from cases_dft import CASES_DFT, CASES_DFT_HZ, apply_poles
from oracle.fdtd2d import OracleDrude, OracleEz2D, OracleLorentz, circle_mask
from oracle.hz2d import OracleHz2D

GOLDEN = os.path.join(os.path.dirname(__file__), 'golden')
ALL_CASES = CASES_DFT + CASES_DFT_HZ


def _digest(a):
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


def is_hz(spec):
    return spec['sim'].get('polarization', 'ez') == 'hz'


def map_parts(mon):
    """The map arrays of a monitor: (ez_dft,) or (hz_dft, ex_dft, ey_dft)."""
    return (mon.ez_dft,) if mon.polarization == 'ez' else (mon.hz_dft, mon.ex_dft, mon.ey_dft)


def map_keys(spec, k, cp):
    """Fixture keys of map k at checkpoint cp, in map_parts order."""
    if not is_hz(spec):
        return (f'map{k}_{cp}',)
    return tuple(f'map{k}_{part}_{cp}' for part in ('hz', 'ex', 'ey'))


def field_names(spec):
    return ('hz', 'ex', 'ey') if is_hz(spec) else ('ez', 'hx', 'hy')


def run_oracle_dft(spec):
    """(oracle, maps, {checkpoint: ([map part tuples], [flux E spectra], {field: digest})}) of a case."""
    sim = dict(spec['sim'])
    sim.pop('polarization', None)
    o = (OracleHz2D if is_hz(spec) else OracleEz2D)(**sim)
    fluxes = apply_ops(o, spec)
    apply_poles(o, spec, OracleDrude, OracleLorentz, lambda cx, cy, r: circle_mask(o.domain, cx, cy, r))
    maps = [o.add_dft_monitor(x0, y0, x1, y1, frequencies=f, downsample=ds) for x0, y0, x1, y1, f, ds in spec['dft']]
    for mon in maps:
        mon.polarization = 'hz' if is_hz(spec) else 'ez'
    o.probe_records = [o.add_field_probe(x, y, comp) for x, y, comp in spec.get('probes', [])]
    snaps = {}
    done = 0
    for cp in spec['checkpoints']:
        o.run(n_steps=cp - done)
        done = cp
        snaps[cp] = ([tuple(a.copy() for a in map_parts(m)) for m in maps], [m.e_acc.copy() for m in fluxes],
                     {n: _digest(getattr(o, n)) for n in field_names(spec)})
    return o, maps, snaps


@pytest.mark.parametrize('spec', ALL_CASES, ids=[c['name'] for c in ALL_CASES])
def test_oracle_maps_match_reference(spec):
    g = np.load(os.path.join(GOLDEN, f"{spec['name']}.npz"))
    o, maps, snaps = run_oracle_dft(spec)
    assert int(g['sample_interval']) == o.sample_interval
    for k, mon in enumerate(maps):
        xs, ys = mon.x_samples, mon.y_samples
        shape = map_parts(mon)[0].shape
        assert [xs.start, xs.stop, mon.downsample, shape[1], ys.start, ys.stop, shape[2]] == g[f'map{k}_box'].tolist()
    for cp, (spectra, flux_e, digests) in snaps.items():
        for name, d in digests.items():
            assert d == str(g[f'sha_{name}_{cp}']), f'{name} at step {cp}'
        for k, parts in enumerate(spectra):
            for got, key in zip(parts, map_keys(spec, k, cp)):
                ref = g[key]
                assert ref.dtype == np.complex64 and got.shape == ref.shape
                np.testing.assert_array_equal(got, ref)
            # the map saw the pulse (a part may stay zero: E_x of a y-invariant E_y wave)
            assert max(np.abs(g[key]).max() for key in map_keys(spec, k, cp)) > 0
        for k, e in enumerate(flux_e):
            np.testing.assert_array_equal(e, g[f'spec_e{k}_{cp}'])


@pytest.mark.parametrize('spec', ALL_CASES, ids=[c['name'] for c in ALL_CASES])
def test_oracle_probes_match_reference(spec):
    g = np.load(os.path.join(GOLDEN, f"{spec['name']}.npz"))
    o, _, _ = run_oracle_dft(spec)
    for k, (ix, iy, _, times, values) in enumerate(o.probe_records):
        assert [ix, iy] == g[f'probe{k}_cell'].tolist()
        np.testing.assert_array_equal(np.array(times), g[f'probe{k}_t'])
        np.testing.assert_array_equal(np.array(values, dtype=np.float32), g[f'probe{k}_v'])
        assert np.abs(g[f'probe{k}_v']).max() > 0
