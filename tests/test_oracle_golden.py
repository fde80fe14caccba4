"""Pin the oracle to open_sol itself: every golden fixture (generated by running the reference's CPU backend, see
tests/golden/make_golden.py) must be reproduced bit for bit -- fields at every checkpoint (SHA-256 and stored
arrays), complex128 line spectra, fluxes and the setup rows."""
import hashlib
import os

import numpy as np
import pytest

from cases import CASES, apply_ops
from oracle.fdtd2d import FACES, OracleEz2D

GOLDEN = os.path.join(os.path.dirname(__file__), 'golden')


def _digest(a):
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


def _golden(name):
    return np.load(os.path.join(GOLDEN, f'{name}.npz'))


def _run_oracle(spec, precision='single'):
    o = OracleEz2D(**spec['sim'], precision=precision)
    mons = apply_ops(o, spec)
    snaps = {}
    done = 0
    for cp in spec['checkpoints']:
        o.run(n_steps=cp - done)
        done = cp
        snaps[cp] = ({n: getattr(o, n).copy() for n in ('ez', 'hx', 'hy')},
                     [(m.e_acc.copy(), m.h_acc.copy(), m.flux()) for m in mons])
    return o, mons, snaps


@pytest.mark.parametrize('spec', CASES, ids=[c['name'] for c in CASES])
def test_oracle_matches_reference_fields_and_spectra(spec):
    g = _golden(spec['name'])
    o, mons, snaps = _run_oracle(spec)
    assert int(g['n_step']) == o.n_step
    assert float(g['time']) == o.time
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


@pytest.mark.parametrize('spec', CASES, ids=[c['name'] for c in CASES])
def test_oracle_matches_reference_setup(spec):
    g = _golden(spec['name'])
    o = OracleEz2D(**spec['sim'])
    apply_ops(o, spec)
    o.finalize()
    assert (o.domain.nx, o.domain.ny) == (int(g['nx']), int(g['ny']))
    assert o.domain.dt == g['dt']
    np.testing.assert_array_equal(o.cb, g['cb'])
    np.testing.assert_array_equal(o.ca, g['ca'])
    for name in ('inv_dx_e', 'inv_dx_h', 'inv_dy_e', 'inv_dy_h'):
        np.testing.assert_array_equal(o.curl[name], g[name])
    for k, src in enumerate(o.sources):
        np.testing.assert_array_equal(src.profile, g[f'profile{k}'])
    for side_index, side in enumerate(o.cpml_sides):
        for kind in ('e', 'h'):
            np.testing.assert_array_equal(getattr(side, f'b_{kind}'), g[f'cpml{side_index}_{kind}_b'])
            np.testing.assert_array_equal(getattr(side, f'a_{kind}'), g[f'cpml{side_index}_{kind}_a'])
            np.testing.assert_array_equal(getattr(side, f'inv_{kind}'), g[f'cpml{side_index}_{kind}_inv'])


def test_oracle_float64_stepper_matches_reference_double():
    spec = CASES[0]
    g = _golden('c1')
    o, mons, snaps = _run_oracle(spec, 'double')
    for cp, (fields, spectra) in snaps.items():
        for name, arr in fields.items():
            assert _digest(arr) == str(g[f'f64_sha_{name}_{cp}'])
        for k, (e, h, flux) in enumerate(spectra):
            np.testing.assert_array_equal(e, g[f'f64_spec_e{k}_{cp}'])
            np.testing.assert_array_equal(flux, g[f'f64_flux{k}_{cp}'])


def test_oracle_duration_tick_count():
    """Simulation.run(duration=80 fs) stops after 1370 ticks (the runner's t < t_end - dt/2 rule)."""
    spec = CASES[0]
    g = _golden('c1')
    o = OracleEz2D(**spec['sim'])
    assert o.steps_for_duration(spec['duration']) == int(g['duration_steps']) == 1370


def test_oracle_thread_count_does_not_change_results(monkeypatch):
    """Rows are parallelised with OpenMP; each cell of a half step is independent, so 1 thread equals many."""
    import subprocess
    import sys
    import json
    code = ("import sys, json, hashlib; sys.path.insert(0, %r); sys.path.insert(0, %r);"
            "from cases import case, apply_ops; from oracle.fdtd2d import OracleEz2D;"
            "s = case('two_sources'); o = OracleEz2D(**s['sim']); apply_ops(o, s); o.run(n_steps=120);"
            "print(hashlib.sha256(o.ez.tobytes()).hexdigest())") % (os.path.dirname(GOLDEN), GOLDEN)
    outs = []
    for threads in ('1', '4'):
        env = dict(os.environ, OMP_NUM_THREADS=threads)
        outs.append(subprocess.run([sys.executable, '-c', code], env=env, capture_output=True, text=True,
                                   check=True).stdout.strip())
    assert outs[0] == outs[1]


def test_flux_sign_and_faces_constant():
    assert FACES == ('x_lo', 'x_hi', 'y_lo', 'y_hi')
