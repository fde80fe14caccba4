"""The B200 engine's host-side H_z setup against the oracle and the golden fixtures on the CPU: grid and dt, curl
spacings, CPML rows, face shares, calibrated tangential sheet profiles, DFT sample interval, flux lines and their
sign, the wall refusal.  No device is touched."""
import os

import numpy as np
import pytest

from cases import apply_ops
from cases_hz import HZ_CASES
from oracle.hz2d import OracleHz2D

import opensol_b200 as ob
from opensol_b200.boundaries import face_shares

GOLDEN = os.path.join(os.path.dirname(__file__), 'golden')


def _oracle_kwargs(spec):
    return {k: v for k, v in spec['sim'].items() if k != 'polarization'}


def _pair(spec):
    sim = ob.Simulation(**spec['sim'], verbose=False)
    apply_ops(sim, spec)
    sim.em.finalize_host()
    o = OracleHz2D(**_oracle_kwargs(spec))
    apply_ops(o, spec)
    o.finalize()
    return sim, o


@pytest.mark.parametrize('spec', HZ_CASES, ids=[c['name'] for c in HZ_CASES])
def test_hz_setup_matches_oracle_and_reference(spec):
    sim, o = _pair(spec)
    g = np.load(os.path.join(GOLDEN, f"{spec['name']}.npz"))
    eng = sim.em.engine
    assert eng.polarization == 'hz'
    assert (eng.nx, eng.ny) == (o.domain.nx, o.domain.ny)
    assert eng.dt == o.domain.dt == g['dt']
    for name, values in eng.rows.curl.items():
        np.testing.assert_array_equal(values, g[name])
    for k, (mine, ref) in enumerate(zip(eng.rows.sides, o.cpml_sides)):
        for attr in ('b_e', 'a_e', 'inv_e', 'b_h', 'a_h', 'inv_h'):
            np.testing.assert_array_equal(getattr(mine, attr), getattr(ref, attr))
    for k, (mine, ref) in enumerate(zip(sim.em.sources, o.sources)):
        assert (mine.axis, mine.position, mine.span) == (ref.axis, ref.position, (ref.lo, ref.hi))
        np.testing.assert_array_equal(mine.profile, g[f'profile{k}'])
    assert eng.sample_interval == o.sample_interval == int(g['sample_interval'])
    for k, (mine, ref) in enumerate(zip(sim.em.monitors, o.monitors)):
        assert (mine.axis, mine.position, mine.span) == (ref.normal_axis, ref.position, (ref.lo, ref.hi))
        assert mine._flux_sign == ref.flux_sign
    for name in ('eps_xx', 'eps_yy'):
        np.testing.assert_array_equal(sim.domain.materials.array(name), getattr(o, name))
    widths_x, widths_y = sim.domain.kernel_widths()
    for mine, ref in zip(eng.shares_x + eng.shares_y,
                         face_shares(widths_x, o.domain.periodic_x) + face_shares(widths_y, o.domain.periodic_y)):
        np.testing.assert_array_equal(mine, ref)


def test_hz_flux_signs():
    sim = ob.Simulation(1e-6, 1e-6, 25e-9, npml=8, polarization='hz', verbose=False)
    mx = sim.add_flux_monitor('y', 0.5e-6, (0.1e-6, 0.9e-6), wavelengths=[700e-9])   # normal x: S_x = +E_y H_z
    my = sim.add_flux_monitor('x', 0.5e-6, (0.1e-6, 0.9e-6), wavelengths=[700e-9])   # normal y: S_y = -E_x H_z
    assert (mx.axis, mx._flux_sign) == ('x', 1.0)
    assert (my.axis, my._flux_sign) == ('y', -1.0)
    ez = ob.Simulation(1e-6, 1e-6, 25e-9, npml=8, verbose=False)
    assert ez.add_flux_monitor('y', 0.5e-6, (0.1e-6, 0.9e-6), wavelengths=[700e-9])._flux_sign == -1.0


def test_hz_sheet_on_the_last_cell_of_a_periodic_axis_wraps():
    """A sheet on the hi face of the last cell is refused only on an open axis (the outer wall); a CPML axis never
    places a line there (the window ends npml cells earlier) and a periodic one wraps to row 0."""
    sim = ob.Simulation(1e-6, 1e-6, 25e-9, npml=0, boundaries='periodic', polarization='hz', verbose=False)
    for axis in ('x', 'y'):
        src = sim.add_line_source(axis, 0.999e-6, wavelength=700e-9)
        assert src.position == 39
    sim.em.finalize_host()
    assert all(np.all(np.isfinite(s.profile)) and np.all(s.profile > 0) for s in sim.em.sources)


def test_hz_dielectric_writes_both_permittivities_and_not_eps_r():
    sim = ob.Simulation(1e-6, 1e-6, 25e-9, npml=8, polarization='hz', verbose=False)
    sim.add_dielectric_rectangle(0.2e-6, 0.2e-6, 0.5e-6, 0.5e-6, eps_r=3.0)
    m = sim.domain.materials
    assert m.array('eps_xx').max() == np.float32(3.0) and m.array('eps_yy').max() == np.float32(3.0)
    assert m.array('eps_r').max() == np.float32(1.0)
    assert sim.em.permittivity_arrays == ('eps_xx', 'eps_yy')


def test_hz_engine_refuses_blocked_kernel_calls():
    sim = ob.Simulation(1e-6, 1e-6, 25e-9, npml=8, polarization='hz', verbose=False)
    with pytest.raises(NotImplementedError):
        sim.em.engine.autotune()
    with pytest.raises(NotImplementedError):
        sim.em.engine.plan_info()
