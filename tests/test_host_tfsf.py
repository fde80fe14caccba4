"""Host side of the TFSF plane-wave box (no GPU): the box checks, and the incident line's parameters (side and line
coefficients, Mur ends, source scale) equal to the oracle's restatement of open_sol's _PlaneWaveBox, which the
golden fixtures tests/golden/tfsf_*.npz pin to the reference."""
import numpy as np
import pytest

from cases_dft import case
from oracle.fdtd2d import OracleEz2D

import opensol_b200 as ob


def _boxes(spec):
    sim = ob.Simulation(**spec['sim'], verbose=False)
    o = OracleEz2D(**spec['sim'])
    for method, args, kwargs in spec['ops']:
        if method == 'add_tfsf':
            return getattr(sim.em, method)(*args, **kwargs), getattr(o, method)(*args, **kwargs)
    raise AssertionError('no TFSF box in the case')


@pytest.mark.parametrize('name', ['tfsf_cylinder', 'tfsf_periodic_y'])
def test_tfsf_parameters_match_oracle(name):
    src, box = _boxes(case(name))
    assert (src.x0, src.x1, src.y0, src.y1) == box.cells
    assert src.aux_x0 == box.aux_x0 and src.AUX_SOURCE_INDEX == box.source_index
    assert src.aux_cells == box.aux_ez.size
    assert src.coef_h == tuple(box.coef_h) and src.coef_e == tuple(box.coef_e) and src.mur == box.mur
    np.testing.assert_array_equal(src.aux_coef_h, box.aux_coef_h)
    np.testing.assert_array_equal(src.aux_coef_e, box.aux_coef_e)
    assert src.source_scale == box.scale
    t = np.linspace(0.0, 4e-14, 7)
    np.testing.assert_array_equal(src.values(t), [np.float32(box.scale * box.temporal(float(x))) for x in t])


def test_tfsf_box_must_keep_a_scattered_ring_inside_the_window():
    sim = ob.Simulation(size_x=1.0e-6, size_y=1.0e-6, dx=25e-9, npml=10, boundaries='pml', verbose=False)
    with pytest.raises(ValueError, match='scattered-field'):
        sim.em.add_tfsf(0.0, 0.2e-6, 0.5e-6, 0.8e-6, wavelength=700e-9)
    hz = ob.Simulation(size_x=1.0e-6, size_y=1.0e-6, dx=25e-9, npml=10, boundaries='pml', polarization='hz',
                       verbose=False)
    with pytest.raises(ValueError, match='scattered-field'):
        hz.em.add_tfsf(0.2e-6, 0.0, 0.8e-6, 0.8e-6, wavelength=700e-9)


@pytest.mark.parametrize('params', [(8e15, 5e13, 2.0), (1.37e16, 1e14, 1.0)])
def test_drude_coefficients_match_oracle(params):
    from oracle.fdtd2d import OracleDrude
    dt = 5.8377e-17
    damping, drive = ob.DrudePole(*params).ade_coefficients(dt)
    o_damping, _, o_drive = OracleDrude(*params).coefficients(dt)
    assert (damping, drive) == (o_damping, o_drive)
    assert ob.DrudePole(*params).susceptibility(2.3e15) == OracleDrude(*params).susceptibility(2.3e15)


def test_lorentz_coefficients_match_oracle():
    from oracle.fdtd2d import OracleLorentz
    dt = 5.8377e-17
    assert ob.LorentzPole(1.5, 3e15, 2e14).ade_coefficients(dt) == OracleLorentz(1.5, 3e15, 2e14).coefficients(dt)


def test_unstable_drude_is_refused():
    sim = ob.Simulation(size_x=1.0e-6, size_y=1.0e-6, dx=25e-9, npml=10, boundaries='pml', verbose=False)
    sim.em.add_drude_rectangle(0.3e-6, 0.3e-6, 0.6e-6, 0.6e-6, ob.DrudePole(1.37e16, 1e14, 1.0))
    sim.em.add_line_source('y', 0.2e-6, wavelength=700e-9)
    with pytest.raises(ValueError, match='unstable'):
        sim.em.finalize_host()


@pytest.mark.parametrize('periodic', [False, True])
def test_hz_pole_face_sets_match_oracle(periodic):
    """The H_z engine's pole face sets (face-averaged cell masks on E_x / E_y, boxed on positive weights) equal the
    oracle's, including the faces below / left of the mask, a wrapped partner on a periodic y axis and graded shares."""
    from oracle.hz2d import OracleHz2D
    from oracle.fdtd2d import OracleDrude
    from opensol_b200.boundaries import face_shares
    from opensol_b200.poles import pole_face_sets
    o = OracleHz2D(1.2e-6, 1.0e-6, 25e-9, npml=8, boundaries='periodic_y' if periodic else 'pml')
    d = o.domain
    mask = np.zeros((d.nx, d.ny), dtype=bool)
    mask[20:31, 0:6] = True            # touches the y = 0 edge: its E_x partner faces wrap on a periodic axis
    mask[25:29, d.ny - 3:] = True      # and the last column
    mask[40:44, 15:22] = True
    o.add_dispersive(OracleDrude(8e15, 5e13), mask)
    shares_x = face_shares(d.kernel_widths[0], d.periodic_x)
    shares_y = face_shares(d.kernel_widths[1], d.periodic_y)
    sets = pole_face_sets(mask, shares_x, shares_y, d.periodic_x, d.periodic_y)
    assert [(c, b) for c, b, _ in sets] == [(f[1], f[2]) for f in o.pole_faces]
    for (_, _, weight), face in zip(sets, o.pole_faces):
        assert weight.dtype == np.float32
        np.testing.assert_array_equal(weight, face[3])
    assert sets[1][1][0].start == 19   # the E_y faces below the mask's first row carry weight too
