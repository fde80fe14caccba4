"""The ModelSpec hook (opensol_b200.modelspec) inside open_sol's own model builder, on the CPU.

A config-1 model (6 x 3 um window at 25 nm, CPML 15 on x, periodic y, an eps_r 2.25 slab, a 600 nm line source, a
two-wavelength flux line; open_sol's README example) is written with open_sol's ModelSpec schema and built by its
builder (open_sol/model/builder.py) twice: with the stepper role assigned to a ``b200_kernels`` node, the built
physics is this package's EMPhysics, and its setup -- grid, dt, the eps_r array the builder painted, the calibrated
source profile, the DFT sample interval, the monitor's cells and frequencies -- equals the oracle's for the same case
bit for bit; with the default stepper the physics stays open_sol's own.  The device engine is not created (no GPU
here): the engine's device synchronisation is replaced by a no-op for the build.

open_sol is imported from its installed copy under baseline/_ref (pip install --target, no dependencies); the test
is skipped where that copy is absent.
"""
import os
import sys
import tempfile

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
REF = os.path.join(ROOT, 'baseline', '_ref')


@pytest.fixture(scope='module')
def open_sol():
    if not os.path.isdir(os.path.join(REF, 'open_sol')):
        pytest.skip('open_sol is not installed under baseline/_ref')
    os.environ.setdefault('NUMBA_CACHE_DIR', os.path.join(tempfile.gettempdir(), 'opensol_numba_cache'))
    if REF not in sys.path:
        sys.path.append(REF)
    import open_sol
    return open_sol


def _spec(open_sol, b200):
    from open_sol.model.spec import (DomainSpec, FeatureSpec, GeometrySpec, MaterialSpec, MeshSpec, ModelSpec,
                                     PhysicsSpec, SolverSpec, StudySpec)
    physics = PhysicsSpec('em', 'em_fdtd_ez', settings={'bc_y_lo': 'periodic', 'bc_y_hi': 'periodic',
                                                        'pml_cells': 15}, features=[
        FeatureSpec('source', 'line_source', ['source_line'],
                    {'waveform': 'gaussian', 'wavelength': 600e-9, 'bandwidth': 0.8, 'amplitude': 1.0}),
        FeatureSpec('flux', 'flux_monitor', ['flux_line'],
                    {'wavelength_start': 500e-9, 'wavelength_stop': 600e-9, 'n_wavelengths': 2})])
    spec = ModelSpec(
        title='config 1',
        domain=DomainSpec(size_x=6e-6, size_y=3e-6),
        geometry=[GeometrySpec('slab', 'rectangle', {'x0': 2.75e-6, 'y0': 0.0, 'x1': 3.25e-6, 'y1': 3e-6}),
                  GeometrySpec('source_line', 'line', {'x0': 1.2e-6, 'y0': 0.0, 'x1': 1.2e-6, 'y1': 3e-6}),
                  GeometrySpec('flux_line', 'line', {'x0': 4.5e-6, 'y0': 0.0, 'x1': 4.5e-6, 'y1': 3e-6})],
        materials=[MaterialSpec('slab', properties={'eps_r': 2.25}, selection=['slab'])],
        physics=[physics],
        meshes=[MeshSpec(mode='uniform', dx=25e-9)],
        study=StudySpec(type='time_dependent', settings={'duration': 80e-15}))
    spec.solver_defaults.backend = 'cpu'
    if b200:
        spec.solvers.append(SolverSpec('b200', 'b200_kernels', {'precision': 'single'}))
        physics.solvers['stepper'] = 'b200'
    return spec


def _oracle():
    from oracle.fdtd2d import OracleEz2D
    o = OracleEz2D(6e-6, 3e-6, 25e-9, npml=15, boundaries='periodic_y')
    o.add_dielectric_rectangle(2.75e-6, 0.0, 3.25e-6, 3e-6, eps_r=2.25)
    o.add_line_source('y', 1.2e-6, wavelength=600e-9, bandwidth=0.8, amplitude=1.0)
    o.add_flux_monitor('y', 4.5e-6, (0.0, 3e-6), wavelengths=[500e-9, 600e-9])
    o.finalize()
    return o


def test_b200_stepper_builds_this_engine_with_the_oracle_setup(open_sol, monkeypatch):
    from open_sol.model.builder import build
    from open_sol.model.schema import get_registry
    import opensol_b200 as ob
    from opensol_b200 import modelspec
    from opensol_b200.engine2d import FDTDEngine2D_Ez
    registry = modelspec.install(get_registry())
    assert modelspec.install(registry) is registry                      # idempotent
    assert registry.solver_type('b200_kernels').precisions == ('single',)
    monkeypatch.setattr(FDTDEngine2D_Ez, 'sync_device', lambda self: None)   # no device here
    session = build(_spec(open_sol, b200=True), registry)
    em = session.sim.runner.physics['em']
    assert isinstance(em, ob.EMPhysics)
    o = _oracle()
    assert (em.engine.nx, em.engine.ny) == (o.domain.nx, o.domain.ny) == (270, 120)
    assert np.float32(em.engine.dt) == np.float32(o.domain.dt)
    np.testing.assert_array_equal(em.domain.materials.array('eps_r'), o.eps_r)
    (source,) = em.sources
    np.testing.assert_array_equal(source.profile, o.sources[0].profile)
    assert (source.axis, source.position, source.span) == ('y', o.sources[0].position,
                                                          (o.sources[0].lo, o.sources[0].hi))
    (monitor,) = [m for m in em.monitors if hasattr(m, 'frequencies')]
    assert monitor.sample_interval == o.sample_interval == 6
    np.testing.assert_array_equal(monitor.frequencies, o.monitors[0].frequencies)
    assert (monitor.position, monitor.span) == (o.monitors[0].position, (o.monitors[0].lo, o.monitors[0].hi))


def test_default_stepper_keeps_open_sols_engine(open_sol):
    from open_sol.model.builder import build
    from open_sol.model.schema import get_registry
    import opensol_b200 as ob
    from opensol_b200 import modelspec
    registry = modelspec.install(get_registry())
    session = build(_spec(open_sol, b200=False), registry)
    em = session.sim.runner.physics['em']
    assert not isinstance(em, ob.EMPhysics)
    assert type(em).__module__.startswith('open_sol.')


def test_double_precision_is_refused(open_sol):
    from open_sol.model.builder import build
    from open_sol.model.schema import get_registry
    from opensol_b200 import modelspec
    registry = modelspec.install(get_registry())
    spec = _spec(open_sol, b200=True)
    spec.solvers[-1].settings['precision'] = 'double'
    with pytest.raises(Exception, match='single|precision'):
        build(spec, registry)
