"""Hook of this engine into open_sol's ModelSpec path (``open_sol.api.run(spec)``, the CLI, studies): the physics
types em_fdtd_ez, em_fdtd_hz and em_fdtd_3d step on the B200 when a spec assigns their 'stepper' solver role to a
solver node of type ``b200_kernels``.

open_sol builds a physics by calling its PhysicsType's ``create(ctx, physics_spec, settings)``
(open_sol/model/builder.py:761-777); for these types that is create_em_physics (open_sol/physics/em/
definition_common.py:997-1006, bound in definition_fdtd.py:444-466) or _create (open_sol/physics/em3d/
definition.py:234-241), which read the stepper's precision from ``ctx.solvers(name)['stepper']``.  ``install``
registers the solver type (a copy of open_sol's ``explicit_kernels`` -- the same 'stepper' role and settings,
single precision only) and wraps those create callbacks: when the built stepper runtime is this package's
``B200Stepper`` the wrapper returns this package's EMPhysics / EMPhysics3D on a domain of the same grid, boundary
configuration and material arrays (shared with open_sol's MaterialGrid, so every later material write the builder
makes reaches the engine); any other stepper keeps open_sol's own create.  The features then apply through the
physics methods both share (add_line_source, add_flux_monitor, add_tfsf, add_dft_monitor, add_field_probe,
add_dipole, add_flux_box, ...); a feature this engine does not build raises when it is applied.

A spec selects the engine with a solver node and an assignment::

    spec.solvers.append(SolverSpec('b200', 'b200_kernels', {'precision': 'single'}))
    spec.physics[0].solvers['stepper'] = 'b200'

Limits: uniform (cubic) Cartesian grids; stepper precision single; no absorption tracking, subpixel smoothing,
conformal boundaries, Bloch phase or half-precision storage.  Material arrays on open_sol's gpu backend (cupy) are
copied to the host once when the physics is created.
"""
from __future__ import annotations

import dataclasses

import numpy as np

from .constants import DTYPE

SOLVER_TYPE = 'b200_kernels'
PHYSICS_TYPES = {'em_fdtd_ez': 'ez', 'em_fdtd_hz': 'hz', 'em_fdtd_3d': '3d'}
_MATERIAL_NAMES_2D = ('eps_r', 'sigma_e', 'mu_r', 'sigma_m', 'eps_xx', 'eps_yy')
_MATERIAL_NAMES_3D = ('eps_r', 'sigma_e', 'mu_r', 'sigma_m', 'eps_xx', 'eps_yy')


@dataclasses.dataclass(frozen=True)
class B200Stepper:
    """Runtime of the 'stepper' role built from a ``b200_kernels`` solver node (open_sol's StepperConfig role)."""
    precision: str = 'single'
    device: int = 0

    def work_counters(self) -> dict:
        return {}


def _create_stepper(ctx, request):
    precision = request.values.get('precision', 'single')
    if precision != 'single':
        raise ValueError(f"solver '{SOLVER_TYPE}' steps float32 fields: precision must be 'single', got "
                         f"{precision!r}")
    return B200Stepper(precision='single', device=int(request.values.get('device', 0) or 0))


def install(registry=None):
    """Register the ``b200_kernels`` solver type and wrap the FDTD physics types' create callbacks in `registry`
    (default: open_sol's process-wide registry); returns the registry.  Idempotent."""
    if registry is None:
        from open_sol.model.schema import get_registry
        registry = get_registry()
    try:
        registry.solver_type(SOLVER_TYPE)
    except KeyError:
        base = registry.solver_type('explicit_kernels')
        precision = [param for param in base.params if param.name == 'precision']
        params = tuple(dataclasses.replace(param, default='single', choices=('single',),
                                           choice_labels=(('single', 'Single precision'),))
                       for param in precision)
        registry.register_solver_type(dataclasses.replace(
            base, name=SOLVER_TYPE, label='B200 FDTD kernels', params=params, precisions=('single',),
            backends=('gpu', 'cpu'), create=_create_stepper, backend_misfit=None,
            description='Hand-written sm_100a kernels of the opensol_b200 engine for em_fdtd_ez / em_fdtd_hz / '
                        'em_fdtd_3d (float32 fields, temporally blocked 2D steps, fused 3D steps); the materials '
                        'are painted on the host and uploaded once.',
            summary='Time stepping on a B200 with the opensol_b200 kernels.'))
    for name, kind in PHYSICS_TYPES.items():
        try:
            physics_type = registry.physics_type(name)
        except KeyError:
            continue
        if getattr(physics_type.create, 'b200_wrapped', False):
            continue
        registry._physics[name] = dataclasses.replace(physics_type, create=_wrap_create(physics_type.create, kind))
    return registry


def _wrap_create(original, kind):
    def create(ctx, physics_spec, settings_values):
        solvers = ctx.solvers(physics_spec.name)
        runtime = solvers.get('stepper') if hasattr(solvers, 'get') else None
        if not isinstance(runtime, B200Stepper):
            return original(ctx, physics_spec, settings_values)
        return create_physics(ctx, physics_spec, settings_values, kind, runtime)

    create.b200_wrapped = True
    create.original = original
    return create


def _host(array):
    """A host numpy view of a material array (cupy arrays are copied)."""
    if isinstance(array, np.ndarray):
        return array
    getter = getattr(array, 'get', None)
    return np.asarray(getter() if getter is not None else array)


def _require_uniform(domain):
    if getattr(domain, 'non_uniform', False):
        raise ValueError(f"solver '{SOLVER_TYPE}' runs uniform grids only (the model's mesh is graded)")
    coordinates = getattr(domain, 'coordinates', 'cartesian')
    if getattr(coordinates, 'grid', coordinates) != 'cartesian' or getattr(coordinates, 'line', False):
        raise ValueError(f"solver '{SOLVER_TYPE}' runs Cartesian grids only, got {coordinates!r}")


def _share_materials(source, target, names):
    """Point target's (this package's) MaterialGrid at source's (open_sol's) arrays of `names`."""
    owned = getattr(source, 'property_names', lambda: ())()
    for name in names:
        if name not in owned:
            continue
        array = _host(getattr(source, name))
        if array.dtype != DTYPE or array.shape != target.shape:
            raise ValueError(f"material array '{name}' is {array.dtype} {array.shape}, the engine needs float32 "
                             f"{target.shape}")
        target._arrays[name] = array
    target.version += 1


def _unsupported_settings(settings_values):
    if settings_values.get('track_absorption'):
        raise ValueError(f"solver '{SOLVER_TYPE}' does not track absorption (setting track_absorption)")


def create_physics(ctx, physics_spec, settings_values, kind, runtime):
    """This package's physics for one physics spec, on a domain equal to ctx.domain."""
    _unsupported_settings(settings_values)
    source = ctx.domain
    _require_uniform(source)
    if kind == '3d':
        physics = _create_3d(source, runtime)
    else:
        physics = _create_2d(source, kind, runtime)
    _write_dispersive(ctx, physics_spec, physics, kind)
    return physics


def _create_2d(source, polarization, runtime):
    from .boundaries import BoundaryConfig
    from .domain import Domain
    from .physics import EMPhysics
    ref = source.boundary_config
    bc = BoundaryConfig(ref.x_lo.value, ref.x_hi.value, ref.y_lo.value, ref.y_hi.value)
    for name in ('cpml_npml', 'cpml_order', 'cpml_sigma_factor', 'cpml_kappa_max', 'cpml_alpha_max', 'bloch_kx',
                 'bloch_ky'):
        setattr(bc, name, getattr(ref, name))
    bc._validate()
    if bc.bloch_kx or bc.bloch_ky:
        raise ValueError(f"solver '{SOLVER_TYPE}' steps real fields only (Bloch wave vector 0)")
    domain = Domain.uniform(source.size_x, source.size_y, float(source.dx), npml=bc.cpml_npml, boundary_config=bc,
                            verbose=False)
    if (domain.grid.nx, domain.grid.ny) != (source.grid.nx, source.grid.ny):
        raise ValueError(f'grid {domain.grid.nx} x {domain.grid.ny} differs from the model grid '
                         f'{source.grid.nx} x {source.grid.ny}')
    _share_materials(source.materials, domain.materials, _MATERIAL_NAMES_2D)
    return EMPhysics(domain, polarization, boundary_config=bc, precision='single', device=runtime.device)


def _create_3d(source, runtime):
    from .domain3d import BoundaryConfig3D, Domain3D
    from .physics3d import EMPhysics3D
    ref = source.boundary_config
    faces = {face: (getattr(ref, face).value if hasattr(getattr(ref, face), 'value') else getattr(ref, face))
             for face in ('x_lo', 'x_hi', 'y_lo', 'y_hi', 'z_lo', 'z_hi')}
    config = BoundaryConfig3D(faces, npml=ref.cpml_npml, order=ref.cpml_order, sigma_factor=ref.cpml_sigma_factor,
                              kappa_max=ref.cpml_kappa_max, alpha_max=ref.cpml_alpha_max,
                              bloch_k=(ref.bloch_kx, ref.bloch_ky, ref.bloch_kz))
    if any(config.bloch_k):
        raise ValueError(f"solver '{SOLVER_TYPE}' steps real fields only (Bloch wave vector 0)")
    domain = Domain3D.uniform(source.size_x, source.size_y, source.size_z, float(source.dx),
                              npml_sides=config.npml_sides, boundary_config=config)
    if domain.shape != (source.grid.nx, source.grid.ny, source.grid.nz):
        raise ValueError(f'grid {domain.shape} differs from the model grid '
                         f'{(source.grid.nx, source.grid.ny, source.grid.nz)}')
    _share_materials(source.materials, domain.materials, _MATERIAL_NAMES_3D)
    return EMPhysics3D(domain, precision='single', device=runtime.device)


def _write_dispersive(ctx, physics_spec, physics, kind):
    """The dispersive poles of the model's material regions, as open_sol's create writes them (its own writer, with
    its pole objects converted to this package's)."""
    if not any(getattr(region, 'dispersion', None) for region in getattr(ctx, 'material_regions', ())):
        return
    if kind == '3d':
        raise ValueError(f"solver '{SOLVER_TYPE}': dispersive materials are built for the 2D engines only")
    from open_sol.physics.em.definition_common import write_dispersive_materials
    targets = ('eps_r',) if kind == 'ez' else ('eps_xx', 'eps_yy')
    write_dispersive_materials(ctx, physics_spec, _PoleAdapter(physics), targets)


class _PoleAdapter:
    """The physics as open_sol's dispersive-material writer calls it: its pole objects become this package's."""

    def __init__(self, physics):
        self._physics = physics

    def add_dispersive(self, pole, mask, **options):
        from .poles import DrudePole, LorentzPole
        if hasattr(pole, 'omega_p'):
            pole = DrudePole(float(pole.omega_p), float(pole.gamma), float(pole.eps_inf))
        elif hasattr(pole, 'omega_0'):
            pole = LorentzPole(float(pole.delta_eps), float(pole.omega_0), float(pole.gamma))
        return self._physics.add_dispersive(pole, _host(mask), **options)

    def materials_changed(self, names):
        self._physics.domain.materials.version += 1
        return self._physics.materials_changed(names)

    def __getattr__(self, name):
        return getattr(self._physics, name)
