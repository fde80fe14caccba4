"""Simulation cases shared by the golden-fixture generator (run on open_sol itself), the oracle pinning tests and the
GPU parity tests.  A case is a constructor call plus a list of method calls and step checkpoints, applied the same
way to open_sol's Simulation, the oracle and the B200 engine."""

CASES = [
    {   # the headline 2D case: 6 x 3 um window, 25 nm cells, CPML 15 in x, periodic y, slab, line source, flux line
        'name': 'c1',
        'sim': {'size_x': 6e-6, 'size_y': 3e-6, 'dx': 25e-9, 'npml': 15, 'boundaries': 'periodic_y'},
        'ops': [
            ['add_dielectric_rectangle', [2.75e-6, 0.0, 3.25e-6, 3e-6], {'eps_r': 2.25}],
            ['add_line_source', ['y', 1.2e-6], {'wavelength': 600e-9, 'bandwidth': 0.8}],
            ['add_flux_monitor', ['y', 4.5e-6, [0.0, 3e-6]], {'wavelengths': [500e-9, 600e-9]}],
        ],
        'checkpoints': [300, 1370],
        'duration': 80e-15,
        'store_fields': [300],
    },
    {   # all-CPML box: cylinder, lossy rectangle (ca != 1), spanned x line source, flux lines along x and y
        'name': 'pml_small',
        'sim': {'size_x': 1.5e-6, 'size_y': 1.2e-6, 'dx': 25e-9, 'npml': 10, 'boundaries': 'pml'},
        'ops': [
            ['add_dielectric_circle', [0.75e-6, 0.7e-6, 0.2e-6], {'eps_r': 4.0}],
            ['add_dielectric_rectangle', [0.2e-6, 0.9e-6, 0.6e-6, 1.1e-6], {'eps_r': 2.0, 'sigma_e': 5e4}],
            ['add_line_source', ['x', 0.35e-6], {'wavelength': 700e-9, 'bandwidth': 0.6, 'span': [0.3e-6, 1.2e-6]}],
            ['add_flux_monitor', ['x', 1.0e-6, [0.2e-6, 1.3e-6]], {'wavelengths': [600e-9, 700e-9, 800e-9]}],
            ['add_flux_monitor', ['y', 1.2e-6, [0.1e-6, 1.1e-6]], {'wavelengths': [650e-9, 750e-9]}],
        ],
        'checkpoints': [250, 500],
        'store_fields': [250, 500],
    },
    {   # periodic x, CPML in y, full-line x source with amplitude 2.5, a slab and a circle
        'name': 'periodic_x',
        'sim': {'size_x': 1.0e-6, 'size_y': 1.5e-6, 'dx': 25e-9, 'npml': 8, 'boundaries': 'periodic_x'},
        'ops': [
            ['add_dielectric_rectangle', [0.0, 0.8e-6, 1.0e-6, 1.0e-6], {'eps_r': 3.0}],
            ['add_dielectric_circle', [0.3e-6, 0.5e-6, 0.15e-6], {'eps_r': 6.0}],
            ['add_line_source', ['x', 0.3e-6], {'frequency': 4.5e14, 'bandwidth': 0.5, 'amplitude': 2.5}],
            ['add_flux_monitor', ['x', 1.2e-6, [0.0, 1.0e-6]], {'frequencies': [4.0e14, 4.5e14, 5.0e14]}],
        ],
        'checkpoints': [400],
        'store_fields': [400],
    },
    {   # periodic in x and y (no CPML), spanned y line source, circle
        'name': 'periodic_xy',
        'sim': {'size_x': 1.0e-6, 'size_y': 0.8e-6, 'dx': 25e-9, 'npml': 15, 'boundaries': 'periodic'},
        'ops': [
            ['add_dielectric_circle', [0.6e-6, 0.4e-6, 0.2e-6], {'eps_r': 2.5}],
            ['add_line_source', ['y', 0.2e-6], {'wavelength': 800e-9, 'bandwidth': 0.5, 'span': [0.1e-6, 0.6e-6]}],
            ['add_flux_monitor', ['y', 0.8e-6, [0.0, 0.8e-6]], {'wavelengths': [800e-9]}],
        ],
        'checkpoints': [300],
        'store_fields': [300],
    },
    {   # two crossing line sources (their shared cell takes both, in add order), all CPML, non-square grid
        'name': 'two_sources',
        'sim': {'size_x': 1.6e-6, 'size_y': 1.0e-6, 'dx': 20e-9, 'npml': 12, 'boundaries': 'pml'},
        'ops': [
            ['add_dielectric_rectangle', [1.0e-6, 0.0, 1.2e-6, 1.0e-6], {'eps_r': 5.0}],
            ['add_line_source', ['y', 0.4e-6], {'wavelength': 650e-9, 'bandwidth': 0.7, 'span': [0.2e-6, 0.8e-6]}],
            ['add_line_source', ['x', 0.5e-6], {'wavelength': 550e-9, 'bandwidth': 0.4, 'span': [0.1e-6, 0.9e-6],
                                                'amplitude': 0.5}],
            ['add_flux_monitor', ['y', 1.4e-6, [0.05e-6, 0.95e-6]], {'wavelengths': [550e-9, 650e-9]}],
            ['add_flux_monitor', ['x', 0.9e-6, [0.1e-6, 1.5e-6]], {'wavelengths': [600e-9]}],
        ],
        'checkpoints': [200, 450],
        'store_fields': [450],
    },
]


def case(name):
    for c in CASES:
        if c['name'] == name:
            return c
    raise KeyError(name)


def apply_ops(target, spec):
    """Apply a case's method calls to a Simulation-like target; returns the flux monitors in add order."""
    monitors = []
    for method, args, kwargs in spec['ops']:
        args = [tuple(a) if isinstance(a, list) else a for a in args]
        kwargs = {k: (tuple(v) if isinstance(v, list) and k == 'span' else v) for k, v in kwargs.items()}
        out = getattr(target, method)(*args, **kwargs)
        if method == 'add_flux_monitor':
            monitors.append(out)
    return monitors
