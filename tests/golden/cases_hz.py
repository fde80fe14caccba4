"""H_z-polarisation cases (H_z at cell centres, E_x / E_y on the hi faces) shared by the golden-fixture generator (run
on open_sol itself), the oracle pinning tests and the GPU parity tests; the same format as cases.py, with the
constructor's polarization='hz'."""

HZ_CASES = [
    {   # all-CPML box: circle, lossy rectangle, spanned E_x sheet (axis 'x'), flux lines with normals y and x
        'name': 'hz_pml',
        'sim': {'size_x': 1.5e-6, 'size_y': 1.2e-6, 'dx': 25e-9, 'npml': 10, 'boundaries': 'pml',
                'polarization': 'hz'},
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
    {   # config-1 geometry in H_z: periodic y, slab, E_y sheet along y, flux line
        'name': 'hz_periodic_y',
        'sim': {'size_x': 3e-6, 'size_y': 1.5e-6, 'dx': 25e-9, 'npml': 15, 'boundaries': 'periodic_y',
                'polarization': 'hz'},
        'ops': [
            ['add_dielectric_rectangle', [1.4e-6, 0.0, 1.7e-6, 1.5e-6], {'eps_r': 2.25}],
            ['add_line_source', ['y', 0.6e-6], {'wavelength': 600e-9, 'bandwidth': 0.8}],
            ['add_flux_monitor', ['y', 2.4e-6, [0.0, 1.5e-6]], {'wavelengths': [500e-9, 600e-9]}],
        ],
        'checkpoints': [300, 600],
        'store_fields': [300],
    },
    {   # periodic x, CPML in y, full-line E_x sheet with amplitude 1.5, circle
        'name': 'hz_periodic_x',
        'sim': {'size_x': 1.0e-6, 'size_y': 1.5e-6, 'dx': 25e-9, 'npml': 8, 'boundaries': 'periodic_x',
                'polarization': 'hz'},
        'ops': [
            ['add_dielectric_circle', [0.3e-6, 0.5e-6, 0.15e-6], {'eps_r': 6.0}],
            ['add_line_source', ['x', 0.3e-6], {'frequency': 4.5e14, 'bandwidth': 0.5, 'amplitude': 1.5}],
            ['add_flux_monitor', ['x', 1.2e-6, [0.0, 1.0e-6]], {'frequencies': [4.0e14, 4.5e14, 5.0e14]}],
        ],
        'checkpoints': [400],
        'store_fields': [400],
    },
]
