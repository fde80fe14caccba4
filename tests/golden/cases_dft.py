"""Cases with field-map (running DFT) monitors, shared by the golden-fixture generator (run on open_sol itself),
the oracle pinning tests and the GPU parity tests.  Same form as cases.py; 'dft' lists the field-map monitors added
through the E_z physics (x0, y0, x1, y1 [m], frequencies [Hz], downsample); 'probes' the field probes (x, y [m],
component); 'poles' dispersive media added after the ops: ['drude_rect', (x0, y0, x1, y1), (omega_p, gamma, eps_inf)],
['drude_circle', (cx, cy, r), (omega_p, gamma, eps_inf)] (eps_r = eps_inf under the pole) or ['lorentz_circle', (cx,
cy, r), (delta_eps, omega_0, gamma)] (add_dispersive on the circle's mask, eps_r kept)."""

CASES_DFT = [
    {   # all-CPML box: cylinder, lossy rectangle, spanned line source, flux line, a full-resolution map and a
        # 3x-downsampled map whose box is not a multiple of 3 cells
        'name': 'dft_pml',
        'sim': {'size_x': 1.5e-6, 'size_y': 1.2e-6, 'dx': 25e-9, 'npml': 10, 'boundaries': 'pml'},
        'ops': [
            ['add_dielectric_circle', [0.75e-6, 0.7e-6, 0.2e-6], {'eps_r': 4.0}],
            ['add_dielectric_rectangle', [0.2e-6, 0.9e-6, 0.6e-6, 1.1e-6], {'eps_r': 2.0, 'sigma_e': 5e4}],
            ['add_line_source', ['x', 0.35e-6], {'wavelength': 700e-9, 'bandwidth': 0.6, 'span': [0.3e-6, 1.2e-6]}],
            ['add_flux_monitor', ['x', 1.0e-6, [0.2e-6, 1.3e-6]], {'wavelengths': [600e-9, 700e-9]}],
        ],
        'dft': [
            [0.3e-6, 0.2e-6, 1.2e-6, 1.0e-6, [4.2e14, 5.0e14], 1],
            [0.1e-6, 0.05e-6, 1.4e-6, 1.15e-6, [4.6e14], 3],
        ],
        'probes': [[0.75e-6, 0.5e-6, 'ez'], [0.12e-6, 0.6e-6, 'hx'], [1.1e-6, 1.15e-6, 'hy']],
        'checkpoints': [250, 500],
    },
    {   # +x plane wave (TFSF box) on a cylinder, all CPML: a map over the box and the scattered-field ring, a flux
        # line and a probe outside the box (scattered field only)
        'name': 'tfsf_cylinder',
        'sim': {'size_x': 2.0e-6, 'size_y': 1.6e-6, 'dx': 25e-9, 'npml': 12, 'boundaries': 'pml'},
        'ops': [
            ['add_dielectric_circle', [1.0e-6, 0.8e-6, 0.25e-6], {'eps_r': 4.0}],
            ['add_tfsf', [0.4e-6, 0.3e-6, 1.6e-6, 1.3e-6], {'wavelength': 700e-9, 'bandwidth': 0.5}],
            ['add_flux_monitor', ['y', 1.8e-6, [0.2e-6, 1.4e-6]], {'wavelengths': [650e-9, 750e-9]}],
        ],
        'dft': [
            [0.2e-6, 0.1e-6, 1.85e-6, 1.5e-6, [4.3e14], 2],
        ],
        'probes': [[1.8e-6, 0.8e-6, 'ez'], [1.0e-6, 0.35e-6, 'hy']],
        'checkpoints': [300, 700],
    },
    {   # periodic y: a TFSF box beside a line source (no shared cell) and a slab inside the box
        'name': 'tfsf_periodic_y',
        'sim': {'size_x': 2.4e-6, 'size_y': 1.0e-6, 'dx': 25e-9, 'npml': 12, 'boundaries': 'periodic_y'},
        'ops': [
            ['add_dielectric_rectangle', [1.0e-6, 0.0, 1.2e-6, 1.0e-6], {'eps_r': 2.5}],
            ['add_tfsf', [0.5e-6, 0.1e-6, 1.6e-6, 0.9e-6], {'frequency': 4.6e14, 'bandwidth': 0.6,
                                                            'amplitude': 2.0}],
            ['add_line_source', ['y', 2.0e-6], {'wavelength': 600e-9, 'bandwidth': 0.5, 'amplitude': 0.5}],
            ['add_flux_monitor', ['y', 2.2e-6, [0.0, 1.0e-6]], {'wavelengths': [600e-9, 650e-9]}],
        ],
        'dft': [
            [0.3e-6, 0.0, 1.9e-6, 0.99e-6, [4.6e14], 3],
        ],
        'probes': [[1.7e-6, 0.5e-6, 'ez']],
        'checkpoints': [350, 600],
    },
    {   # a Drude rectangle and a Lorentz circle (on an eps 2 background), all CPML; the line source crosses the
        # Lorentz circle (its calibration takes the pole's susceptibility); a probe inside the metal
        'name': 'poles_pml',
        'sim': {'size_x': 1.6e-6, 'size_y': 1.4e-6, 'dx': 25e-9, 'npml': 10, 'boundaries': 'pml'},
        'ops': [
            ['add_dielectric_circle', [0.5e-6, 0.9e-6, 0.15e-6], {'eps_r': 2.0}],
            ['add_line_source', ['y', 0.5e-6], {'wavelength': 800e-9, 'bandwidth': 0.5, 'span': [0.2e-6, 1.2e-6]}],
            ['add_flux_monitor', ['y', 1.4e-6, [0.1e-6, 1.3e-6]], {'wavelengths': [750e-9, 850e-9]}],
        ],
        'poles': [['drude_rect', [0.9e-6, 0.4e-6, 1.2e-6, 1.0e-6], [8e15, 5e13, 2.0]],
                  ['lorentz_circle', [0.5e-6, 0.9e-6, 0.15e-6], [1.5, 3e15, 2e14]]],
        'dft': [
            [0.6e-6, 0.2e-6, 1.5e-6, 1.2e-6, [3.8e14], 2],
        ],
        'probes': [[1.0e-6, 0.7e-6, 'ez'], [0.5e-6, 0.9e-6, 'hx']],
        'checkpoints': [300, 700],
    },
    {   # two overlapping Drude media (their currents summed on the union box), periodic x
        'name': 'poles_two_drude',
        'sim': {'size_x': 1.2e-6, 'size_y': 1.6e-6, 'dx': 25e-9, 'npml': 10, 'boundaries': 'periodic_x'},
        'ops': [
            ['add_line_source', ['x', 0.3e-6], {'wavelength': 700e-9, 'bandwidth': 0.6}],
            ['add_flux_monitor', ['x', 1.3e-6, [0.0, 1.2e-6]], {'wavelengths': [650e-9, 750e-9]}],
        ],
        'poles': [['drude_circle', [0.5e-6, 0.8e-6, 0.2e-6], [9e15, 1e14, 2.5]],
                  ['drude_rect', [0.6e-6, 0.7e-6, 1.0e-6, 1.0e-6], [6e15, 3e13, 2.0]]],
        'dft': [
            [0.1e-6, 0.5e-6, 1.1e-6, 1.2e-6, [4.3e14], 1],
        ],
        'probes': [[0.55e-6, 0.85e-6, 'ez']],
        'checkpoints': [250, 500],
    },
    {   # periodic y, CPML in x: a map crossing the slab and one touching the y edge of the grid
        'name': 'dft_periodic_y',
        'sim': {'size_x': 2.0e-6, 'size_y': 1.0e-6, 'dx': 25e-9, 'npml': 12, 'boundaries': 'periodic_y'},
        'ops': [
            ['add_dielectric_rectangle', [1.0e-6, 0.0, 1.3e-6, 1.0e-6], {'eps_r': 2.25}],
            ['add_line_source', ['y', 0.5e-6], {'wavelength': 650e-9, 'bandwidth': 0.7}],
            ['add_flux_monitor', ['y', 1.6e-6, [0.0, 1.0e-6]], {'wavelengths': [650e-9]}],
        ],
        'dft': [
            [0.7e-6, 0.0, 1.8e-6, 0.99e-6, [4.0e14, 4.6e14, 5.2e14], 2],
        ],
        'probes': [[1.2e-6, 0.0, 'ez']],
        'checkpoints': [300, 600],
    },
]


# H_z polarisation: maps of H_z and of E_x / E_y collocated to the cell centres; one box starts on the periodic
# axis's cell 0 at full resolution (its E partner face wraps to the last face)
CASES_DFT_HZ = [
    {   # all-CPML box: circle, lossy rectangle, E_x sheet, flux line; a full-resolution and a 2x-downsampled map
        'name': 'dft_hz_pml',
        'sim': {'size_x': 1.5e-6, 'size_y': 1.2e-6, 'dx': 25e-9, 'npml': 10, 'boundaries': 'pml',
                'polarization': 'hz'},
        'ops': [
            ['add_dielectric_circle', [0.75e-6, 0.7e-6, 0.2e-6], {'eps_r': 4.0}],
            ['add_dielectric_rectangle', [0.2e-6, 0.9e-6, 0.6e-6, 1.1e-6], {'eps_r': 2.0, 'sigma_e': 5e4}],
            ['add_line_source', ['x', 0.35e-6], {'wavelength': 700e-9, 'bandwidth': 0.6, 'span': [0.3e-6, 1.2e-6]}],
            ['add_flux_monitor', ['x', 1.0e-6, [0.2e-6, 1.3e-6]], {'wavelengths': [600e-9, 700e-9]}],
        ],
        'dft': [
            [0.3e-6, 0.2e-6, 1.2e-6, 1.0e-6, [4.2e14, 5.0e14], 1],
            [0.1e-6, 0.05e-6, 1.4e-6, 1.15e-6, [4.6e14], 2],
        ],
        'probes': [[0.75e-6, 0.5e-6, 'hz'], [0.5e-6, 0.6e-6, 'ex']],
        'checkpoints': [250, 500],
    },
    {   # +x plane wave (TFSF box, incident E_y) on a cylinder in H_z, all CPML; flux line, map and probe outside
        'name': 'tfsf_hz_cylinder',
        'sim': {'size_x': 2.0e-6, 'size_y': 1.6e-6, 'dx': 25e-9, 'npml': 12, 'boundaries': 'pml',
                'polarization': 'hz'},
        'ops': [
            ['add_dielectric_circle', [1.0e-6, 0.8e-6, 0.25e-6], {'eps_r': 4.0}],
            ['add_tfsf', [0.4e-6, 0.3e-6, 1.6e-6, 1.3e-6], {'wavelength': 700e-9, 'bandwidth': 0.5}],
            ['add_flux_monitor', ['y', 1.8e-6, [0.2e-6, 1.4e-6]], {'wavelengths': [650e-9, 750e-9]}],
        ],
        'dft': [
            [0.2e-6, 0.1e-6, 1.85e-6, 1.5e-6, [4.3e14], 2],
        ],
        'probes': [[1.8e-6, 0.8e-6, 'hz'], [1.0e-6, 0.35e-6, 'ey']],
        'checkpoints': [300, 700],
    },
    {   # periodic y: a full-resolution map from y = 0 (wrapped partner faces) and a 3x-downsampled one
        'name': 'dft_hz_periodic_y',
        'sim': {'size_x': 2.0e-6, 'size_y': 1.0e-6, 'dx': 25e-9, 'npml': 12, 'boundaries': 'periodic_y',
                'polarization': 'hz'},
        'ops': [
            ['add_dielectric_rectangle', [1.0e-6, 0.0, 1.3e-6, 1.0e-6], {'eps_r': 2.25}],
            ['add_line_source', ['y', 0.5e-6], {'wavelength': 650e-9, 'bandwidth': 0.7}],
            ['add_flux_monitor', ['y', 1.6e-6, [0.0, 1.0e-6]], {'wavelengths': [650e-9]}],
        ],
        'dft': [
            [0.7e-6, 0.0, 1.8e-6, 0.6e-6, [4.0e14, 5.2e14], 1],
            [0.4e-6, 0.1e-6, 1.5e-6, 0.99e-6, [4.6e14], 3],
        ],
        'probes': [[1.2e-6, 0.0, 'ey']],
        'checkpoints': [300, 600],
    },
    {   # H_z poles: a Drude rectangle and a Lorentz circle on E_x / E_y face sets (face-averaged cell masks), all
        # CPML; the E_y sheet crosses the Lorentz circle (its calibration takes the pole's susceptibility); probes of
        # E_x / E_y inside the metal
        'name': 'poles_hz_pml',
        'sim': {'size_x': 1.6e-6, 'size_y': 1.4e-6, 'dx': 25e-9, 'npml': 10, 'boundaries': 'pml',
                'polarization': 'hz'},
        'ops': [
            ['add_dielectric_circle', [0.5e-6, 0.9e-6, 0.15e-6], {'eps_r': 2.0}],
            ['add_line_source', ['y', 0.5e-6], {'wavelength': 800e-9, 'bandwidth': 0.5, 'span': [0.2e-6, 1.2e-6]}],
            ['add_flux_monitor', ['y', 1.4e-6, [0.1e-6, 1.3e-6]], {'wavelengths': [750e-9, 850e-9]}],
        ],
        'poles': [['drude_rect', [0.9e-6, 0.4e-6, 1.2e-6, 1.0e-6], [8e15, 5e13, 2.0]],
                  ['lorentz_circle', [0.5e-6, 0.9e-6, 0.15e-6], [1.5, 3e15, 2e14]]],
        'dft': [
            [0.6e-6, 0.2e-6, 1.5e-6, 1.2e-6, [3.8e14], 2],
        ],
        'probes': [[1.0e-6, 0.7e-6, 'ex'], [1.1e-6, 0.5e-6, 'ey'], [0.5e-6, 0.9e-6, 'hz']],
        'checkpoints': [300, 700],
    },
    {   # two overlapping Drude media (each face set corrected in turn) on a periodic y axis, one spanning the whole
        # y range (its last E_x faces pair with the wrapped first cells); an E_x sheet
        'name': 'poles_hz_periodic_y',
        'sim': {'size_x': 1.6e-6, 'size_y': 1.2e-6, 'dx': 25e-9, 'npml': 10, 'boundaries': 'periodic_y',
                'polarization': 'hz'},
        'ops': [
            ['add_line_source', ['x', 0.25e-6], {'wavelength': 700e-9, 'bandwidth': 0.6, 'span': [0.1e-6, 1.5e-6]}],
            ['add_flux_monitor', ['y', 1.3e-6, [0.0, 1.2e-6]], {'wavelengths': [650e-9, 750e-9]}],
        ],
        'poles': [['drude_rect', [0.8e-6, 0.0, 1.0e-6, 1.2e-6], [6e15, 3e13, 2.0]],
                  ['drude_circle', [0.9e-6, 0.6e-6, 0.2e-6], [9e15, 1e14, 2.5]]],
        'dft': [
            [0.1e-6, 0.0, 1.5e-6, 1.2e-6, [4.3e14], 1],
        ],
        'probes': [[0.9e-6, 0.6e-6, 'ex'], [0.85e-6, 1.18e-6, 'ey']],
        'checkpoints': [250, 500],
    },
]


def case(name):
    for c in CASES_DFT + CASES_DFT_HZ:
        if c['name'] == name:
            return c
    raise KeyError(name)


def apply_poles(target, spec, drude_class, lorentz_class, circle_mask):
    """Add a case's 'poles' to a Simulation-like target: drude_class(omega_p, gamma, eps_inf), lorentz_class(delta_eps,
    omega_0, gamma) and circle_mask(cx, cy, r) are the target's own."""
    for kind, where, params in spec.get('poles', []):
        if kind == 'drude_rect':
            target.add_drude_rectangle(*where, drude_class(*params))
        elif kind == 'drude_circle':
            target.add_drude_circle(*where, drude_class(*params))
        else:
            target.add_dispersive(lorentz_class(*params), circle_mask(*where))
