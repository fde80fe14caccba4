"""3D cases shared by the golden-fixture generator (run on open_sol itself), the oracle pinning tests and the GPU parity
tests.  A case is a uniform cubic-cell domain (window cells + CPML padding), a boundary configuration, seeded material
paint (spheres and boxes written into the float32 eps_r / sigma_e / mu_r / sigma_m arrays, later wins), one dipole and
flux monitors, and step checkpoints.  paint() is the one writer of the material arrays, so every consumer steps the
very same grid.
"""
import numpy as np

DX = 20e-9

CASES3D = [
    {
        # config-3 shape in miniature: CPML on all faces, seeded dielectric spheres, z dipole at the centre, a closed
        # 8-frequency flux box
        'name': 'c3_small',
        'window': (24, 24, 24), 'npml': 6,
        'faces': {},
        'spheres': {'count': 10, 'seed': 11, 'radius': (40e-9, 160e-9), 'eps_r': (2.0, 12.0)},
        'boxes': [],
        'dipole': {'orientation': 'z', 'at': (0.5, 0.5, 0.5), 'wavelength': 1310e-9, 'bandwidth': 0.5,
                   'moment': 1e-12},
        'flux_box': {'lo': (0.2, 0.2, 0.2), 'hi': (0.8, 0.8, 0.8),
                     'wavelengths': tuple(np.linspace(1100e-9, 1500e-9, 8).tolist())},
        'flux_planes': [],
        'checkpoints': (40, 160),
    },
    {
        # periodic x, a pec and a pmc face on y, CPML on z; lossy (sigma_e) and magnetic (mu_r, sigma_m) blocks; an x
        # dipole; two z flux planes
        'name': 'c3_mixed',
        'window': (16, 20, 28), 'npml': 5,
        'faces': {'x_lo': 'periodic', 'x_hi': 'periodic', 'y_lo': 'pec', 'y_hi': 'pmc'},
        'spheres': {'count': 4, 'seed': 5, 'radius': (40e-9, 100e-9), 'eps_r': (2.0, 6.0)},
        'boxes': [
            {'lo': (0.0, 0.1, 0.55), 'hi': (0.5, 0.6, 0.8), 'values': {'eps_r': 3.0, 'sigma_e': 2.0e4}},
            {'lo': (0.3, 0.5, 0.15), 'hi': (0.9, 0.9, 0.35), 'values': {'mu_r': 2.0, 'sigma_m': 5.0e8}},
        ],
        'dipole': {'orientation': 'x', 'at': (0.45, 0.5, 0.45), 'wavelength': 900e-9, 'bandwidth': 0.6,
                   'moment': 1e-12},
        'flux_box': None,
        'flux_planes': [{'normal': 'z', 'at': 0.2, 'wavelengths': (800e-9, 900e-9, 1000e-9)},
                        {'normal': 'z', 'at': 0.85, 'wavelengths': (800e-9, 900e-9, 1000e-9)}],
        'checkpoints': (50, 140),
    },
]


def case3d(name):
    for c in CASES3D:
        if c['name'] == name:
            return c
    raise KeyError(name)


def grid_shape(spec):
    """Total cells per axis: window plus CPML padding on the cpml faces (uniform cubic cells)."""
    shape = []
    for axis, count in zip('xyz', spec['window']):
        pad = sum(spec['npml'] for side in ('lo', 'hi') if spec['faces'].get(f'{axis}_{side}', 'cpml') == 'cpml')
        shape.append(count + pad)
    return tuple(shape)


def window_size(spec):
    return tuple(count * DX for count in spec['window'])


def origins(spec):
    return tuple(spec['npml'] if spec['faces'].get(f'{axis}_lo', 'cpml') == 'cpml' else 0 for axis in 'xyz')


def cell_centres(spec):
    """Physical cell-centre coordinates (float64) per axis: (k - origin + 0.5) dx."""
    shape, origin = grid_shape(spec), origins(spec)
    return tuple((np.arange(n, dtype=np.float64) - o + 0.5) * DX for n, o in zip(shape, origin))


def paint(spec):
    """float32 eps_r, sigma_e, mu_r, sigma_m arrays of the case (sigma_m None unless a box sets it)."""
    shape = grid_shape(spec)
    arrays = {'eps_r': np.ones(shape, np.float32), 'sigma_e': np.zeros(shape, np.float32),
              'mu_r': np.ones(shape, np.float32)}
    if any('sigma_m' in box['values'] for box in spec['boxes']):
        arrays['sigma_m'] = np.zeros(shape, np.float32)
    cx, cy, cz = cell_centres(spec)
    size = window_size(spec)
    s = spec['spheres']
    if s['count']:
        rng = np.random.default_rng(s['seed'])
        radius = rng.uniform(*s['radius'], s['count'])
        centre = rng.uniform(0.15, 0.85, (s['count'], 3)) * np.asarray(size)
        eps = rng.uniform(*s['eps_r'], s['count'])
        for (x0, y0, z0), r, e in zip(centre, radius, eps):
            mask = ((cx[:, None, None] - x0) ** 2 + (cy[None, :, None] - y0) ** 2
                    + (cz[None, None, :] - z0) ** 2) <= r * r
            arrays['eps_r'][mask] = np.float32(e)
    for box in spec['boxes']:
        lo = np.asarray(box['lo']) * np.asarray(size)
        hi = np.asarray(box['hi']) * np.asarray(size)
        mask = ((cx[:, None, None] >= lo[0]) & (cx[:, None, None] <= hi[0]) & (cy[None, :, None] >= lo[1])
                & (cy[None, :, None] <= hi[1]) & (cz[None, None, :] >= lo[2]) & (cz[None, None, :] <= hi[2]))
        for name, value in box['values'].items():
            arrays[name][mask] = np.float32(value)
    return arrays


def boundary_faces(spec):
    """Face type per FACES_3D face (missing = cpml)."""
    return {f'{axis}_{side}': spec['faces'].get(f'{axis}_{side}', 'cpml') for axis in 'xyz' for side in ('lo', 'hi')}


def roofline_3d_oracle(precision='single', total_cells=512, npml=12, n_spheres=500, seed=2025):
    """(OracleEM3D, flux box) of the 3D benchmark workload (opensol_b200.workloads.roofline_3d_physics: a
    total_cells^3 grid incl. npml CPML cells per face, n_spheres seeded dielectric spheres painted in draw order on the
    cells whose centre lies within the radius, a centred z dipole, a closed 8-frequency flux box), finalized.  The
    spheres are painted here, over each sphere's bounding box of cell centres, from the same seeded draws as the
    workload."""
    from oracle.fdtd3d import OracleEM3D
    from opensol_b200 import workloads
    from opensol_b200.constants import C0
    spec = workloads.ROOFLINE_3D
    dx = spec['dx']
    window = (total_cells - 2 * npml) * dx
    o = OracleEM3D(window, window, window, dx, npml=npml, precision=precision)
    rng = np.random.default_rng(seed)
    radius = rng.uniform(*spec['radius'], n_spheres)
    centres = rng.uniform(0.15 * window, 0.85 * window, (n_spheres, 3))
    eps = rng.uniform(*spec['eps_r'], n_spheres)
    cell_centres = [0.5 * (e[:-1] + e[1:]) for e in o.edges]
    eps_r = o.materials['eps_r']
    for centre, r, e in zip(centres, radius, eps):
        box = []
        for a in range(3):
            lo = int(np.searchsorted(cell_centres[a], centre[a] - r, side='left'))
            hi = int(np.searchsorted(cell_centres[a], centre[a] + r, side='right'))
            box.append(slice(lo, hi))
        x, y, z = (cell_centres[a][box[a]] for a in range(3))
        inside = ((x[:, None, None] - centre[0]) ** 2 + (y[None, :, None] - centre[1]) ** 2
                  + (z[None, None, :] - centre[2]) ** 2) <= r * r
        eps_r[tuple(box)][inside] = np.float32(e)
    o.add_dipole(0.5 * window, 0.5 * window, 0.5 * window, orientation='z', dipole_moment=1e-12,
                 wavelength=spec['wavelength'], bandwidth=spec['bandwidth'])
    f0 = C0 / spec['wavelength']
    bw = spec['bandwidth']
    freqs = np.linspace(f0 * (1 - bw / 2), f0 * (1 + bw / 2), spec['n_freqs'])
    box = o.add_flux_box((0.2 * window,) * 3, (0.8 * window,) * 3, frequencies=freqs)
    o.finalize()
    return o, box
