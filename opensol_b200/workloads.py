"""Seeded synthetic workloads of the FDTD benchmarks, applied through the public scripting API (any target with
add_dielectric_circle / add_dielectric_rectangle / add_line_source / add_flux_monitor).

roofline_2d: an 8192 x 8192 total grid (8152 x 8152 window + 20 CPML cells per side) at dx = 20 nm, 2000 dielectric
cylinders (centres uniform in the window interior, radius U(50, 200) nm, eps_r U(2, 12), painted in draw order), a
Gaussian line source at 1550 nm with relative bandwidth 0.5 along y near the lo-x edge, and four 16-frequency flux
lines (x = 10 % / 90 % and y = 10 % / 90 % of the window, frequencies spread over the source band); 10,000 steps.
"""
from __future__ import annotations

import numpy as np

from .constants import C0

ROOFLINE_2D = {
    'total_cells': 8192, 'dx': 20e-9, 'npml': 20, 'n_cylinders': 2000, 'radius': (50e-9, 200e-9),
    'eps_r': (2.0, 12.0), 'wavelength': 1550e-9, 'bandwidth': 0.5, 'n_freqs': 16, 'steps': 10_000, 'seed': 2024,
}


def roofline_2d_sim_args(total_cells=8192, dx=20e-9, npml=20):
    """Simulation(size_x, size_y, dx, npml, boundaries='pml') arguments of a total_cells^2 grid incl. the CPML."""
    window = (total_cells - 2 * npml) * dx
    return {'size_x': window, 'size_y': window, 'dx': dx, 'npml': npml, 'boundaries': 'pml'}


def roofline_2d_ops(total_cells=8192, dx=20e-9, npml=20, n_cylinders=2000, seed=2024, amplitude=1.0):
    """The method calls of the roofline workload, as (method, args, kwargs) in draw order."""
    spec = ROOFLINE_2D
    window = (total_cells - 2 * npml) * dx
    rng = np.random.default_rng(seed)
    radius = rng.uniform(*spec['radius'], n_cylinders)
    centres = rng.uniform(0.15 * window, 0.85 * window, (n_cylinders, 2))
    eps = rng.uniform(*spec['eps_r'], n_cylinders)
    ops = [('add_dielectric_circle', (float(cx), float(cy), float(r)), {'eps_r': float(e)})
           for (cx, cy), r, e in zip(centres, radius, eps)]
    f0 = C0 / spec['wavelength']
    bw = spec['bandwidth']
    freqs = np.linspace(f0 * (1 - bw / 2), f0 * (1 + bw / 2), spec['n_freqs']).tolist()
    ops.append(('add_line_source', ('y', 0.08 * window), {'wavelength': spec['wavelength'], 'bandwidth': bw,
                                                          'amplitude': amplitude}))
    for axis, frac in (('y', 0.10), ('y', 0.90), ('x', 0.10), ('x', 0.90)):
        ops.append(('add_flux_monitor', (axis, frac * window, (0.0, window)), {'frequencies': freqs}))
    return ops


def apply(target, ops):
    """Apply (method, args, kwargs) calls; returns the flux monitors in add order."""
    monitors = []
    for method, args, kwargs in ops:
        out = getattr(target, method)(*args, **kwargs)
        if method == 'add_flux_monitor':
            monitors.append(out)
    return monitors


# 3D: a 512^3 total grid (488^3 window + 12 CPML cells per face) at dx = 20 nm, 500 dielectric spheres (centres uniform
# in the window interior, radius U(40, 160) nm, eps_r U(2, 12), painted in draw order), a z-polarised Gaussian dipole
# at the centre at 1310 nm (relative bandwidth 0.5, moment 1e-12 A m) and a closed 8-frequency flux box (faces at 20 %
# and 80 % of the window); 2,000 steps.
ROOFLINE_3D = {
    'total_cells': 512, 'dx': 20e-9, 'npml': 12, 'n_spheres': 500, 'radius': (40e-9, 160e-9), 'eps_r': (2.0, 12.0),
    'wavelength': 1310e-9, 'bandwidth': 0.5, 'n_freqs': 8, 'steps': 2_000, 'seed': 2025,
}


def roofline_3d_physics(total_cells=512, npml=12, n_spheres=500, seed=2025, device=0):
    """(EMPhysics3D, flux box) of the 3D workload on a total_cells^3 grid incl. the CPML, not yet finalized."""
    from .domain3d import BoundaryConfig3D, Domain3D
    from .physics3d import EMPhysics3D
    spec = ROOFLINE_3D
    dx = spec['dx']
    window = (total_cells - 2 * npml) * dx
    config = BoundaryConfig3D(npml=npml)
    domain = Domain3D.uniform(window, window, window, dx, npml_sides=config.npml_sides, boundary_config=config)
    physics = EMPhysics3D(domain, device=device)
    rng = np.random.default_rng(seed)
    radius = rng.uniform(*spec['radius'], n_spheres)
    centres = rng.uniform(0.15 * window, 0.85 * window, (n_spheres, 3))
    eps = rng.uniform(*spec['eps_r'], n_spheres)
    for (cx, cy, cz), r, e in zip(centres, radius, eps):
        physics.add_dielectric_sphere(float(cx), float(cy), float(cz), float(r), eps_r=float(e))
    physics.add_dipole(0.5 * window, 0.5 * window, 0.5 * window, orientation='z', dipole_moment=1e-12,
                       wavelength=spec['wavelength'], bandwidth=spec['bandwidth'])
    f0 = C0 / spec['wavelength']
    bw = spec['bandwidth']
    freqs = np.linspace(f0 * (1 - bw / 2), f0 * (1 + bw / 2), spec['n_freqs']).tolist()
    box = physics.add_flux_box((0.2 * window,) * 3, (0.8 * window,) * 3, frequencies=freqs)
    return physics, box


# Adjoint: a 1024 x 1024 total grid (984 x 984 window + 20 CPML cells per side) at dx = 20 nm, a 200 x 200-cell design
# region at the window centre with eps_r U(1, 12.1) (seeded), a Gaussian line source at 1550 nm (bandwidth 0.5) along y
# at 15 % of the window, and the objective: the DFT flux at 1550 nm through a line along y at 85 % of the window after
# 8,000 steps, with checkpoints every 256 steps.
ADJOINT_2D = {'total_cells': 1024, 'dx': 20e-9, 'npml': 20, 'design': 200, 'eps_r': (1.0, 12.1),
              'wavelength': 1550e-9, 'bandwidth': 0.5, 'steps': 8000, 'checkpoint_every': 256, 'seed': 2026}


def adjoint_2d_problem(total_cells=1024, design=200, steps=8000, checkpoint_every=256, seed=2026, device=0):
    """(Simulation, flux monitor, design box (i0, i1, j0, j1), design eps_r (design, design) float32) of the adjoint
    workload, finalized."""
    from .simulation import Simulation
    spec = ADJOINT_2D
    dx, npml = spec['dx'], spec['npml']
    window = (total_cells - 2 * npml) * dx
    sim = Simulation(window, window, dx, npml=npml, boundaries='pml', verbose=False, device=device)
    i0 = j0 = (total_cells - design) // 2
    box = (i0, i0 + design, j0, j0 + design)
    eps = np.random.default_rng(seed).uniform(*spec['eps_r'], (design, design)).astype(np.float32)
    sim.domain.materials.array('eps_r')[box[0]:box[1], box[2]:box[3]] = eps
    sim.add_line_source('y', 0.15 * window, wavelength=spec['wavelength'], bandwidth=spec['bandwidth'])
    monitor = sim.add_flux_monitor('y', 0.85 * window, (0.0, window), wavelengths=[spec['wavelength']])
    sim.em.finalize()
    return sim, monitor, box, eps
