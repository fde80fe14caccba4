"""Generate tests/golden/adjoint_c5_fd.npz: the reference-computed gradient of the adjoint workload
(opensol_b200.workloads.adjoint_2d_problem: a 1024 x 1024 total grid, a 200 x 200-cell design box of seeded eps_r,
a 1550 nm line source and the 1550 nm DFT flux through a downstream line after 8,000 steps).

open_sol has no FDTD adjoint, so the reference gradient is a central finite difference of open_sol's own float64
stepper (EMPhysics(..., precision='double'), open_sol/physics/em/__init__.py:73-88): for each of 32 seeded cells of
the design box, eps_r of that cell is moved to float32(eps_r +- 1e-4 eps_r), the whole 8,000-step run is made from
rest each time, and dJ/deps_r = (J+ - J-) / (eps+ - eps-).

    python tests/golden/make_golden_adjoint.py /path/to/reference

65 float64 runs of 1024^2 x 8,000 steps: about 25 minutes on 8 host cores.
"""
import hashlib
import os
import sys
import tempfile
import time

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
N_CELLS = 32
CELL_SEED = 77
REL_STEP = 1e-4


def problem():
    """(simulation arguments, design box, eps_r of the box, source and monitor positions) of the workload."""
    from opensol_b200 import workloads
    import numpy as np
    spec = workloads.ADJOINT_2D
    total, dx, npml, design = spec['total_cells'], spec['dx'], spec['npml'], spec['design']
    window = (total - 2 * npml) * dx
    i0 = (total - design) // 2
    box = (i0, i0 + design, i0, i0 + design)
    eps = np.random.default_rng(spec['seed']).uniform(*spec['eps_r'], (design, design)).astype(np.float32)
    return {'window': window, 'dx': dx, 'npml': npml, 'box': box, 'eps': eps, 'spec': spec}


def objective(p, eps_box):
    """J of one float64 open_sol run of the workload with eps_box on the design box."""
    from open_sol import Simulation
    from open_sol.physics.em import EMPhysics
    from open_sol.simulation import _resolve_em_boundary
    window, spec = p['window'], p['spec']
    base = Simulation(window, window, p['dx'], npml=p['npml'], boundaries='pml')
    sim = Simulation.multiphysics(base.domain)
    sim.add_physics('em', EMPhysics(base.domain, 'ez', _resolve_em_boundary('pml', p['npml']), precision='double'))
    i0, i1, j0, j1 = p['box']
    sim.domain.materials.eps_r[i0:i1, j0:j1] = eps_box
    sim.add_line_source('y', 0.15 * window, wavelength=spec['wavelength'], bandwidth=spec['bandwidth'])
    mon = sim.add_flux_monitor('y', 0.85 * window, (0.0, window), wavelengths=[spec['wavelength']])
    sim.run(n_steps=spec['steps'], print_every=0)
    return float(mon.flux()[0])


def main():
    import numpy as np
    reference = sys.argv[1] if len(sys.argv) > 1 else os.environ.get('OPENSOL_REFERENCE')
    if not reference:
        raise SystemExit('usage: make_golden_adjoint.py /path/to/reference')
    os.environ.setdefault('NUMBA_CACHE_DIR', os.path.join(tempfile.gettempdir(), 'opensol_numba_cache'))
    sys.dont_write_bytecode = True
    sys.path.insert(0, ROOT)
    sys.path.insert(0, reference)
    p = problem()
    eps = p['eps']
    design = eps.shape[0]
    rng = np.random.default_rng(CELL_SEED)
    flat = rng.choice(design * design, N_CELLS, replace=False)
    cells = np.stack([flat // design, flat % design], axis=1).astype(np.int64)
    t = time.time()
    j0 = objective(p, eps)
    print(f'J = {j0!r} ({time.time() - t:.0f} s per run)', flush=True)
    fd = np.empty(N_CELLS)
    steps = np.empty((N_CELLS, 2), np.float32)
    for n, (a, b) in enumerate(cells):
        d = REL_STEP * float(eps[a, b])
        values = []
        for sign in (1.0, -1.0):
            moved = eps.copy()
            moved[a, b] = np.float32(float(eps[a, b]) + sign * d)
            steps[n, 0 if sign > 0 else 1] = moved[a, b]
            values.append(objective(p, moved))
        fd[n] = (values[0] - values[1]) / (float(steps[n, 0]) - float(steps[n, 1]))
        print(f'cell {n} ({a}, {b}): dJ/deps = {fd[n]!r}', flush=True)
    path = os.path.join(HERE, 'adjoint_c5_fd.npz')
    np.savez_compressed(path, cells=cells, fd=fd, eps_steps=steps, J=np.float64(j0),
                        eps_sha=hashlib.sha256(eps.tobytes()).hexdigest(), box=np.asarray(p['box']),
                        rel_step=np.float64(REL_STEP), n_steps=np.int64(p['spec']['steps']))
    print(f'wrote {path}')


if __name__ == '__main__':
    main()
