"""Generate the 3D golden fixtures of tests/golden/ by running open_sol's em_fdtd_3d engine itself (CPU backend) on the
cases of cases3d.py, twice: with the numba twins (open_sol's default CPU kernels) and with the numpy twins
(OPEN_SOL_CPU_KERNELS=numpy semantics, switched through open_sol.core.kernels.set_numba(False)).

Run in a container that holds the reference source tree (read-only):

    python tests/golden/make_golden3d.py /path/to/reference

Each case writes <name>.npz with, per twin kind ('numba_' / 'numpy_' prefix): SHA-256 digests of the six fields at
every checkpoint, the central x and z planes of every field, every monitor's flux and the SHA-256 of its complex128
spectra; plus the setup rows (dt, DFT sample interval, material-id digest and eps table, dipole cell, weight and
dual volume, CPML row maps / recursion / gain rows, kappa-folded curl spacings).  material_index3d.npz holds open_sol's
material index of arrays with more distinct values than the id limit (its re-quantisation path).
"""
import hashlib
import json
import os
import sys
import tempfile

HERE = os.path.dirname(os.path.abspath(__file__))


def digest(array):
    import numpy as np
    return hashlib.sha256(np.ascontiguousarray(array).tobytes()).hexdigest()


def build_reference(spec):
    import numpy as np
    from cases3d import DX, boundary_faces, paint, window_size
    from open_sol.core.domain3d import Domain3D
    from open_sol.physics.em3d.boundaries3d import BoundaryConfig3D
    from open_sol.physics.em3d.physics3d import EMPhysics3D
    config = BoundaryConfig3D(boundary_faces(spec), npml=spec['npml'])
    sx, sy, sz = window_size(spec)
    domain = Domain3D.uniform(sx, sy, sz, DX, npml_sides=config.npml_sides, boundary_config=config)
    arrays = paint(spec)
    domain.materials.add_properties({name: (1.0 if name in ('eps_r', 'mu_r') else 0.0) for name in arrays})
    for name, values in arrays.items():
        getattr(domain.materials, name)[...] = values
    physics = EMPhysics3D(domain)
    d = spec['dipole']
    physics.add_dipole(*(f * s for f, s in zip(d['at'], (sx, sy, sz))), orientation=d['orientation'],
                       dipole_moment=d['moment'], wavelength=d['wavelength'], bandwidth=d['bandwidth'])
    monitors = []
    if spec['flux_box'] is not None:
        b = spec['flux_box']
        monitors.append(physics.add_flux_box(tuple(f * s for f, s in zip(b['lo'], (sx, sy, sz))),
                                             tuple(f * s for f, s in zip(b['hi'], (sx, sy, sz))),
                                             wavelengths=list(b['wavelengths'])))
    for p in spec['flux_planes']:
        size = {'x': sx, 'y': sy, 'z': sz}[p['normal']]
        monitors.append(physics.add_flux_plane(p['normal'], p['at'] * size, wavelengths=list(p['wavelengths'])))
    physics.finalize()
    return physics, monitors, arrays


def planes_of(monitor):
    return [plane for _, plane in monitor.faces] if hasattr(monitor, 'faces') else [monitor]


def run_case(spec, prefix):
    import numpy as np
    physics, monitors, _ = build_reference(spec)
    engine = physics.engine
    out = {}
    done = 0
    for cp in spec['checkpoints']:
        for _ in range(cp - done):
            physics.step()
        done = cp
        fields = physics.fields
        for name in ('ex', 'ey', 'ez', 'hx', 'hy', 'hz'):
            arr = np.asarray(getattr(fields, name))
            out[f'{prefix}sha_{name}_{cp}'] = digest(arr)
            out[f'{prefix}{name}_xmid_{cp}'] = np.array(arr[arr.shape[0] // 2])
            out[f'{prefix}{name}_zmid_{cp}'] = np.array(arr[:, :, arr.shape[2] // 2])
        for k, monitor in enumerate(monitors):
            out[f'{prefix}flux{k}_{cp}'] = np.asarray(monitor.flux())
            spectra = [np.asarray(pair[key]) for plane in planes_of(monitor) for pair in plane._pairs
                       for key in ('e_dft', 'h_dft')]
            out[f'{prefix}sha_spectra{k}_{cp}'] = digest(np.concatenate([s.reshape(-1) for s in spectra]))
    out[f'{prefix}n_step'] = np.int64(engine.n_step)
    out[f'{prefix}time'] = np.float64(engine.time)
    return out, physics, monitors


def setup_rows(physics, monitors):
    import numpy as np
    engine = physics.engine
    out = {'dt': np.float32(engine.dt), 'shape': np.asarray(engine.shape, np.int64),
           'sample_interval': np.int64(monitors[0].sample_interval if monitors else 1),
           'sha_material_id': digest(np.asarray(engine.material_id)),
           'table_eps_z': np.asarray(engine.table_eps_z), 'table_sigma': np.asarray(engine.table_sigma),
           'table_mu': np.asarray(engine.table_mu), 'table_sigma_m': np.asarray(engine.table_sigma_m)}
    for axis in range(3):
        out[f'inv_e{axis}'] = np.asarray(engine.inv_e[axis])
        out[f'inv_h{axis}'] = np.asarray(engine.inv_h[axis])
    for layer in engine.cpml:
        key = f'cpml_{layer.axis}{layer.kind}'
        out[key + '_row_map'] = np.asarray(layer.row_map)
        out[key + '_b'] = np.asarray(layer.b)
        out[key + '_gain'] = np.asarray(layer.gain)
    source = physics.sources[0]
    out['dipole_cell'] = np.asarray(source.cell, np.int64)
    out['dipole_weight'] = np.asarray(source.weight)
    out['dipole_volume'] = np.float64(source.volume)
    for k, monitor in enumerate(monitors):
        out[f'monitor{k}_frequencies'] = np.asarray(monitor.frequencies)
        out[f'monitor{k}_planes'] = np.asarray([(plane.normal_axis, plane.edge, *sum(plane.bounds, ()))
                                                for plane in planes_of(monitor)], np.int64)
    return out


def binned_index_cases():
    """(limit, arrays) of the re-quantisation cases: a continuous eps alone above the limit, and a continuous eps with
    a four-level sigma whose joint count needs the level budgets halved."""
    import numpy as np
    rng = np.random.default_rng(21)
    shape = (40, 30, 20)
    eps = rng.uniform(1.0, 12.0, shape).astype(np.float32)
    sigma = (rng.integers(0, 4, shape).astype(np.float32) * np.float32(2.5e3))
    ones = np.ones(shape, np.float32)
    zeros = np.zeros(shape, np.float32)
    return [(300, {'eps_r': eps, 'sigma_e': zeros, 'mu_r': ones}),
            (5000, {'eps_r': eps, 'sigma_e': sigma, 'mu_r': ones})]


def binned_index_fixture():
    """open_sol's material index on arrays with more distinct values than the id limit (re-quantised levels)."""
    import numpy as np
    from open_sol.physics.em3d.material_index3d import build_material_index
    out = {}
    for case, (limit, arrays) in enumerate(binned_index_cases()):
        shape = arrays['eps_r'].shape
        ids = np.zeros(shape, np.uint16)
        chunks = [(slice(start, min(start + 7, shape[0])),) for start in range(0, shape[0], 7)]
        tables, errors, deltas = build_material_index(arrays, chunks, ids, limit, {})
        out[f'case{case}_ids'] = ids
        for name, table in tables.items():
            out[f'case{case}_table_{name}'] = np.asarray(table)
        for name, error in errors.items():
            out[f'case{case}_error_{name}'] = np.float64(error)
            out[f'case{case}_delta_{name}'] = np.float64(deltas[name])
    return out


def main():
    reference = sys.argv[1] if len(sys.argv) > 1 else os.environ.get('OPENSOL_REFERENCE')
    if not reference:
        raise SystemExit('usage: make_golden3d.py /path/to/reference')
    os.environ.setdefault('NUMBA_CACHE_DIR', os.path.join(tempfile.gettempdir(), 'opensol_numba_cache'))
    sys.dont_write_bytecode = True
    sys.path.insert(0, reference)
    sys.path.insert(0, HERE)
    import numpy as np
    from cases3d import CASES3D
    from open_sol.core.kernels import set_numba
    index = {}
    for spec in CASES3D:
        set_numba(None)
        out, physics, monitors = run_case(spec, 'numba_')
        out.update(setup_rows(physics, monitors))
        set_numba(False)
        numpy_out, _, _ = run_case(spec, 'numpy_')
        set_numba(None)
        out.update(numpy_out)
        path = os.path.join(HERE, f"{spec['name']}.npz")
        np.savez_compressed(path, **out)
        index[spec['name']] = sorted(out)
        print(f"{spec['name']}: {len(out)} entries, shape {tuple(out['shape'])}, m {int(out['sample_interval'])}, "
              f"dt {float(out['dt']):.6g}")
    binned = binned_index_fixture()
    np.savez_compressed(os.path.join(HERE, 'material_index3d.npz'), **binned)
    index['material_index3d'] = sorted(binned)
    with open(os.path.join(HERE, 'index3d.json'), 'w') as f:
        json.dump({'generated_by': 'tests/golden/make_golden3d.py (open_sol em_fdtd_3d, CPU backend, numba and numpy '
                                   'twins)', 'cases': index}, f, indent=1)


if __name__ == '__main__':
    main()
