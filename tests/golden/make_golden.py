"""Generate the golden fixtures of tests/golden/ by running open_sol itself (its CPU backend, numba twins, float32
and float64 steppers) on the cases of cases.py.

Run in a container that holds the reference source tree (read-only):

    python tests/golden/make_golden.py /path/to/reference

Each case writes <name>.npz: field arrays at the stored checkpoints, SHA-256 digests of every field at every
checkpoint, the flux monitors' complex128 spectra and fluxes, and setup rows (cb, calibrated profiles, curl
spacings, CPML recursion rows, DFT sample interval).  config-1 ('c1') is also run with the float64 stepper (fields'
digests, spectra and fluxes under the 'f64_' prefix) and once with run(duration=80 fs) to record its tick count.
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


def build_reference(spec, precision):
    from open_sol import Simulation
    from open_sol.physics.em import EMPhysics
    from open_sol.simulation import _resolve_em_boundary
    sim_kwargs = dict(spec['sim'])
    sim = Simulation(**sim_kwargs)
    if precision == 'double':
        bc = _resolve_em_boundary(sim_kwargs.get('boundaries'), sim_kwargs.get('npml', 15))
        domain = sim.domain
        sim = Simulation.multiphysics(domain)
        sim.add_physics('em', EMPhysics(domain, 'ez', bc, precision='double'))
    return sim


def run_case(spec, precision='single'):
    import numpy as np
    from cases import apply_ops
    sim = build_reference(spec, precision)
    monitors = apply_ops(sim, spec)
    out = {}
    done = 0
    for cp in spec['checkpoints']:
        sim.run(n_steps=cp - done, print_every=0)
        done = cp
        fields = sim.em.fields
        for name in ('ez', 'hx', 'hy'):
            arr = np.array(getattr(fields, name))
            out[f'sha_{name}_{cp}'] = digest(arr)
            if cp in spec.get('store_fields', ()) and precision == 'single':
                out[f'{name}_{cp}'] = arr
        for k, mon in enumerate(monitors):
            out[f'flux{k}_{cp}'] = np.asarray(mon.flux())
            out[f'spec_e{k}_{cp}'] = np.array(mon._spectra.spectra[0])
            out[f'spec_h{k}_{cp}'] = np.array(mon._spectra.spectra[1])
    eng = sim.em.engine
    out['n_step'] = np.int64(eng.n_step)
    out['time'] = np.float64(eng.time)
    out['dt'] = np.float32(eng.dt)
    out['nx'], out['ny'] = np.int64(eng.nx), np.int64(eng.ny)
    out['sample_interval'] = np.int64(monitors[0].sample_interval if monitors else 1)
    if precision == 'single':
        out['cb'] = np.array(eng.cb)
        out['ca'] = np.array(eng.ca)
        for name in ('inv_dx_e', 'inv_dx_h', 'inv_dy_e', 'inv_dy_h'):
            out[name] = np.array(getattr(eng, f'_{name}_1d'))
        for k, src in enumerate(sim.em.sources):
            out[f'profile{k}'] = np.array(src.profile)
            out[f'source_line{k}'] = np.array([0 if src.axis == 'x' else 1, src.position,
                                               *(src.span if src.span is not None else (-1, -1))])
        cpml = sim.em.boundary_mgr.cpml
        if cpml is not None:
            for side_index, side in enumerate(cpml._sides):
                for kind in ('e', 'h'):
                    rows = getattr(side, kind)
                    out[f'cpml{side_index}_{kind}_b'] = np.array(rows.b).reshape(-1)
                    out[f'cpml{side_index}_{kind}_a'] = np.array(rows.a).reshape(-1)
                    out[f'cpml{side_index}_{kind}_inv'] = np.array(rows.inv_spacing).reshape(-1)
        for k, mon in enumerate(monitors):
            out[f'monitor{k}'] = np.array([0 if mon.axis == 'x' else 1, mon.position, *mon.span])
    return out


def duration_steps(spec):
    from cases import apply_ops
    sim = build_reference(spec, 'single')
    apply_ops(sim, spec)
    sim.run(duration=spec['duration'], print_every=0)
    return sim.em.engine.n_step


def main():
    reference = sys.argv[1] if len(sys.argv) > 1 else os.environ.get('OPENSOL_REFERENCE')
    if not reference:
        raise SystemExit('usage: make_golden.py /path/to/reference')
    os.environ.setdefault('NUMBA_CACHE_DIR', os.path.join(tempfile.gettempdir(), 'opensol_numba_cache'))
    sys.dont_write_bytecode = True
    sys.path.insert(0, reference)
    sys.path.insert(0, HERE)
    import numpy as np
    from cases import CASES
    index = {}
    for spec in CASES:
        out = run_case(spec, 'single')
        if spec['name'] == 'c1':
            f64 = run_case(spec, 'double')
            for key, value in f64.items():
                if key.startswith(('sha_', 'flux', 'spec_')):
                    out['f64_' + key] = value
            out['duration_steps'] = np.int64(duration_steps(spec))
        path = os.path.join(HERE, f"{spec['name']}.npz")
        np.savez_compressed(path, **out)
        index[spec['name']] = sorted(out)
        print(f"{spec['name']}: {len(out)} entries, n_step {int(out['n_step'])}, m {int(out['sample_interval'])}")
    with open(os.path.join(HERE, 'index.json'), 'w') as f:
        json.dump({'generated_by': 'tests/golden/make_golden.py (open_sol CPU backend, numba twins)',
                   'cases': index}, f, indent=1)


if __name__ == '__main__':
    main()
