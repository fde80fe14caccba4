"""Generate the H_z golden fixtures of tests/golden/ by running open_sol itself (its CPU backend, numba twins) on the
cases of cases_hz.py.

Run in a container that holds the reference source tree (read-only):

    python tests/golden/make_golden_hz.py /path/to/reference

Each case writes <name>.npz: SHA-256 digests of H_z, E_x, E_y at every checkpoint, the fields at the stored
checkpoints, every flux monitor's complex128 spectra and flux, and the setup rows (face coefficients ca_x, cb_x, ca_y,
cb_y, da, db, curl spacings, CPML recursion rows, calibrated sheet profiles, dt, DFT sample interval).
"""
import json
import os
import sys
import tempfile

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, HERE)
from make_golden import digest   # noqa: E402


def run_case(spec):
    import numpy as np
    from cases import apply_ops
    from open_sol import Simulation
    sim = Simulation(**spec['sim'])
    monitors = apply_ops(sim, spec)
    out = {}
    done = 0
    for cp in spec['checkpoints']:
        sim.run(n_steps=cp - done, print_every=0)
        done = cp
        fields = sim.em.fields
        for name in ('hz', 'ex', 'ey'):
            arr = np.array(getattr(fields, name))
            out[f'sha_{name}_{cp}'] = digest(arr)
            if cp in spec.get('store_fields', ()):
                out[f'{name}_{cp}'] = arr
        for k, mon in enumerate(monitors):
            out[f'flux{k}_{cp}'] = np.asarray(mon.flux())
            out[f'spec_e{k}_{cp}'] = np.array(mon._spectra.spectra[0])
            out[f'spec_h{k}_{cp}'] = np.array(mon._spectra.spectra[1])
    eng = sim.em.engine
    out['n_step'] = np.int64(eng.n_step)
    out['dt'] = np.float32(eng.dt)
    out['nx'], out['ny'] = np.int64(eng.nx), np.int64(eng.ny)
    out['sample_interval'] = np.int64(monitors[0].sample_interval if monitors else 1)
    for name in ('ca_x', 'cb_x', 'ca_y', 'cb_y', 'da', 'db'):
        out[name] = np.array(getattr(eng, name))
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


def main():
    reference = sys.argv[1] if len(sys.argv) > 1 else os.environ.get('OPENSOL_REFERENCE')
    if not reference:
        raise SystemExit('usage: make_golden_hz.py /path/to/reference')
    os.environ.setdefault('NUMBA_CACHE_DIR', os.path.join(tempfile.gettempdir(), 'opensol_numba_cache'))
    sys.dont_write_bytecode = True
    sys.path.insert(0, reference)
    import numpy as np
    from cases_hz import HZ_CASES
    index = {}
    for spec in HZ_CASES:
        out = run_case(spec)
        np.savez_compressed(os.path.join(HERE, f"{spec['name']}.npz"), **out)
        index[spec['name']] = sorted(out)
        print(f"{spec['name']}: {len(out)} entries, n_step {int(out['n_step'])}, m {int(out['sample_interval'])}")
    with open(os.path.join(HERE, 'index_hz.json'), 'w') as f:
        json.dump({'generated_by': 'tests/golden/make_golden_hz.py (open_sol CPU backend, numba twins)',
                   'cases': index}, f, indent=1)


if __name__ == '__main__':
    main()
