"""Generate tests/golden/c2_full.npz: the whole 8192 x 8192 roofline workload (opensol_b200.workloads.roofline_2d:
2000 seeded cylinders, a 1550 nm line source, four 16-frequency flux lines) run for 10,000 steps on the CPU.

Three runs of the same workload, each checkpointed at step 600 (past the first flux-line crossing) and at 10,000:

* open_sol itself (its CPU backend, numba twins, float32 stepper), when a reference tree is given;
* the oracle's float32 build (oracle/ez2d.c through oracle/fdtd2d.py), which must give the same bytes;
* the oracle's float64 build (the restatement of open_sol's precision='double' stepper).

Stored: SHA-256 digests of E_z / H_x / H_y and of every monitor's complex128 E / H spectra at each checkpoint, the
four (16,) float64 flux arrays at each checkpoint from the float32 and the float64 runs, the tick count and the DFT
sample interval.  Whole fields and spectra (gigabytes) are not stored; the digests pin them bit for bit.

    python tests/golden/make_golden_c2_full.py [/path/to/reference]

About 35 minutes on 8 host cores (reference ~11 min, oracle float32 ~10 min, float64 ~14 min); without a reference
path only the two oracle runs are made.
"""
import hashlib
import os
import sys
import tempfile
import time

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
CHECKPOINTS = (600, 10_000)


def digest(array):
    import numpy as np
    return hashlib.sha256(np.ascontiguousarray(array).tobytes()).hexdigest()


def record(out, prefix, step, fields, spectra, fluxes):
    for name, arr in fields.items():
        out[f'{prefix}sha_{name}_{step}'] = digest(arr)
    for k, (e, h) in enumerate(spectra):
        out[f'{prefix}sha_spec_e{k}_{step}'] = digest(e)
        out[f'{prefix}sha_spec_h{k}_{step}'] = digest(h)
    for k, f in enumerate(fluxes):
        out[f'{prefix}flux{k}_{step}'] = f


def run_oracle(precision):
    import numpy as np
    from oracle.fdtd2d import OracleEz2D
    from opensol_b200 import workloads
    o = OracleEz2D(**workloads.roofline_2d_sim_args(), precision=precision)
    mons = workloads.apply(o, workloads.roofline_2d_ops())
    out, done = {}, 0
    for cp in CHECKPOINTS:
        o.run(n_steps=cp - done)
        done = cp
        record(out, '', cp, {n: getattr(o, n) for n in ('ez', 'hx', 'hy')},
               [(m.e_acc, m.h_acc) for m in mons], [np.asarray(m.flux(), np.float64) for m in mons])
    out['n_step'] = np.int64(o.n_step)
    out['sample_interval'] = np.int64(o.sample_interval)
    return out


def run_reference(reference):
    import numpy as np
    os.environ.setdefault('NUMBA_CACHE_DIR', os.path.join(tempfile.gettempdir(), 'opensol_numba_cache'))
    sys.path.insert(0, reference)
    from open_sol import Simulation
    from opensol_b200 import workloads
    sim = Simulation(**workloads.roofline_2d_sim_args())
    mons = workloads.apply(sim, workloads.roofline_2d_ops())
    out, done = {}, 0
    for cp in CHECKPOINTS:
        sim.run(n_steps=cp - done, print_every=0)
        done = cp
        fields = sim.em.fields
        record(out, '', cp, {n: np.array(getattr(fields, n)) for n in ('ez', 'hx', 'hy')},
               [(np.array(m._spectra.spectra[0]), np.array(m._spectra.spectra[1])) for m in mons],
               [np.asarray(m.flux(), np.float64) for m in mons])
    out['n_step'] = np.int64(sim.em.engine.n_step)
    out['sample_interval'] = np.int64(mons[0].sample_interval)
    return out


def main():
    import numpy as np
    sys.dont_write_bytecode = True
    sys.path.insert(0, ROOT)
    reference = sys.argv[1] if len(sys.argv) > 1 else os.environ.get('OPENSOL_REFERENCE')
    out = {}
    t = time.time()
    single = run_oracle('single')
    print(f'oracle float32: {time.time() - t:.0f} s', flush=True)
    out.update(single)
    if reference:
        t = time.time()
        ref = run_reference(reference)
        print(f'open_sol float32: {time.time() - t:.0f} s', flush=True)
        mismatch = sorted(k for k in ref if not np.array_equal(np.asarray(ref[k]), np.asarray(single[k])))
        if mismatch:
            raise SystemExit(f'the oracle differs from open_sol on: {mismatch}')
        out['reference_checked'] = np.bool_(True)
    else:
        out['reference_checked'] = np.bool_(False)
    t = time.time()
    double = run_oracle('double')
    print(f'oracle float64: {time.time() - t:.0f} s', flush=True)
    for cp in CHECKPOINTS:
        for k in range(4):
            out[f'f64_flux{k}_{cp}'] = double[f'flux{k}_{cp}']
    path = os.path.join(HERE, 'c2_full.npz')
    np.savez_compressed(path, **out)
    for k in range(4):
        f32, f64 = out[f'flux{k}_10000'], out[f'f64_flux{k}_10000']
        rel = np.abs(f32 - f64).max() / np.abs(f64).max()
        print(f'monitor {k}: float32 vs float64 flux, max error relative to the peak {rel:.3e}')
    print(f'wrote {path} ({len(out)} entries)')


if __name__ == '__main__':
    main()
