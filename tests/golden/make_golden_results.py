"""Generate the results.npz fixtures of tests/golden/ by running open_sol itself (CPU backend) on two field-map cases
of cases_dft.py (E_z 'dft_pml', H_z 'dft_hz_pml') and writing their monitors' result dicts with open_sol's own
results.npz writer.

Run in a container that holds the reference source tree (read-only):

    python tests/golden/make_golden_results.py /path/to/reference

Each case writes results_<name>.npz exactly as open_sol's save_results writes results.npz: one result per monitor,
keyed 'em.flux<k>' (flux_result with the physics: power, power_per_cw, mirror factor), 'em.map<k>' (dft_result at
frequency index 0 with the physics: intensity, intensity_per_cw_factor, centres, extent) and 'em.probe<k>'
(probe_result with the renderer's unit), after the case's last checkpoint.
"""
import os
import sys
import tempfile

HERE = os.path.dirname(os.path.abspath(__file__))
CASE_NAMES = ('dft_pml', 'dft_hz_pml')


def run_case(spec):
    from open_sol import Simulation
    from open_sol.physics.em.materials import DrudePole, LorentzPole
    from open_sol.physics.em.results import dft_result, flux_result, probe_result
    from cases import apply_ops
    from cases_dft import apply_poles
    sim = Simulation(**spec['sim'])
    fluxes = apply_ops(sim, spec)
    apply_poles(sim.em, spec, DrudePole, LorentzPole, sim.domain.circle_mask)
    maps = [sim.em.add_dft_monitor(x0, y0, x1, y1, frequencies=freqs, downsample=ds)
            for x0, y0, x1, y1, freqs, ds in spec['dft']]
    probes = [sim.em.add_field_probe(x, y, comp) for x, y, comp in spec.get('probes', [])]
    sim.run(n_steps=spec['checkpoints'][-1], print_every=0)
    results = {}
    for k, mon in enumerate(fluxes):
        results[f'em.flux{k}'] = flux_result(mon, sim.em)
    for k, mon in enumerate(maps):
        results[f'em.map{k}'] = dft_result(mon, sim.domain, freq_index=0, physics=sim.em)
    for k, probe in enumerate(probes):
        unit = sim.em.renderer().field_info(probe.field_component).unit
        results[f'em.probe{k}'] = probe_result(probe, unit)
    return results


def main():
    reference = sys.argv[1] if len(sys.argv) > 1 else os.environ.get('OPENSOL_REFERENCE')
    if not reference:
        raise SystemExit('usage: make_golden_results.py /path/to/reference')
    os.environ.setdefault('NUMBA_CACHE_DIR', os.path.join(tempfile.gettempdir(), 'opensol_numba_cache'))
    sys.dont_write_bytecode = True
    sys.path.insert(0, reference)
    sys.path.insert(0, HERE)
    from pathlib import Path
    from open_sol.io.model_io import _write_npz
    from open_sol.io.results_io import ResultsData, _results_arrays, json_safe
    from cases_dft import case
    for name in CASE_NAMES:
        data = ResultsData(summary={}, results=run_case(case(name)))
        arrays, metadata = _results_arrays(data)
        _write_npz(Path(HERE) / f'results_{name}.npz', arrays, json_safe(metadata), atomic=False)
        print(f'results_{name}.npz: {len(arrays)} arrays, results {sorted(data.results)}')


if __name__ == '__main__':
    main()
