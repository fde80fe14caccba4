"""The device adjoint (opensol_b200.adjoint) against the float64 discrete adjoint of the oracle and against central
finite differences of the float64 oracle stepper, on a small 2D case with CPML on every side, a dielectric bar, a
line source, a two-frequency flux line and a 10 x 10 design box; checkpoints every 64 steps of 400 (the last segment
partial).  Bar: 1e-3 relative (gradients relative to the box's largest |dJ/deps|)."""
import numpy as np
import pytest

from oracle import adjoint2d
from oracle.fdtd2d import OracleEz2D

import opensol_b200 as ob
from opensol_b200.adjoint import FluxAdjoint2D, flux_objective

pytestmark = pytest.mark.gpu
GRAD_RTOL = 1e-3
BOX = (45, 55, 37, 47)
N_STEPS = 400


def _eps_box():
    return np.random.default_rng(0).uniform(1.0, 12.1, (10, 10)).astype(np.float32)


def _setup(target, eps):
    target.add_dielectric_rectangle(0.9e-6, 0.2e-6, 1.1e-6, 1.4e-6, eps_r=2.5)
    eps_r = target.eps_r if isinstance(target, OracleEz2D) else target.domain.materials.array('eps_r')
    eps_r[BOX[0]:BOX[1], BOX[2]:BOX[3]] = eps
    target.add_line_source('y', 0.3e-6, wavelength=1.0e-6, bandwidth=0.6)
    return target.add_flux_monitor('y', 1.7e-6, (0.0, 1.6e-6), wavelengths=[1.0e-6, 1.1e-6])


def _oracle(eps, precision='double'):
    o = OracleEz2D(2.0e-6, 1.6e-6, 25e-9, npml=10, boundaries='pml', precision=precision)
    _setup(o, eps)
    o.finalize()
    return o


def _product(eps):
    sim = ob.Simulation(2.0e-6, 1.6e-6, 25e-9, npml=10, boundaries='pml', verbose=False)
    mon = _setup(sim, eps)
    sim.em.finalize()
    return sim, mon


def test_adjoint_gradient_against_oracle_adjoint_and_fd():
    eps = _eps_box()
    sim, mon = _product(eps)
    adj = FluxAdjoint2D(sim, mon, 0, BOX, N_STEPS, checkpoint_every=64)
    J = adj.forward()
    o = _oracle(eps, 'single')
    o.run(n_steps=N_STEPS)
    assert J == float(o.monitors[0].flux()[0])                 # the forward is the engine's own, bit-exact
    g = adj.backward()
    box = (slice(BOX[0], BOX[1]), slice(BOX[2], BOX[3]))
    J64, g64 = adjoint2d.gradient(lambda: _oracle(eps), N_STEPS, box)
    scale = np.abs(g64).max()
    assert np.abs(g - g64).max() <= GRAD_RTOL * scale, np.abs(g - g64).max() / scale
    for a, b in [(0, 0), (4, 6), (9, 9)]:
        d = 1e-4 * float(eps[a, b])
        ep, em = eps.copy(), eps.copy()
        ep[a, b] = np.float32(eps[a, b] + d)
        em[a, b] = np.float32(eps[a, b] - d)
        fd = []
        for e in (ep, em):
            o = _oracle(e)
            o.run(n_steps=N_STEPS)
            fd.append(o.monitors[0].flux()[0])
        fd = (fd[0] - fd[1]) / (float(ep[a, b]) - float(em[a, b]))
        assert abs(g[a, b] - fd) <= GRAD_RTOL * abs(fd), (a, b, g[a, b], fd)
    # a second forward / backward on the same object gives the same gradient
    J2 = adj.forward(eps)
    assert J2 == J
    np.testing.assert_array_equal(adj.backward(), g)
    adj.close()


def test_torch_autograd_function():
    import torch
    eps = _eps_box()
    sim, mon = _product(eps)
    adj = FluxAdjoint2D(sim, mon, 1, BOX, 200, checkpoint_every=50)
    f = flux_objective(adj)
    x = torch.tensor(eps, dtype=torch.float64, requires_grad=True)
    J = f(x)
    (2.0 * J).backward()
    np.testing.assert_allclose(x.grad.numpy(), 2.0 * adj.backward(), rtol=0, atol=0)
    adj.close()


def test_adjoint_c5_against_open_sols_float64_finite_differences():
    """The adjoint workload at its stated size (1024^2 incl. 20 CPML cells per side, a 200 x 200 design box of seeded
    eps_r, the 1550 nm flux objective after 8,000 steps, checkpoints every 256) against the reference-computed
    gradient: central finite differences of open_sol's own float64 stepper on 32 seeded cells of the box
    (tests/golden/adjoint_c5_fd.npz, made by tests/golden/make_golden_adjoint.py).  Bar: GRAD_RTOL relative, as the
    norm of the difference over the 32 cells and cell by cell against the largest of them."""
    import hashlib
    import os
    from opensol_b200 import workloads
    g = np.load(os.path.join(os.path.dirname(__file__), 'golden', 'adjoint_c5_fd.npz'))
    spec = workloads.ADJOINT_2D
    sim, monitor, box, eps = workloads.adjoint_2d_problem()
    assert hashlib.sha256(eps.tobytes()).hexdigest() == str(g['eps_sha'])
    assert tuple(box) == tuple(int(v) for v in g['box'])
    adj = FluxAdjoint2D(sim, monitor, 0, box, spec['steps'], checkpoint_every=spec['checkpoint_every'])
    J = adj.forward()
    grad = adj.backward()
    cells = g['cells']
    fd = g['fd']
    got = grad[cells[:, 0], cells[:, 1]]
    norm_error = float(np.linalg.norm(got - fd) / np.linalg.norm(fd))
    cell_error = float(np.abs(got - fd).max() / np.abs(fd).max())
    print(f'J float32 {J!r} vs open_sol float64 {float(g["J"])!r}; gradient error: norm {norm_error:.2e}, '
          f'worst cell {cell_error:.2e}')
    assert abs(J - float(g['J'])) <= 1e-4 * abs(float(g['J']))
    assert norm_error <= GRAD_RTOL
    assert cell_error <= GRAD_RTOL
    adj.close()
