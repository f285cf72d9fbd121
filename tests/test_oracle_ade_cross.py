"""Dispersive media of every kind on a grid, C++ oracle against the
vectorised numpy restatement (oracle/ade_ref.py): fields bit for bit, which
pins the capture of E before the E update (kinds 3 and 4) and the order of
the updates around the field update."""
import numpy as np
import pytest

import oracle
from oracle import ade_ref, numpy_ref


def _block(i0, i1, j0, j1, k0, k1):
    return np.mgrid[i0:i1, j0:j1, k0:k1].reshape(3, -1).T.astype(np.int64)


@pytest.mark.parametrize("materials, steps", [
    ([(0, (2e11, 1e10), _block(2, 5, 2, 5, 2, 5), 1.0), (2, (1e-11, 3.0), _block(6, 9, 6, 9, 6, 9), 2.0),
      (3, (3e11, 5e9, 1.5), _block(2, 5, 6, 9, 7, 10), 1.5)], 70),
    ([(1, (3e11, 5e9, 1.5), _block(3, 6, 3, 6, 3, 6), 1.0), (4, (2e11, 1e10), _block(7, 10, 2, 6, 6, 10), 2.5)], 40),
])
def test_dispersive_grid_restatements_agree_bitwise(materials, steps):
    dims = (12, 11, 13)
    lines = [oracle.uniform_lines(n, d) for n, d in zip(dims, (1.0e-3, 0.8e-3, 1.2e-3))]
    dt, delta = oracle.grid_timestep(*lines)
    s = oracle.OracleSim(*dims, dt, delta)
    c12 = s.coefficients()
    for kind, params, cells, eps_inf in materials:
        s.add_dispersive(kind, params, cells, eps_inf)
    t = (np.arange(steps) - 12.0) / 4.0
    samples = np.exp(-t * t).astype(np.float32)
    exc = [((5, 5, 6), 2, True, samples), ((6, 4, 7), 0, True, -0.5 * samples)]
    for pos, d, soft, smp in exc:
        s.add_excitation_sampled(pos, d, soft, smp)
    s.run_batch(steps)
    zero = np.zeros((6,) + dims, np.float32)
    got = ade_ref.run(c12, zero, steps, dt, materials, exc)
    ref = np.asarray(s.fields(), np.float32).reshape(got.shape)
    assert np.isfinite(ref).all() and np.abs(ref).max() > 0
    assert not np.array_equal(got, numpy_ref.run(c12, zero, steps, exc))  # the media act
    np.testing.assert_array_equal(got, ref)


def test_lumped_rlc_on_a_grid_agrees_bitwise():
    """Parallel and series elements (an element after a dispersive block on
    the same step) against the restatement, fields bit for bit."""
    dims = (12, 11, 13)
    lines = [oracle.uniform_lines(n, d) for n, d in zip(dims, (1.0e-3, 0.8e-3, 1.2e-3))]
    dt, delta = oracle.grid_timestep(*lines)
    s = oracle.OracleSim(*dims, dt, delta)
    c12 = s.coefficients()
    materials = [(0, (2e11, 1e10), _block(7, 10, 6, 9, 2, 5), 1.0)]
    rlc = [((4, 5, 6), 2, 0, 50.0, 1e-9, 1e-12), ((6, 6, 8), 0, 1, 20.0, 2e-9, 5e-13),
           ((5, 3, 4), 1, 0, 0.0, 0.0, 2e-12)]
    for kind, params, cells, eps_inf in materials:
        s.add_dispersive(kind, params, cells, eps_inf)
    for pos, d, t_, r, l, c in rlc:
        s.add_lumped_rlc(pos, d, t_, r, l, c)
    steps = 60
    t = (np.arange(steps) - 12.0) / 4.0
    exc = [((5, 5, 6), 2, True, np.exp(-t * t).astype(np.float32))]
    for pos, d, soft, smp in exc:
        s.add_excitation_sampled(pos, d, soft, smp)
    s.run_batch(steps)
    zero = np.zeros((6,) + dims, np.float32)
    got = ade_ref.run(c12, zero, steps, dt, materials, exc, rlc, delta)
    ref = np.asarray(s.fields(), np.float32).reshape(got.shape)
    assert not np.array_equal(got, ade_ref.run(c12, zero, steps, dt, materials, exc))  # the elements act
    np.testing.assert_array_equal(got, ref)
