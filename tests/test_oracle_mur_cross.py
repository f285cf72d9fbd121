"""The C++ oracle's Mur faces against an independent numpy restatement
(oracle/mur_ref.py): first order as the reference's MurAbc, second order on
the face interiors, all faces or some, bit for bit.  The engine's Mur
kernels are checked against the C++ oracle, so this ties both to the
scheme."""
import numpy as np
import pytest

import oracle
from oracle import mur_ref, numpy_ref


@pytest.mark.parametrize("order, enabled, vphase", [
    (1, (1, 1, 1, 1, 1, 1), 0.0),
    (2, (1, 1, 1, 1, 1, 1), 0.0),
    (2, (1, 0, 0, 1, 1, 1), 0.0),
    (1, (0, 1, 1, 0, 1, 0), 2.0e8),
    (2, (1, 1, 0, 1, 0, 1), 2.5e8),
])
def test_mur_restatements_agree_bitwise(order, enabled, vphase):
    dims = (13, 12, 15)
    spacing = (1.0e-3, 0.8e-3, 1.2e-3)
    lines = [oracle.uniform_lines(n, d) for n, d in zip(dims, spacing)]
    dt, delta = oracle.grid_timestep(*lines)
    s = oracle.OracleSim(*dims, dt, delta)
    s.set_material(2.5, 1.0, 0.0, 0.0, (4, 9, 3, 8, 5, 10))
    s.enable_mur(enabled, order, vphase)
    steps = 90
    t = (np.arange(steps) - 18.0) / 5.0
    samples = np.exp(-t * t).astype(np.float32)
    exc = [((6, 6, 7), 2, True, samples), ((7, 5, 8), 1, True, -0.7 * samples)]
    c12 = s.coefficients()
    for pos, d, soft, smp in exc:
        s.add_excitation_sampled(pos, d, soft, smp)
    s.run_batch(steps)
    zero = np.zeros((6,) + dims, np.float32)
    got = mur_ref.run(c12, zero, steps, dt, delta, enabled, order, vphase, exc)
    ref = np.asarray(s.fields(), np.float32).reshape(got.shape)
    assert np.abs(ref).max() > 0
    assert not np.array_equal(got, numpy_ref.run(c12, zero, steps, exc))  # the faces act
    np.testing.assert_array_equal(got, ref)


def test_second_order_interior_changes_the_result():
    """The second-order branch is exercised: on the same run it differs from
    first order."""
    dims = (13, 12, 15)
    lines = [oracle.uniform_lines(n, d) for n, d in zip(dims, (1.0e-3, 0.8e-3, 1.2e-3))]
    dt, delta = oracle.grid_timestep(*lines)
    c12 = oracle.OracleSim(*dims, dt, delta).coefficients()
    t = (np.arange(90) - 18.0) / 5.0
    exc = [((6, 6, 7), 2, True, np.exp(-t * t).astype(np.float32))]
    zero = np.zeros((6,) + dims, np.float32)
    a = mur_ref.run(c12, zero, 90, dt, delta, (1,) * 6, 1, 0.0, exc)
    b = mur_ref.run(c12, zero, 90, dt, delta, (1,) * 6, 2, 0.0, exc)
    assert np.abs(a - b).max() > 1e-3


from hypothesis import given, settings, strategies as st  # noqa: E402


@settings(max_examples=12, deadline=None)
@given(dims=st.tuples(st.integers(7, 12), st.integers(7, 12), st.integers(7, 12)),
       enabled=st.tuples(*[st.integers(0, 1)] * 6), order=st.sampled_from([1, 2]))
def test_mur_restatements_agree_on_random_layouts(dims, enabled, order):
    """Random grid sizes, enabled faces and order."""
    lines = [oracle.uniform_lines(n, d) for n, d in zip(dims, (1.0e-3, 0.9e-3, 1.1e-3))]
    dt, delta = oracle.grid_timestep(*lines)
    s = oracle.OracleSim(*dims, dt, delta)
    s.enable_mur(enabled, order, 0.0)
    c12 = s.coefficients()
    steps = 40
    t = (np.arange(steps) - 8.0) / 3.0
    exc = [(tuple(n // 2 for n in dims), 1, True, np.exp(-t * t).astype(np.float32))]
    s.add_excitation_sampled(*exc[0][:3], exc[0][3])
    s.run_batch(steps)
    zero = np.zeros((6,) + dims, np.float32)
    got = mur_ref.run(c12, zero, steps, dt, delta, enabled, order, 0.0, exc)
    np.testing.assert_array_equal(got, np.asarray(s.fields(), np.float32).reshape(got.shape))
