"""The C++ oracle's uniaxial PML against an independent numpy restatement
(oracle/upml_ref.py): the reference's kind 0 (short runs: it grows without
bound) and the corrected kind 1, regions, flux hooks and the kind-1
coefficient changes bit for bit.  The engine's UPML kernels are checked
against the C++ oracle, so this ties both to the formulas."""
import numpy as np
import pytest

import oracle
from oracle import numpy_ref, upml_ref


@pytest.mark.parametrize("kind, layers, steps", [
    (0, (3, 3, 3, 3, 3, 3), 25),
    (0, (2, 4, 0, 3, 3, 0), 25),
    (1, (3, 3, 3, 3, 3, 3), 80),
    (1, (2, 4, 0, 3, 4, 2), 80),
])
def test_upml_restatements_agree_bitwise(kind, layers, steps):
    dims = (13, 12, 14)
    spacing = (1.0e-3, 0.8e-3, 1.2e-3)
    lines = [oracle.uniform_lines(n, d) for n, d in zip(dims, spacing)]
    dt, delta = oracle.grid_timestep(*lines)
    s = oracle.OracleSim(*dims, dt, delta)
    s.set_material(2.0, 1.0, 0.0, 0.0, (5, 8, 4, 8, 5, 9))
    c12 = s.coefficients()
    s.enable_upml(layers, 3.0, 1e-6, kind)
    t = (np.arange(steps) - 12.0) / 4.0
    samples = np.exp(-t * t).astype(np.float32)
    exc = [((6, 6, 7), 2, True, samples), ((7, 5, 6), 0, True, 0.5 * samples)]
    for pos, d, soft, smp in exc:
        s.add_excitation_sampled(pos, d, soft, smp)
    s.run_batch(steps)
    zero = np.zeros((6,) + dims, np.float32)
    got, c_used = upml_ref.run(c12, zero, steps, dt, delta, layers, 3.0, 1e-6, kind, exc)
    np.testing.assert_array_equal(np.stack(c_used), np.asarray(s.coefficients(), np.float32).reshape(12, *dims))
    ref = np.asarray(s.fields(), np.float32).reshape(got.shape)
    assert np.isfinite(ref).all() and np.abs(ref).max() > 0
    assert not np.array_equal(got, numpy_ref.run(c12, zero, steps, exc))  # the regions act
    np.testing.assert_array_equal(got, ref)


from hypothesis import given, settings, strategies as st  # noqa: E402


@settings(max_examples=10, deadline=None)
@given(dims=st.tuples(st.integers(7, 11), st.integers(7, 11), st.integers(7, 11)),
       layers=st.tuples(*[st.integers(0, 3)] * 6), kind=st.sampled_from([0, 1]))
def test_upml_restatements_agree_on_random_layouts(dims, layers, kind):
    """Random grid sizes, layer counts (absent faces included) and kind;
    short runs (kind 0 grows without bound)."""
    lines = [oracle.uniform_lines(n, d) for n, d in zip(dims, (1.0e-3, 0.9e-3, 1.1e-3))]
    dt, delta = oracle.grid_timestep(*lines)
    s = oracle.OracleSim(*dims, dt, delta)
    c12 = s.coefficients()
    if kind == 1 and max(layers) == 0:
        layers = (2,) + layers[1:]
    s.enable_upml(layers, 3.0, 1e-6, kind)
    steps = 20
    t = (np.arange(steps) - 6.0) / 2.0
    exc = [(tuple(n // 2 for n in dims), 2, True, np.exp(-t * t).astype(np.float32))]
    s.add_excitation_sampled(*exc[0][:3], exc[0][3])
    s.run_batch(steps)
    zero = np.zeros((6,) + dims, np.float32)
    got, c_used = upml_ref.run(c12, zero, steps, dt, delta, layers, 3.0, 1e-6, kind, exc)
    np.testing.assert_array_equal(np.stack(c_used), np.asarray(s.coefficients(), np.float32).reshape(12, *dims))
    np.testing.assert_array_equal(got, np.asarray(s.fields(), np.float32).reshape(got.shape))
