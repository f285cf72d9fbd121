"""The C++ oracle's TF/SF source against an independent numpy restatement
(oracle/tfsf_ref.py): the reference's kind 0 and the corrected kind 1, every
propagation axis and both polarizations, bit for bit.  The engine's TF/SF
kernel is checked against the C++ oracle, so this ties both to the
formulas."""
import numpy as np
import pytest

import oracle
from oracle import numpy_ref, tfsf_ref


@pytest.mark.parametrize("kind, direction, polarization, layer, vphase", [
    (0, 0, 0, 4, 0.0),
    (0, 2, 1, 3, 0.0),
    (0, 5, 0, 6, 2.2e8),
    (1, 0, 0, 4, 0.0),
    (1, 2, 1, 3, 0.0),
    (1, 4, 0, 5, 2.5e8),
    (1, 4, 1, 2, 0.0),
])
def test_tfsf_restatements_agree_bitwise(kind, direction, polarization, layer, vphase):
    dims = (12, 11, 13)
    spacing = (1.0e-3, 0.8e-3, 1.2e-3)
    lines = [oracle.uniform_lines(n, d) for n, d in zip(dims, spacing)]
    dt, delta = oracle.grid_timestep(*lines)
    s = oracle.OracleSim(*dims, dt, delta)
    s.set_material(2.0, 1.0, 0.0, 0.0, (6, 9, 5, 8, 6, 10))
    c12 = s.coefficients()
    freq, amp, steps = 20e9, 1.5, 60
    s.enable_tfsf(direction, polarization, freq, amp, layer, vphase, kind)
    s.run_batch(steps)
    zero = np.zeros((6,) + dims, np.float32)
    got = tfsf_ref.run(c12, zero, steps, dt, delta, direction, polarization, freq, amp, layer, vphase, kind)
    ref = np.asarray(s.fields(), np.float32).reshape(got.shape)
    assert np.isfinite(ref).all() and np.abs(ref).max() > 0
    assert not np.array_equal(got, numpy_ref.run(c12, zero, steps))
    np.testing.assert_array_equal(got, ref)


from hypothesis import given, settings, strategies as st  # noqa: E402


@settings(max_examples=12, deadline=None)
@given(dims=st.tuples(st.integers(6, 11), st.integers(6, 11), st.integers(6, 11)),
       direction=st.integers(0, 5), polarization=st.integers(0, 1), kind=st.sampled_from([0, 1]),
       layer_frac=st.floats(0.2, 0.8))
def test_tfsf_restatements_agree_on_random_layouts(dims, direction, polarization, kind, layer_frac):
    """Random grid sizes, directions, polarizations and plane positions
    (kind 1 takes the forward directions only, as its set-up requires)."""
    if kind == 1:
        direction -= direction % 2
    n = dims[direction // 2]
    layer = max(1, min(n - 2, int(layer_frac * n)))
    lines = [oracle.uniform_lines(m, d) for m, d in zip(dims, (1.0e-3, 0.9e-3, 1.1e-3))]
    dt, delta = oracle.grid_timestep(*lines)
    s = oracle.OracleSim(*dims, dt, delta)
    c12 = s.coefficients()
    s.enable_tfsf(direction, polarization, 15e9, 1.0, layer, 0.0, kind)
    steps = 35
    s.run_batch(steps)
    zero = np.zeros((6,) + dims, np.float32)
    got = tfsf_ref.run(c12, zero, steps, dt, delta, direction, polarization, 15e9, 1.0, layer, 0.0, kind)
    np.testing.assert_array_equal(got, np.asarray(s.fields(), np.float32).reshape(got.shape))
