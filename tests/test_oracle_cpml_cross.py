"""The C++ oracle's CPML against an independent numpy restatement
(oracle/cpml_ref.py, written from src/extensions/cpml.rs:68-155 and the two
corrections this project applies).  Profiles and fields must agree bit for
bit: the engine's CPML kernels are checked against the C++ oracle, so this
ties both to the formulas."""
import numpy as np
import pytest

import oracle
from oracle import cpml_ref, numpy_ref


def _sim(layers, alpha_max=0.0, kappa_max=1.0, steps=70):
    dims = (14, 11, 16)
    spacing = (1.0e-3, 0.8e-3, 1.2e-3)
    lines = [oracle.uniform_lines(n, d) for n, d in zip(dims, spacing)]
    dt, delta = oracle.grid_timestep(*lines)
    s = oracle.OracleSim(*dims, dt, delta)
    s.set_material(3.0, 1.0, 0.02, 0.0, (5, 9, 3, 7, 6, 11))
    s.enable_cpml(layers, 3.0, 1e-6, alpha_max, kappa_max)
    t = (np.arange(steps) - 20.0) / 6.0
    samples = (np.exp(-t * t) * np.sin(0.7 * np.arange(steps))).astype(np.float32)
    exc = [((7, 5, 8), 2, True, samples), ((6, 6, 7), 0, True, 0.5 * samples)]
    c12 = s.coefficients()
    for pos, d, soft, smp in exc:
        s.add_excitation_sampled(pos, d, soft, smp)
    s.run_batch(steps)
    return s, c12, dt, delta, exc


@pytest.mark.parametrize("layers, alpha_max, kappa_max", [
    ((4, 4, 3, 3, 5, 5), 0.0, 1.0),
    ((3, 5, 0, 4, 6, 2), 0.05, 4.0),
    ((2, 0, 3, 3, 0, 4), 0.0, 2.5),
])
def test_cpml_restatements_agree_bitwise(layers, alpha_max, kappa_max):
    steps = 70
    s, c12, dt, delta, exc = _sim(layers, alpha_max, kappa_max, steps)
    zero = np.zeros((6,) + s.shape, np.float32)
    fields, profs = cpml_ref.run(c12, zero, steps, dt, delta, layers, 3.0, 1e-6, alpha_max, kappa_max, exc)
    for f in range(6):
        got = s.cpml_profile(f)
        if profs[f] is None:
            assert got["b_e"].size == 0
            continue
        for k, v in profs[f].items():
            np.testing.assert_array_equal(got[k].astype(np.float32), v, err_msg=f"face {f} {k}")
    ref = s.fields()
    assert np.abs(ref).max() > 0
    # the slabs act: the same run without them differs
    assert not np.array_equal(fields, numpy_ref.run(c12, zero, steps, exc))
    np.testing.assert_array_equal(fields, np.asarray(ref, np.float32).reshape(fields.shape))


from hypothesis import given, settings, strategies as st  # noqa: E402


@settings(max_examples=12, deadline=None)
@given(dims=st.tuples(st.integers(6, 12), st.integers(6, 12), st.integers(6, 12)),
       layers=st.tuples(*[st.integers(0, 4)] * 6),
       alpha=st.sampled_from([0.0, 0.02]), kappa=st.sampled_from([1.0, 3.0]))
def test_cpml_restatements_agree_on_random_layouts(dims, layers, alpha, kappa):
    """Random grid sizes and per-face layer counts (absent faces included)."""
    if max(layers) == 0:
        layers = (1,) + layers[1:]
    for a in range(3):  # both faces of an axis must fit the axis
        if layers[2 * a] + layers[2 * a + 1] > dims[a]:
            layers = layers[:2 * a] + (1, 1) + layers[2 * a + 2:]
    lines = [oracle.uniform_lines(n, d) for n, d in zip(dims, (1.0e-3, 0.9e-3, 1.1e-3))]
    dt, delta = oracle.grid_timestep(*lines)
    s = oracle.OracleSim(*dims, dt, delta)
    s.enable_cpml(layers, 3.0, 1e-6, alpha, kappa)
    c12 = s.coefficients()
    steps = 30
    t = (np.arange(steps) - 8.0) / 3.0
    pos = tuple(n // 2 for n in dims)
    exc = [(pos, 2, True, np.exp(-t * t).astype(np.float32))]
    s.add_excitation_sampled(*exc[0][:3], exc[0][3])
    s.run_batch(steps)
    zero = np.zeros((6,) + dims, np.float32)
    fields, _ = cpml_ref.run(c12, zero, steps, dt, delta, layers, 3.0, 1e-6, alpha, kappa, exc)
    np.testing.assert_array_equal(fields, np.asarray(s.fields(), np.float32).reshape(fields.shape))
