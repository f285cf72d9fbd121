"""A size-independent property of the update: scaling every source by a
power of two scales every field value by it exactly, since each f32 product
and sum of the step (CPML psi and Mur face state included) scales without a
new rounding.  Checked on the oracle with CPML, a dielectric block and a
lossy block, and with second-order Mur."""
import numpy as np
import pytest

import oracle


def _run(scale, boundary):
    dims = (14, 12, 16)
    lines = [oracle.uniform_lines(n, d) for n, d in zip(dims, (1.0e-3, 0.8e-3, 1.2e-3))]
    dt, delta = oracle.grid_timestep(*lines)
    s = oracle.OracleSim(*dims, dt, delta)
    s.set_material(4.0, 1.0, 0.0, 0.0, (4, 8, 3, 7, 5, 10))
    s.set_material(2.0, 1.0, 0.05, 0.0, (9, 12, 6, 10, 8, 13))
    if boundary == "cpml":
        s.enable_cpml((3, 4, 3, 3, 4, 2))
    else:
        s.enable_mur((1,) * 6, 2)
    steps = 120
    t = (np.arange(steps) - 20.0) / 6.0
    samples = (np.float32(scale) * np.exp(-t * t) * np.sin(0.6 * np.arange(steps))).astype(np.float32)
    s.add_excitation_sampled((7, 6, 8), 2, True, samples)
    s.add_excitation_sampled((6, 5, 9), 0, True, (np.float32(0.5) * samples).astype(np.float32))
    s.run_batch(steps)
    return np.asarray(s.fields(), np.float32)


@pytest.mark.parametrize("boundary", ["cpml", "mur2"])
@pytest.mark.parametrize("k", [-3, 5])
def test_power_of_two_scaling_is_exact(boundary, k):
    base = _run(1.0, boundary)
    scaled = _run(2.0 ** k, boundary)
    assert np.abs(base).max() > 0
    np.testing.assert_array_equal(scaled, base * np.float32(2.0 ** k))
