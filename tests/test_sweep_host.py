"""Host side of the batched port sweep (no GPU): the seeded patch workload
and the sweep's argument checks."""
import numpy as np
import pytest

import openems_b200 as oe
from openems_b200 import workloads as W
from openems_b200.sweep import Sweep


def test_patch_specs_are_seeded_and_in_range():
    a, b = W.patch_specs(64, seed=4), W.patch_specs(64, seed=4)
    assert a == b
    assert W.patch_specs(8, seed=5) != a[:8]
    for s in a:
        assert all(48 <= n <= 160 for n in s.dims)
        assert 2.2 <= s.eps_r <= 10.2 and 2 <= s.h_cells <= 6
        margin = s.layers + 4
        assert s.x0 >= margin - 1 and s.x0 + s.W <= s.dims[0] - margin + 1
        assert s.y0 >= margin - 1 and s.y0 + s.L <= s.dims[1] - margin + 1
        assert s.x0 <= s.fx < s.x0 + s.W and s.y0 <= s.fy < s.y0 + s.L
        assert s.k_patch + 1 < s.dims[2] - s.layers
    mean_cells = np.mean([s.cells for s in a])
    assert 0.9e6 < mean_cells < 1.8e6


def test_patch_instance_geometry():
    spec = W.PatchSpec((40, 36, 30), 4.4, 3, 14, 12, 13, 12, 20, 16, k_ground=8, layers=6)
    inst = W.patch_sweep_instance(spec)
    c = inst.operator.coefficients()
    kg, kp = spec.k_ground, spec.k_patch
    assert np.all(c[0:6, 10, 10, kg] == 0)                 # ground plane
    assert np.all(c[0:6, 20, 16, kg + 2:kp] == 0)          # feed wire
    assert np.all(c[0:6, 13:27, 12:24, kp] == 0)           # patch
    assert c[5, 20, 16, kg + 1] != 0                        # port edge stays live
    assert c[3, 10, 10, kg + 1] == pytest.approx(c[3, 10, 10, kp + 2] / 4.4, rel=1e-6)


def test_sweep_argument_checks():
    with pytest.raises(oe.ConfigError):
        Sweep([], concurrency=1)
    with pytest.raises(oe.ConfigError):
        Sweep([1e9], concurrency=0)
    sw = Sweep([1e9, 2e9], concurrency=2)
    spec = W.PatchSpec((40, 36, 30), 4.4, 3, 14, 12, 13, 12, 20, 16, k_ground=8, layers=6)
    inst = W.patch_sweep_instance(spec)
    assert sw.add(inst) == 0
    bad = W.patch_sweep_instance(spec)
    bad.port_position = (40, 0, 0)
    with pytest.raises(oe.ConfigError):
        sw.add(bad)
    bad = W.patch_sweep_instance(spec)
    bad.port_resistance = 0.0
    with pytest.raises(oe.ConfigError):
        sw.add(bad)
    with pytest.raises(oe.ConfigError):
        sw.result(0)  # not run yet
    with pytest.raises(oe.ConfigError):
        sw.result(5)
    with pytest.raises(oe.ConfigError):
        sw.finish(0)  # not started
    with pytest.raises(oe.ConfigError):
        sw.finish(-1)
