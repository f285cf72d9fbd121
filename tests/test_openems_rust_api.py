"""The reference's Python module surface (src/python/mod.rs) on CPU: names,
arguments, errors and the excitations it builds."""
import math

import pytest

from openems_b200 import fdtd
from openems_b200 import openems_rust as ems


def test_grid_and_constants():
    g = ems.Grid.uniform(10, 20, 30, 1e-3)
    assert g.num_cells() == 6000 and g.cell_size() == pytest.approx((1e-3,) * 3)
    h = ems.Grid.from_lines([0, 1e-3, 3e-3], [0, 2e-3], [0, 1e-3, 2e-3, 3e-3])
    assert h.num_cells() == 2 * 1 * 3 and h.cell_size() == pytest.approx((1e-3, 2e-3, 1e-3))
    assert ems.C0 == 299792458.0 and ems.EPS0 == 8.854187817e-12 and ems.VERSION == "1.0.0"


def test_engine_types_and_boundaries():
    s = ems.OpenEMS(num_timesteps=123)
    assert s.num_timesteps == 123 and ems.OpenEMS().num_timesteps == 10000
    for e in ("gpu", "GPU_V2", "cuda"):
        s.set_engine_type(e)
    for e in ("parallel", "basic", "simd", "quantum"):
        with pytest.raises(RuntimeError):
            s.set_engine_type(e)
    s.set_boundary_cond(["pec", "0", "pml", "pml_6", "mur", "3"])
    assert [f.kind for f in s.faces] == ["pec", "pec", "pml", "pml", "mur", "pml"]
    assert [f.layers for f in s.faces] == [0, 0, 8, 6, 0, 8]
    for bad in (["pec"] * 5, ["pmc"] + ["pec"] * 5, ["pml_x"] + ["pec"] * 5, ["wall"] + ["pec"] * 5):
        with pytest.raises(RuntimeError):
            s.set_boundary_cond(bad)
    with pytest.raises(RuntimeError, match="Grid not set"):
        ems.OpenEMS().run()


def test_excitations_as_the_reference_builds_them():
    """Excitation::gaussian(f0, fc / f0) at the given cell, the centre for
    (0, 0, 0); set_gauss_excite replaces the list."""
    s = ems.OpenEMS()
    s.add_gauss_excite(2e9, 1e9, direction=1, position=(3, 4, 5))
    s.add_gauss_excite(2e9, 1e9)
    a, b = (s._excitation(x, (32, 32, 32)) for x in s.excitations)
    ref = fdtd.Excitation.gaussian(2e9, 0.5, 1, (3, 4, 5))
    assert a.params == ref.params and a.position == (3, 4, 5) and a.direction == 1
    assert b.position == (16, 16, 16) and b.direction == 2
    s.set_gauss_excite(0.0, 4e9)
    assert len(s.excitations) == 1
    c = s._excitation(s.excitations[0], (10, 10, 10))
    tau = 1 / (math.pi * 2e9)
    assert c.params == pytest.approx((4 * tau, tau)) and c.position == (5, 5, 5)


def test_stats_repr():
    st = ems.SimulationStats(100, 1.23456, 789.012, 1.0, 0.5)
    assert repr(st) == "SimulationStats(timesteps=100, wall_time=1.235s, speed=789.01 MC/s)"
