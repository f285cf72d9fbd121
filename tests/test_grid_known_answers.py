"""The reference's grid unit tests for the hot path's inputs (Grid::uniform,
Grid::cartesian, set_unit, cell_size: src/geometry/mod.rs, tests module),
replayed on the Python Grid and on the C++ host operator that builds the
engine's coefficients (oems_operator_create / _create_uniform, whose
dimensions and cell sizes the timestep and coefficients use).  CPU only."""
import numpy as np
import pytest

import openems_b200 as oe


def test_uniform_grid():
    """test_uniform_grid: 10 x 20 x 30 cells of 1 mm."""
    g = oe.Grid.uniform(10, 20, 30, 0.001)
    assert g.dimensions() == (10, 20, 30)
    assert g.cell_size() == pytest.approx((0.001, 0.001, 0.001), abs=1e-10)
    op = oe.Operator(g, oe.BoundaryConditions.all_pec())
    assert op.dimensions() == (10, 20, 30)


def test_cartesian_constructor():
    """test_cartesian_constructor: 4 / 3 / 5 lines give 3 / 2 / 4 cells."""
    g = oe.Grid.cartesian([0.0, 0.001, 0.003, 0.006], [0.0, 0.002, 0.004],
                          [0.0, 0.001, 0.002, 0.003, 0.004])
    assert g.dimensions() == (3, 2, 4)
    op = oe.Operator(g, oe.BoundaryConditions.all_pec())
    assert op.dimensions() == (3, 2, 4)
    # the smallest spacing per axis sets the cell size the timestep uses
    assert g.cell_size() == pytest.approx((0.001, 0.002, 0.001), abs=1e-10)


def test_set_unit_scaling():
    """test_set_unit_scaling: 1-unit cells at unit 1 mm are 1 mm cells."""
    g = oe.Grid.uniform(10, 10, 10, 1.0)
    g.set_unit(0.001)
    assert g.cell_size() == pytest.approx((0.001, 0.001, 0.001), abs=1e-10)
    # the operator scales the lines by the unit: same timestep as 1 mm lines
    dt_unit = oe.Operator(g, oe.BoundaryConditions.all_pec()).timestep()
    dt_mm = oe.Operator(oe.Grid.uniform(10, 10, 10, 0.001), oe.BoundaryConditions.all_pec()).timestep()
    assert dt_unit == pytest.approx(dt_mm, rel=1e-12)


def test_grid_bounds_and_volume():
    """test_grid_bounds (10 x 20 x 30 mm spans) and test_grid_volume (a
    10^3 grid of 1 mm cells holds 1e-6 m^3)."""
    g = oe.Grid.uniform(10, 20, 30, 0.001)
    assert (g.x_lines[0], g.x_lines[-1]) == pytest.approx((0.0, 0.01), abs=1e-10)
    assert (g.y_lines[0], g.y_lines[-1]) == pytest.approx((0.0, 0.02), abs=1e-10)
    assert (g.z_lines[0], g.z_lines[-1]) == pytest.approx((0.0, 0.03), abs=1e-10)
    c = oe.Grid.uniform(10, 10, 10, 0.001)
    volume = float(np.prod([(v[-1] - v[0]) * c.unit for v in (c.x_lines, c.y_lines, c.z_lines)]))
    assert abs(volume - 1e-6) < 1e-15


# ---- src/fdtd/operator.rs tests module: creation, vacuum coefficients, the
# ---- Nyquist step count, the CFL bound and coefficient copies -------------

def _op5():
    """create_test_grid (operator.rs tests): 5 cells of 1 mm per axis."""
    lines = [0.0, 0.001, 0.002, 0.003, 0.004, 0.005]
    return oe.Operator(oe.Grid.cartesian(lines, lines, lines), oe.BoundaryConditions.all_pec())


def test_operator_creation_and_vacuum_coefficients():
    op = _op5()
    assert op.timestep() > 0.0 and op.dimensions() == (5, 5, 5)
    c = op.coefficients()
    for d in range(3):
        assert abs(c[d, 2, 2, 2] - 1.0) < 1e-6          # Ca = 1
        assert c[3 + d, 2, 2, 2] > 0.0                  # Cb = dt / (eps0 delta) > 0
        assert abs(c[6 + d, 2, 2, 2] - 1.0) < 1e-6      # Da = 1
        assert c[9 + d, 2, 2, 2] < 0.0                  # Db carries the minus sign


def test_nyquist_timesteps():
    op = _op5()
    steps = op.nyquist_timesteps(1e9)
    assert steps > 100 and op.nyquist_timesteps(10e9) < steps


def test_timestep_cfl_condition():
    """1 / 2 / 0.5 mm cells: dt below the CFL bound of the three spacings,
    within 10% of it (the 0.99 factor)."""
    g = oe.Grid.cartesian([0.0, 0.001, 0.002, 0.003], [0.0, 0.002, 0.004, 0.006], [0.0, 0.0005, 0.001])
    dt = oe.Operator(g, oe.BoundaryConditions.all_pec()).timestep()
    bound = 1.0 / (oe.C0 * np.sqrt(1.0 / 0.001 ** 2 + 1.0 / 0.002 ** 2 + 1.0 / 0.0005 ** 2))
    assert 0.9 * bound < dt < bound


def test_coefficient_copies():
    """test_e_coefficient_clone / test_h_coefficient_clone: a copied operator
    keeps the coefficients."""
    op = _op5()
    op.set_material(3.0, 2.0, 0.1, 0.0, (1, 4, 1, 4, 1, 4))
    cp = op.clone()
    assert np.array_equal(op.coefficients(), cp.coefficients())



# ---- src/fdtd/timestep.rs and the Simulation's host-side surface -------------

def test_timestep_info():
    """TimestepInfo::calculate: dt = 0.99 of the CFL limit (the operator's
    dt), Nyquist 1 / (2 dt), 18 f32 arrays per cell."""
    g = oe.Grid.cartesian([0.0, 0.001, 0.002, 0.003], [0.0, 0.002, 0.004, 0.006], [0.0, 0.0005, 0.001])
    ti = oe.TimestepInfo.calculate(g)
    assert ti.dt == pytest.approx(0.99 * ti.dt_max, rel=1e-15)
    assert ti.dt == pytest.approx(oe.Operator(g, oe.BoundaryConditions.all_pec()).timestep(), rel=1e-12)
    assert ti.nyquist_freq == pytest.approx(1.0 / (2.0 * ti.dt))
    assert ti.num_cells == 3 * 3 * 2 and ti.memory_bytes == 18 * 18 * 4
    assert ti.timesteps_for_duration(10 * ti.dt) == 10
    assert ti.timesteps_per_period(1.0 / (7 * ti.dt)) == pytest.approx(7.0)
    assert ti.memory_display() == "1.27 KB"
    assert oe.TimestepInfo.calculate(oe.Grid.uniform(2, 2, 2, 1e-3)).memory_display() == "576 B"
    assert oe.TimestepInfo.calculate(oe.Grid.uniform(100, 100, 100, 1e-3)).memory_display() == "68.66 MB"


def test_simulation_builder_on_the_host():
    """The reference's builder chain before setup (no GPU needed): state
    Created, the setters return the simulation, a CPU engine type is
    refused (only the CUDA engine exists)."""
    sim = oe.Simulation(oe.Grid.uniform(8, 8, 8, 1e-3))
    assert sim.state() is oe.SimulationState.Created
    assert sim.set_verbose(0).set_show_progress(False).set_batch_size(None) is sim
    assert sim.set_engine_type(oe.EngineType.Cuda) is sim
    assert sim.timestep_info().dt == pytest.approx(sim.timestep(), rel=1e-12)
