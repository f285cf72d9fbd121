"""The reference's BasicEngine and VectorField3D unit tests
(src/fdtd/basic_engine.rs, src/arrays/field.rs, tests modules), replayed on
the CUDA engine through its public surface (the EngineImpl mirror): a
5 x 5 x 5 grid of 1 mm cells from explicit mesh lines."""
import numpy as np
import pytest

import openems_b200 as oe

pytestmark = pytest.mark.gpu


def _engine():
    """create_test_operator (basic_engine.rs tests): lines 0..5 mm per axis."""
    lines = [0.0, 0.001, 0.002, 0.003, 0.004, 0.005]
    op = oe.Operator(oe.Grid.cartesian(lines, lines, lines), oe.BoundaryConditions.all_pec())
    return op, oe.Engine(op)


def _zero(op):
    nx, ny, nz = op.dimensions()
    return np.zeros((3, nx, ny, nz), dtype=np.float32), np.zeros((3, nx, ny, nz), dtype=np.float32)


def test_engine_creation():
    """test_basic_engine_creation: timestep 0, 5 cells per axis."""
    op, eng = _engine()
    assert eng.current_timestep() == 0
    assert eng.dims == (5, 5, 5)
    eng.close()


def test_engine_reset():
    """test_basic_engine_reset: written fields and the step counter clear."""
    op, eng = _engine()
    e, h = _zero(op)
    e[0, 2, 2, 2] = 1.0
    eng.write_fields(e, h)
    dt = op.timestep()
    eng.run_batch(oe.EngineBatch(num_steps=3, excitations=[]))
    assert eng.current_timestep() == 3
    eng.reset()
    e2, h2 = eng.read_fields()
    assert e2[0, 2, 2, 2] == 0.0 and not np.any(e2) and not np.any(h2)
    assert eng.current_timestep() == 0
    eng.close()


def test_engine_field_access():
    """test_basic_engine_field_access: Ez(2,2,2) = 3 and Hx(1,1,1) = 2 read back."""
    op, eng = _engine()
    e, h = _zero(op)
    e[2, 2, 2, 2] = 3.0
    h[0, 1, 1, 1] = 2.0
    eng.write_fields(e, h)
    e2, h2 = eng.read_fields()
    assert e2[2, 2, 2, 2] == 3.0 and h2[0, 1, 1, 1] == 2.0
    eng.close()


def test_engine_energy():
    """test_basic_engine_energy_computation and test_vector_field: E = 1, 2, 3
    at one cell gives an E energy of 14; H = 2 at another an H energy of 4;
    the total is their sum."""
    op, eng = _engine()
    e, h = _zero(op)
    e[0, 1, 1, 1], e[1, 1, 1, 1], e[2, 1, 1, 1] = 1.0, 2.0, 3.0
    h[1, 3, 3, 3] = 2.0
    eng.write_fields(e, h)
    ee, he = eng.energy()
    assert ee == 14.0 and he == 4.0
    eng.close()


def test_update_touches_the_fields():
    """test_update_h_basic / test_update_e_basic: E at (2,2,2) drives H
    around it, H drives E at interior cells; E stays 0 on the i, j, k = 0
    planes (the E update starts at 1)."""
    op, eng = _engine()
    e, h = _zero(op)
    e[2, 2, 2, 2] = 1.0
    e[1, 2, 2, 2] = 0.5
    eng.write_fields(e, h)
    eng.run_batch(oe.EngineBatch(num_steps=1, excitations=[]))
    e2, h2 = eng.read_fields()
    assert np.any(h2)
    assert not np.any(e2[:, 0, :, :]) and not np.any(e2[:, :, 0, :]) and not np.any(e2[:, :, :, 0])
    eng.close()
