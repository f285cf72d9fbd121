"""The engine interface on the CUDA engine against the oracle.

`openems_b200.EngineInterface` / `EngineInterfaceMut` read and write the
engine's resident fields through oems_engine_sample / _integral / _set_cells.
Every value is compared bit for bit with `oracle.interface_ref` (the scalar
restatement of src/fdtd/engine_interface.rs, pinned to the reference's tests
in tests/test_oracle_interface.py) on the same fields: the reference's tests
replayed through the engine, then seeded fields on a graded grid with a unit,
positions on, between and outside the mesh lines, every interpolation,
integrals in every direction, ordered writes and 2-byte storage.
"""
import numpy as np
import pytest

import openems_b200 as oe
from oracle.interface_ref import EPS0, InterfaceRef

pytestmark = pytest.mark.gpu

N10 = 10
P = [0.005, 0.005, 0.005]


def _uniform_engine(**kw):
    grid = oe.Grid.uniform(N10, N10, N10, 0.001)
    op = oe.Operator(grid, oe.BoundaryConditions.all_pec())
    return grid, op, oe.Engine(op, **kw)


def _zero(dims):
    return np.zeros((3,) + tuple(dims), np.float32), np.zeros((3,) + tuple(dims), np.float32)


def _lines(g):
    return [g.x_lines, g.y_lines, g.z_lines]


# ---- the reference's tests (src/fdtd/engine_interface.rs:597-1213) ----------

def test_reference_tests_through_the_engine():
    grid, op, eng = _uniform_engine()
    e, h = _zero(eng.dims)
    e[:, 5, 5, 5] = [1.0, 2.0, 3.0]
    h[:, 5, 5, 5] = [0.1, 0.2, 0.3]
    eng.write_fields(e, h)
    it = oe.EngineInterface(eng, grid, 1e-12)
    # test_engine_interface_creation, test_set_time, test_dt_accessor, test_dims_accessor
    assert it.timestep() == 0 and it.time() == 0.0 and it.dt() == 1e-12 and it.dims() == (10, 10, 10)
    it.set_time(100, 1e-9)
    assert it.timestep() == 100 and it.time() == 1e-9
    # test_field_access, test_h_field_raw_access
    assert it.get_e_field_raw(5, 5, 5) == [1.0, 2.0, 3.0]
    assert it.get_h_field_raw(5, 5, 5) == [float(np.float32(v)) for v in (0.1, 0.2, 0.3)]
    # test_no_interpolation_mode
    assert it.with_interpolation(oe.InterpolationType.NoInterpolation).get_e_field([0.0055] * 3)[0] == 1.0

    e, h = _zero(eng.dims)
    e[0].fill(1.0)
    h[0].fill(1.0)
    eng.write_fields(e, h)
    # test_energy_calculation, test_interpolation_types, test_h_field_with_interpolation,
    # test_h_field_cell_interpolation
    assert it.calc_fast_energy() > 0.0
    assert it.with_interpolation(oe.InterpolationType.NodeInterpolate).get_e_field(P)[0] > 0.0
    assert it.get_h_field(P)[0] > 0.0
    assert it.with_interpolation(oe.InterpolationType.CellInterpolate).get_h_field(P)[0] > 0.0

    # test_voltage_integral: -0.4 V (the stop snaps to cell 4)
    e[0].fill(100.0)
    eng.write_fields(e, h)
    v = oe.EngineInterface(eng, grid).calc_voltage_integral([0.0, 0.005, 0.005], [0.005, 0.005, 0.005])
    assert v < 0.0 and v == pytest.approx(-0.4, rel=1e-12)

    # test_get_d_field_with_epsilon / _free_space, test_get_b_field_with_mu / _free_space
    e, h = _zero(eng.dims)
    e[0].fill(1.0), e[1].fill(2.0), e[2].fill(3.0)
    h[0].fill(1.0), h[1].fill(2.0), h[2].fill(3.0)
    eng.write_fields(e, h)
    eps = np.full((3, N10, N10, N10), 2.0, np.float32)
    mu = np.full((3, N10, N10, N10), 1.5, np.float32)
    it = oe.EngineInterface(eng, grid, 1e-12).with_epsilon(eps).with_mu(mu)
    assert it.op_eps is not None and it.op_mu is not None
    assert it.get_d_field(P) == [2.0, 4.0, 6.0]
    assert it.get_b_field(P) == [1.5, 3.0, 4.5]
    assert oe.EngineInterface(eng, grid).get_d_field(P)[0] == EPS0
    assert oe.EngineInterface(eng, grid).get_b_field(P)[0] == oe.MU0

    # test_calc_e_energy / test_calc_h_energy
    e[:] = 1.0
    h[:] = 1.0
    eng.write_fields(e, h)
    it = oe.EngineInterface(eng, grid)
    assert it.calc_e_energy() == pytest.approx(0.5 * EPS0 * 3000.0, rel=1e-12)
    assert it.calc_h_energy() == pytest.approx(0.5 * oe.MU0 * 3000.0, rel=1e-12)

    # test_get_j_field, test_get_rot_h_field, test_current_integral_y_normal / _z_normal
    e, h = _zero(eng.dims)
    h[2] = (np.arange(N10, dtype=np.float32) * np.float32(0.1))[None, :, None]
    eng.write_fields(e, h)
    assert any(abs(x) > 0.0 for x in it.get_j_field(P))
    e, h = _zero(eng.dims)
    h[1] = (np.arange(N10, dtype=np.float32) * np.float32(0.1))[None, None, :]
    eng.write_fields(e, h)
    assert any(abs(x) > 0.0 for x in it.get_rot_h_field(P))
    e, h = _zero(eng.dims)
    h[0].fill(1.0), h[2].fill(0.5)
    eng.write_fields(e, h)
    assert it.calc_current_integral([0.0, 0.005, 0.0], [0.005, 0.005, 0.005], 1) == pytest.approx(-0.008, rel=1e-12)
    e, h = _zero(eng.dims)
    h[0].fill(1.0), h[1].fill(0.5)
    eng.write_fields(e, h)
    assert abs(it.calc_current_integral([0.0, 0.0, 0.005], [0.005, 0.005, 0.005], 2)) > 0.0

    # test_cell_interpolation_mode: 5 (node) and 5.5 (cell) at x = 5 mm
    e, h = _zero(eng.dims)
    e[0] = np.arange(N10, dtype=np.float32)[:, None, None]
    eng.write_fields(e, h)
    assert it.with_interpolation(oe.InterpolationType.NodeInterpolate).get_e_field(P)[0] == 5.0
    assert it.with_interpolation(oe.InterpolationType.CellInterpolate).get_e_field(P)[0] == pytest.approx(5.5, abs=1e-12)
    eng.close()


def test_reference_mutable_tests_through_the_engine():
    """test_mutable_interface, test_mutable_add_e_field, test_mutable_set_h_field,
    test_mutable_field_mut_accessors, test_mutable_interface_accessors,
    test_mutable_interface_set_time."""
    grid, op, eng = _uniform_engine()
    m = oe.EngineInterfaceMut(eng, grid, 1e-12)
    m.set_e_field(5, 5, 5, [1.0, 2.0, 3.0])
    e, h = eng.read_fields()
    assert e[:, 5, 5, 5].tolist() == [1.0, 2.0, 3.0]
    m.add_e_field(5, 5, 5, [0.5, 1.0, 1.5])
    assert m.e_field()[:, 5, 5, 5].tolist() == [1.5, 3.0, 4.5]
    m.set_h_field(3, 3, 3, [0.1, 0.2, 0.3])
    assert np.array_equal(m.h_field()[:, 3, 3, 3], np.float32([0.1, 0.2, 0.3]))
    with m.e_field_mut() as ef:
        ef[0, 1, 1, 1] = 5.0
    with m.h_field_mut() as hf:
        hf[1, 2, 2, 2] = 7.0
    e, h = eng.read_fields()
    assert e[0, 1, 1, 1] == 5.0 and h[1, 2, 2, 2] == 7.0 and e[0, 5, 5, 5] == 1.5
    assert m.grid().dimensions() == (10, 10, 10)
    m.set_time(50, 5e-10)
    assert m.timestep == 50 and m.time == 5e-10 and m.dt() == 1e-12
    eng.close()


# ---- seeded fields on a graded grid, bit for bit against the oracle ---------

def _graded(seed=11, storage="f32"):
    rng = np.random.default_rng(seed)
    dims = (13, 9, 17)
    # lines in mm (unit 1e-3), graded cells of 0.5..1.5 mm
    lines = [np.concatenate([[0.0], np.cumsum(rng.uniform(0.5, 1.5, n))]) for n in dims]
    grid = oe.Grid(*lines, unit=1e-3)
    op = oe.Operator(grid, oe.BoundaryConditions.all_pec())
    eng = oe.Engine(op, storage=storage)
    e = rng.standard_normal((3,) + dims).astype(np.float32)
    h = (rng.standard_normal((3,) + dims) * 0.01).astype(np.float32)
    eng.write_fields(e, h)
    e, h = eng.read_fields()  # the stored values (2-byte storage rounds them)
    return rng, grid, eng, e, h


def _queries(rng, grid, n=600):
    """Positions in metres: inside, exactly on mesh lines, below the first
    and past the last line, and NaN."""
    ax_lines = _lines(grid)
    lo = np.array([v[0] for v in ax_lines]) * grid.unit
    hi = np.array([v[-1] for v in ax_lines]) * grid.unit
    p = rng.uniform(lo - 0.1 * (hi - lo), hi + 0.1 * (hi - lo), (n, 3))
    for ax in range(3):
        on = rng.integers(0, len(ax_lines[ax]), n // 4)
        p[: n // 4, ax] = ax_lines[ax][on] * grid.unit
    p[-3:, :] = [[np.nan, 0.0, 0.0], [0.0, np.nan, 0.001], [-1.0, 1.0, np.nan]]
    return p


@pytest.mark.parametrize("storage", ["f32", "f16"])
def test_samples_match_the_oracle(storage):
    rng, grid, eng, e, h = _graded(storage=storage)
    q = _queries(rng, grid)
    eps = rng.uniform(1.0, 5.0, (3,) + eng.dims).astype(np.float32)
    for interp in oe.InterpolationType:
        it = oe.EngineInterface(eng, grid).with_interpolation(interp).with_epsilon(eps)
        ref = InterfaceRef(e, h, _lines(grid), grid.unit, interp=int(interp), eps=eps)
        ev, cells = it.sample(oe._native.SAMPLE_E, q)
        hv = it.h_fields(q)
        dv = it.d_fields(q)
        bv = it.b_fields(q)
        for n in range(q.shape[0]):
            assert tuple(cells[n]) == ref.snap(q[n]), n
            np.testing.assert_array_equal(ev[n], ref.get_e_field(q[n]), err_msg=f"E {interp} {n}")
            np.testing.assert_array_equal(hv[n], ref.get_h_field(q[n]), err_msg=f"H {interp} {n}")
            np.testing.assert_array_equal(dv[n], ref.get_d_field(q[n]), err_msg=f"D {interp} {n}")
            np.testing.assert_array_equal(bv[n], ref.get_b_field(q[n]), err_msg=f"B {interp} {n}")
    it = oe.EngineInterface(eng, grid)
    ref = InterfaceRef(e, h, _lines(grid), grid.unit)
    rv = it.rot_h_fields(q)
    for n in range(q.shape[0]):
        np.testing.assert_array_equal(rv[n], ref.get_rot_h_field(q[n]), err_msg=f"curl H {n}")
    cells = rng.integers(0, eng.dims, (50, 3))
    raw, _ = it.sample(oe._native.SAMPLE_H, cells, cells=True)
    for n, c in enumerate(cells):
        np.testing.assert_array_equal(raw[n], ref.get_h_field_raw(*c))
    eng.close()


def test_integrals_match_the_oracle():
    rng, grid, eng, e, h = _graded(seed=5)
    it = oe.EngineInterface(eng, grid)
    ref = InterfaceRef(e, h, _lines(grid), grid.unit)
    q = _queries(rng, grid, 40)[:-3]
    for n in range(0, len(q) - 1, 2):
        a, b = q[n], q[n + 1]
        assert it.calc_voltage_integral(a, b) == ref.calc_voltage_integral(a, b)
        for normal in (0, 1, 2, 7):
            assert it.calc_current_integral(a, b, normal) == ref.calc_current_integral(a, b, normal)
    assert it.calc_e_energy() == pytest.approx(ref.calc_e_energy(), rel=1e-12)
    assert it.calc_h_energy() == pytest.approx(ref.calc_h_energy(), rel=1e-12)
    assert it.calc_fast_energy() == pytest.approx(ref.calc_fast_energy(), rel=1e-12)
    with pytest.raises(oe.ConfigError):
        it.calc_current_integral(q[0], q[1], -1)
    eng.close()


def test_ordered_writes_match_the_oracle():
    """set / add in list order, a cell named more than once included."""
    rng, grid, eng, e, h = _graded(seed=3)
    ref = InterfaceRef(e.copy(), h.copy(), _lines(grid), grid.unit)
    m = oe.EngineInterfaceMut(eng, grid)
    cells = rng.integers(0, eng.dims, (40, 3))
    cells[10:20] = cells[0]
    vals = rng.standard_normal((40, 3)).astype(np.float32)
    m.add_e_fields(cells, vals)
    m.set_h_fields(cells[::-1], vals)
    for c, v in zip(cells, vals):
        ref.add_e_field(*c, v)
    for c, v in zip(cells[::-1], vals):
        ref.set_h_field(*c, v)
    e2, h2 = eng.read_fields()
    np.testing.assert_array_equal(e2, ref.e)
    np.testing.assert_array_equal(h2, ref.h)
    with pytest.raises(oe.ConfigError):
        m.set_e_field(eng.dims[0], 0, 0, [1.0, 2.0, 3.0])
    eng.close()


def test_probe_evaluated_on_demand():
    """Engine.evaluate_probe: VoltageProbe / CurrentProbe::sample on the
    present fields (the f32 ordered sums) and the f64 integral terms."""
    rng, grid, eng, e, h = _graded(seed=9)
    op = oe.Operator(grid, oe.BoundaryConditions.all_pec())
    for probe in (oe.voltage_probe((1, 2, 3), (1, 2, 12), 2), oe.current_probe((2, 1, 4), (9, 6, 4), 2),
                  oe.voltage_integral(op, (1, 1, 1), (8, 6, 12))):
        want32, want64 = np.float32(0.0), 0.0
        for comp, (i, j, k), w in probe.terms:
            v = (e if comp < 3 else h)[comp % 3, i, j, k]
            want32 = want32 + v if w >= 0 else want32 - v
            want64 = want64 + w * float(v)
        want = float(want32) if probe.mode == 0 else want64
        assert eng.evaluate_probe(probe) == want
    eng.close()


def test_bad_queries_are_refused():
    grid, op, eng = _uniform_engine()
    it = oe.EngineInterface(eng, grid)
    with pytest.raises(oe.InvalidArgumentError):
        it.sample(oe._native.SAMPLE_E, np.zeros((2, 2)))
    with pytest.raises(oe.ConfigError):
        it.sample(oe._native.SAMPLE_E, [[10, 0, 0]], cells=True)
    with pytest.raises(oe.ConfigError):
        oe.EngineInterface(eng, oe.Grid.uniform(9, 10, 10, 0.001))
    eng.close()
