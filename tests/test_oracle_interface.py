"""The engine-interface oracle against the reference's own tests.

Each test below replays one test of src/fdtd/engine_interface.rs (tests
module, :597-1213) on `oracle.interface_ref`, with the reference's fields,
grid (Grid::uniform(10, 10, 10, 0.001)), positions and assertions, so the
restatement is pinned to the reference's expectations.  The GPU engine's
interface is checked against this oracle bit for bit in
tests/test_gpu_engine_interface.py.
"""
import numpy as np
import pytest

from oracle.interface_ref import (CELL_INTERPOLATE, EPS0, MU0, NODE_INTERPOLATE, NO_INTERPOLATION,
                                  InterfaceRef)

N = 10
LINES = [np.arange(N + 1) * 0.001] * 3
P = [0.005, 0.005, 0.005]


def fields():
    return np.zeros((3, N, N, N), np.float32), np.zeros((3, N, N, N), np.float32)


def iface(e, h, **kw):
    return InterfaceRef(e, h, LINES, 1.0, 1e-12, **kw)


def test_engine_interface_creation_and_set_time():
    """test_engine_interface_creation, test_set_time, test_dt_accessor, test_dims_accessor."""
    e, h = fields()
    assert iface(e, h).dt == 1e-12
    assert tuple(iface(e, h).dims) == (10, 10, 10)
    assert InterfaceRef(e, h, LINES, 1.0, 1.5e-12).dt == 1.5e-12


def test_field_access():
    """test_field_access / test_h_field_raw_access."""
    e, h = fields()
    e[:, 5, 5, 5] = [1.0, 2.0, 3.0]
    h[:, 5, 5, 5] = [0.1, 0.2, 0.3]
    ref = iface(e, h)
    assert ref.get_e_field_raw(5, 5, 5) == [1.0, 2.0, 3.0]
    assert np.allclose(ref.get_h_field_raw(5, 5, 5), [0.1, 0.2, 0.3], atol=1e-6)


def test_energy_calculation():
    """test_energy_calculation, test_calc_e_energy, test_calc_h_energy."""
    e, h = fields()
    e[0].fill(1.0)
    assert iface(e, h).calc_fast_energy() > 0.0
    e[:] = 1.0
    assert iface(e, h).calc_e_energy() == pytest.approx(0.5 * EPS0 * 3.0 * 1000.0, rel=1e-12)
    h[:] = 1.0
    assert iface(e, h).calc_h_energy() == pytest.approx(0.5 * MU0 * 3.0 * 1000.0, rel=1e-12)


def test_interpolation_types():
    """test_interpolation_types / test_h_field_with_interpolation / test_h_field_cell_interpolation."""
    e, h = fields()
    e[0].fill(1.0)
    h[0].fill(1.0)
    assert iface(e, h, interp=NODE_INTERPOLATE).get_e_field(P)[0] > 0.0
    assert iface(e, h, interp=NODE_INTERPOLATE).get_h_field(P)[0] > 0.0
    assert iface(e, h, interp=CELL_INTERPOLATE).get_h_field(P)[0] > 0.0
    # a uniform field interpolates to itself
    assert iface(e, h, interp=NODE_INTERPOLATE).get_e_field(P) == [1.0, 0.0, 0.0]


def test_voltage_integral():
    """test_voltage_integral: E_x = 100 V/m from x = 0 to 5 mm.  The stop
    lies on a mesh line, so it snaps to cell 4 and the path has 4 cells."""
    e, h = fields()
    e[0].fill(100.0)
    v = iface(e, h).calc_voltage_integral([0.0, 0.005, 0.005], [0.005, 0.005, 0.005])
    assert v < 0.0
    assert v == pytest.approx(-0.4, rel=1e-12)


def test_mutable_interface():
    """test_mutable_interface, test_mutable_add_e_field, test_mutable_set_h_field,
    test_mutable_field_mut_accessors, test_mutable_interface_accessors."""
    e, h = fields()
    ref = iface(e, h)
    ref.set_e_field(5, 5, 5, [1.0, 2.0, 3.0])
    ref.add_e_field(5, 5, 5, [0.5, 1.0, 1.5])
    assert ref.get_e_field_raw(5, 5, 5) == [1.5, 3.0, 4.5]
    ref.set_h_field(3, 3, 3, [0.1, 0.2, 0.3])
    assert np.allclose(ref.get_h_field_raw(3, 3, 3), [0.1, 0.2, 0.3], atol=1e-6)


def test_d_and_b_fields():
    """test_with_epsilon_coefficient, test_with_mu_coefficient,
    test_get_d_field_with_epsilon / _free_space, test_get_b_field_with_mu / _free_space."""
    e, h = fields()
    e[0].fill(1.0), e[1].fill(2.0), e[2].fill(3.0)
    h[0].fill(1.0), h[1].fill(2.0), h[2].fill(3.0)
    eps = np.full((3, N, N, N), 2.0, np.float32)
    mu = np.full((3, N, N, N), 1.5, np.float32)
    assert iface(e, h, eps=eps).get_d_field(P) == [2.0, 4.0, 6.0]
    assert iface(e, h, mu=mu).get_b_field(P) == [1.5, 3.0, 4.5]
    assert iface(e, h).get_d_field(P)[0] == EPS0
    assert iface(e, h).get_b_field(P)[0] == MU0


def test_j_and_rot_h():
    """test_get_j_field (Hz = 0.1 j) and test_get_rot_h_field (Hy = 0.1 k)."""
    e, h = fields()
    h[2] = (np.arange(N, dtype=np.float32) * np.float32(0.1))[None, :, None]
    j = iface(e, h).get_j_field(P)
    assert any(abs(v) > 0.0 for v in j)
    # at the snapped cell (4, 4, 4): dHz/dy = (Hz[j=5] - Hz[j=4]) in f32 / 1 mm
    assert j[0] == float(h[2, 4, 5, 4] - h[2, 4, 4, 4]) / 0.001
    e, h = fields()
    h[1] = (np.arange(N, dtype=np.float32) * np.float32(0.1))[None, None, :]
    r = iface(e, h).get_rot_h_field(P)
    assert r[0] == 0.0 - float(h[1, 4, 4, 5] - h[1, 4, 4, 4]) / 0.001


def test_current_integrals():
    """test_current_integral_y_normal / _z_normal."""
    e, h = fields()
    h[0].fill(1.0), h[2].fill(0.5)
    i_y = iface(e, h).calc_current_integral([0.0, 0.005, 0.0], [0.005, 0.005, 0.005], 1)
    assert abs(i_y) > 0.0
    # 4 x 4 cells (both ends snap to cell 4) of (Hz dx - Hx dz) = (0.5 - 1) mm
    assert i_y == pytest.approx(16 * (0.5 * 0.001 - 1.0 * 0.001), rel=1e-12)
    e, h = fields()
    h[0].fill(1.0), h[1].fill(0.5)
    assert abs(iface(e, h).calc_current_integral([0.0, 0.0, 0.005], [0.005, 0.005, 0.005], 2)) > 0.0


def test_cell_interpolation_mode():
    """test_cell_interpolation_mode: E_x = i; at the node of cell 4 (the
    reference's scan puts x = 5 mm into cell 4) node interpolation gives
    4 + 1 = 5 (fraction 1), cell interpolation moves half a cell on."""
    e, h = fields()
    e[0] = np.arange(N, dtype=np.float32)[:, None, None]
    cell = iface(e, h, interp=CELL_INTERPOLATE).get_e_field(P)
    node = iface(e, h, interp=NODE_INTERPOLATE).get_e_field(P)
    assert cell[0] > 0.0 and node[0] > 0.0
    assert node[0] == 5.0
    assert cell[0] == pytest.approx(5.5, abs=1e-12)


def test_no_interpolation_mode():
    """test_no_interpolation_mode: 5.5 mm snaps to cell 5."""
    e, h = fields()
    e[0, 5, 5, 5] = 10.0
    assert iface(e, h, interp=NO_INTERPOLATION).get_e_field([0.0055, 0.0055, 0.0055])[0] == 10.0


def test_snap_quirks():
    """Grid::find_cell_x: a coordinate on a line belongs to the lower cell, one
    below the first line or past the last goes to the last cell, and the grid
    unit divides the coordinate first."""
    e, h = fields()
    ref = iface(e, h)
    assert ref.snap([0.003, 0.0, 0.0099]) == (2, 0, 9)
    assert ref.snap([-1e-6, 0.02, float("nan")]) == (9, 9, 9)
    lines = [np.arange(N + 1) * 1.0] * 3
    assert InterfaceRef(e, h, lines, unit=1e-3).snap([0.0045, 0.0, 0.0]) == (4, 0, 0)


# ---- the Python mirror's host-side checks (no library call reached) ----------

class _HostOnlyEngine:
    """Carries what EngineInterface reads on the host: dims and dt."""
    dims = (10, 10, 10)
    dt = 1e-12
    handle = None


def test_mirror_refuses_mismatched_grid_and_bad_shapes():
    import openems_b200 as oe
    eng = _HostOnlyEngine()
    with pytest.raises(oe.ConfigError):
        oe.EngineInterface(eng, oe.Grid.uniform(9, 10, 10, 0.001))
    it = oe.EngineInterface(eng, oe.Grid.uniform(10, 10, 10, 0.001))
    assert it.dt() == 1e-12 and it.dims() == (10, 10, 10) and it.timestep() == 0
    assert it.with_interpolation(oe.InterpolationType.CellInterpolate) is it
    with pytest.raises(oe.InvalidArgumentError):
        it.sample(0, np.zeros((4, 2)))
    with pytest.raises(oe.InvalidArgumentError):
        it.with_epsilon(np.ones((3, 10, 10, 9), np.float32))
    with pytest.raises(oe.ConfigError):
        it.calc_current_integral([0, 0, 0], [1, 1, 1], -1)
    m = oe.EngineInterfaceMut(eng, oe.Grid.uniform(10, 10, 10, 0.001))
    with pytest.raises(oe.InvalidArgumentError):
        m.set_e_fields([[1, 2, 3], [4, 5, 6]], [[1.0, 2.0, 3.0]])
    m.set_time(7, 3e-12)
    assert (m.timestep, m.time, m.dt()) == (7, 3e-12, 1e-12)


def test_integral_terms_agree_with_the_interface_restatement():
    """The host's integral term lists (recorded per step as f64 probes) and
    the interface restatement give the same voltage integral bit for bit;
    the current integrals round each product into the sum, where the
    reference rounds the cell's difference first, so they agree to a few
    ulps of the terms."""
    import openems_b200 as oe
    rng = np.random.default_rng(4)
    lines = [np.concatenate([[0.0], np.cumsum(rng.uniform(0.5e-3, 1.5e-3, n))]) for n in (9, 7, 11)]
    grid = oe.Grid(*lines)
    op = oe.Operator(grid, oe.BoundaryConditions.all_pec())
    e = rng.standard_normal((3, 9, 7, 11)).astype(np.float32)
    h = rng.standard_normal((3, 9, 7, 11)).astype(np.float32)
    ref = InterfaceRef(e, h, lines, 1.0)
    centre = lambda c: [0.5 * (lines[a][c[a]] + lines[a][c[a] + 1]) for a in range(3)]

    def f64_sum(t):
        acc = 0.0
        for comp, (i, j, k), w in t.terms:
            acc += w * float((e if comp < 3 else h)[comp % 3, i, j, k])
        return acc

    for s, t in (((1, 2, 3), (7, 5, 9)), ((8, 0, 10), (0, 6, 0)), ((4, 4, 4), (4, 4, 4))):
        assert f64_sum(oe.voltage_integral(op, s, t)) == ref.calc_voltage_integral(centre(s), centre(t))
        for normal in (0, 1, 2):
            a = f64_sum(oe.current_integral(op, s, t, normal))
            b = ref.calc_current_integral(centre(s), centre(t), normal)
            assert abs(a - b) <= 1e-12 * max(1.0, abs(b)) * 64


def test_vectorised_restatement_agrees_with_the_scalar_one():
    """snap and node interpolation vectorised (searchsorted in place of the
    scan) against the scalar restatement, bit for bit, on a graded grid with
    a unit: positions inside, on mesh lines, outside and NaN."""
    from oracle.interface_ref import node_vec, snap_vec
    rng = np.random.default_rng(8)
    dims = (9, 7, 11)
    lines = [np.concatenate([[0.0], np.cumsum(rng.uniform(0.5, 1.5, n))]) for n in dims]
    unit = 1e-3
    e = rng.standard_normal((3,) + dims).astype(np.float32)
    h = np.zeros_like(e)
    ref = InterfaceRef(e, h, lines, unit, interp=NODE_INTERPOLATE)
    hi = np.array([l[-1] for l in lines]) * unit
    pos = rng.uniform(-0.1 * hi, 1.1 * hi, (400, 3))
    for ax in range(3):
        pos[:100, ax] = lines[ax][rng.integers(0, len(lines[ax]), 100)] * unit
    pos[-2:] = [[np.nan, 0.0, 0.0], [0.0, 0.0, np.nan]]
    cells = snap_vec(lines, unit, dims, pos)
    vals = node_vec(e, lines, unit, dims, pos)
    for n in range(len(pos)):
        assert tuple(cells[n]) == ref.snap(pos[n]), n
        np.testing.assert_array_equal(vals[n], ref.get_e_field(pos[n]), err_msg=str(n))
