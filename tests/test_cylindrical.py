"""Cylindrical FDTD host side (src/fdtd/cylindrical.rs): the reference's own
tests for the grid and operator, the operator's coefficients against the
cell-by-cell oracle bit for bit, the vectorised oracle against the loop
restatement, and the engine's refusals that need no device."""
import math

import numpy as np
import pytest

from oracle import cylindrical_ref as ref
from openems_b200 import _native as N
from openems_b200.cylindrical import CylindricalEngine, CylindricalGrid, CylindricalOperator


# -- the reference's tests (src/fdtd/cylindrical.rs:644-760) ---------------

def test_grid_creation():
    g = CylindricalGrid.uniform(0.001, 0.01, 10, 16, 0.0, 0.02, 20)
    assert (g.n_rho, g.n_alpha, g.n_z) == (10, 16, 20)
    assert g.closed_alpha and not g.r0_included


def test_grid_with_r0():
    g = CylindricalGrid([i * 0.001 for i in range(11)], [i * math.pi / 4 for i in range(9)],
                        [i * 0.002 for i in range(11)])
    assert g.r0_included and g.closed_alpha


def test_cell_volume():
    g = CylindricalGrid.uniform(0.005, 0.015, 10, 16, 0.0, 0.02, 10)
    assert g.get_cell_volume((5, 0, 5)) > 0.0
    assert g.get_cell_volume((9, 0, 5)) > g.get_cell_volume((0, 0, 5))


def test_alpha_wrapping():
    g = CylindricalGrid.uniform(0.005, 0.015, 10, 16, 0.0, 0.02, 10)
    assert g.map_alpha_index(-1) == 15
    assert g.map_alpha_index(16) == 0
    assert g.map_alpha_index(5) == 5
    op = CylindricalGrid([0.01, 0.02], [0.0, 1.0], [0.0, 0.01])
    assert not op.closed_alpha and op.map_alpha_index(-3) == 0 and op.map_alpha_index(7) == 7


def test_operator_size():
    g = CylindricalGrid([0.01, 0.02, 0.03], [0.0, math.pi / 2, math.pi], [0.0, 0.01, 0.02])
    op = CylindricalOperator(g, 1e-12)
    assert op.vv()[0].size == 8
    assert not g.closed_alpha


def test_edge_length_and_area():
    g = CylindricalGrid.uniform(0.005, 0.015, 10, 16, 0.0, 0.02, 10)
    assert g.get_edge_length(1, (9, 0, 0)) > g.get_edge_length(1, (0, 0, 0))
    assert g.get_node_area(2, (5, 0, 5)) > 0.0


# -- coefficients and timestep ---------------------------------------------

GRIDS = {
    "closed": (list(np.linspace(0.005, 0.015, 6)), [j * 2 * math.pi / 8 for j in range(9)],
               list(np.linspace(0.0, 0.01, 6))),
    "r0": ([i * 0.001 for i in range(7)], [j * math.pi / 4 for j in range(9)], [k * 0.002 for k in range(6)]),
    "open": ([0.01, 0.012, 0.015, 0.02, 0.026], [0.0, 0.2, 0.45, 0.7], [0.0, 0.001, 0.003, 0.004, 0.006]),
}


@pytest.mark.parametrize("name", sorted(GRIDS))
def test_coefficients_bit_exact(name):
    rho, alpha, z = GRIDS[name]
    op = CylindricalOperator(CylindricalGrid(rho, alpha, z), 1.3e-12)
    vi, iv = ref.coefficients(rho, alpha, z, 1.3e-12)
    for c in range(3):
        assert np.array_equal(op.vi()[c].view(np.uint32), vi[c].view(np.uint32)), ("vi", c)
        assert np.array_equal(op.iv()[c].view(np.uint32), iv[c].view(np.uint32)), ("iv", c)
        assert np.all(op.vv()[c] == 1.0) and np.all(op.ii()[c] == 1.0)
    g = op.grid()
    assert (g.closed_alpha, g.r0_included) == ref.flags(rho, alpha)
    if name == "r0":  # zero area / length on the axis -> zero coefficient
        assert np.all(op.vi()[0][0] == 0.0) and np.all(op.iv()[1][0] == 0.0) and op.vi_r0 is not None


@pytest.mark.parametrize("name", sorted(GRIDS))
def test_calculate_timestep(name):
    g = CylindricalGrid(*GRIDS[name])
    dt = math.inf
    for i in range(g.n_rho):
        for j in range(g.n_alpha):
            for k in range(g.n_z):
                cs = g.get_cell_size(i, j, k)
                r = max(g.get_radius(i), cs[0] * 0.5)
                dy = r * cs[1]
                dt = min(dt, 1.0 / (299_792_458.0 * math.sqrt(1.0 / (cs[0] * cs[0]) + 1.0 / (dy * dy)
                                                               + 1.0 / (cs[2] * cs[2]))))
    assert CylindricalOperator(g, 1e-12).calculate_timestep() == dt * 0.95


# -- the oracle's two forms agree ------------------------------------------

@pytest.mark.parametrize("name", sorted(GRIDS))
def test_oracle_vectorised_matches_loops(name):
    rho, alpha, z = GRIDS[name]
    closed, r0 = ref.flags(rho, alpha)
    op = CylindricalOperator(CylindricalGrid(rho, alpha, z), 0.5 * CylindricalOperator(
        CylindricalGrid(rho, alpha, z), 1.0).calculate_timestep())
    vi, iv = op.vi(), op.iv()
    rng = np.random.default_rng(7)
    shape = vi[0].shape
    e0 = [rng.standard_normal(shape).astype(np.float32) for _ in range(3)]
    h0 = [(rng.standard_normal(shape) * 1e-3).astype(np.float32) for _ in range(3)]
    ea, ha = [a.copy() for a in e0], [a.copy() for a in h0]
    eb, hb = [a.copy() for a in e0], [a.copy() for a in h0]
    for _ in range(3):
        ref.step_loops(ea, ha, vi, iv, closed, r0)
    ref.step(eb, hb, vi, iv, closed, r0, steps=3)
    for a, b in zip(ea + ha, eb + hb):
        assert np.array_equal(a.view(np.uint32), b.view(np.uint32))
    if r0:
        assert np.all(ea[1][0] == 0.0)


# -- refusals before any device work ---------------------------------------

def test_engine_refuses_bad_grids():
    with pytest.raises(N.GridError):
        CylindricalEngine(CylindricalOperator(CylindricalGrid([0.01, 0.02], [0.0, 1.0], [0.0]), 1e-12))
    with pytest.raises(N.GridError):  # through R = 0 with a single rho cell
        CylindricalEngine(CylindricalOperator(CylindricalGrid([0.0, 0.01], [0.0, 1.0], [0.0, 0.01]), 1e-12))


# -- impulse responses derived by hand from the reference's update lines -----
# update_voltage (src/fdtd/cylindrical.rs:441-486): with E = 0 and one H value
# of 1, E_rho gains +vi where the impulse is the cell's own hz / -vi where it is
# hz(j - 1) ... ; update_current (:540-583) likewise from one E value.

def _impulse_step(g, comp, pos, field):
    op = CylindricalOperator(g, 1e-13)
    shape = g.dimensions()
    e = [np.zeros(shape, np.float32) for _ in range(3)]
    h = [np.zeros(shape, np.float32) for _ in range(3)]
    (h if field == "h" else e)[comp][pos] = 1.0
    ref.step(e, h, op.vi(), op.iv(), g.closed_alpha, g.r0_included)
    return op, e, h


def _expect_only(arrs, expected):
    """Every array zero except the listed (component, index) -> value."""
    for c, a in enumerate(arrs):
        want = np.zeros_like(a)
        for (cc, idx), v in expected.items():
            if cc == c:
                want[idx] += v
        assert np.array_equal(a, want), (c, np.argwhere(a != want)[:4])


CLOSED = CylindricalGrid.uniform(0.005, 0.015, 5, 6, 0.0, 0.01, 5)


def test_voltage_impulse_from_hz_wraps_alpha():
    i, j, k = 2, 5, 2  # j = n_alpha - 1: its j + 1 neighbour is j = 0 on a closed mesh
    op, e, _ = _impulse_step(CLOSED, 2, (i, j, k), "h")
    vi = op.vi()
    _expect_only(e, {(0, (i, j, k)): vi[0][i, j, k], (0, (i, 0, k)): -vi[0][i, 0, k],
                     (1, (i, j, k)): -vi[1][i, j, k], (1, (i + 1, j, k)): vi[1][i + 1, j, k]})


def test_voltage_impulse_from_halpha_and_hrho():
    i, j, k = 2, 3, 2
    op, e, _ = _impulse_step(CLOSED, 1, (i, j, k), "h")
    vi = op.vi()
    _expect_only(e, {(0, (i, j, k)): -vi[0][i, j, k], (0, (i, j, k + 1)): vi[0][i, j, k + 1],
                     (2, (i, j, k)): vi[2][i, j, k], (2, (i + 1, j, k)): -vi[2][i + 1, j, k]})
    op, e, _ = _impulse_step(CLOSED, 0, (i, j, k), "h")
    _expect_only(e, {(1, (i, j, k)): vi[1][i, j, k], (1, (i, j, k + 1)): -vi[1][i, j, k + 1],
                     (2, (i, j, k)): -vi[2][i, j, k], (2, (i, j + 1, k)): vi[2][i, j + 1, k]})


def test_current_impulse_from_ez_and_clamped_edges():
    i, j, k = 2, 0, 2  # j = 0: its j - 1 neighbour is the last alpha cell
    op, e, h = _impulse_step(CLOSED, 2, (i, j, k), "e")
    iv = op.iv()
    _expect_only(e, {(2, (i, j, k)): np.float32(1.0)})  # H was zero: the voltage pass leaves E alone
    _expect_only(h, {(0, (i, j, k)): iv[0][i, j, k], (0, (i, 5, k)): -iv[0][i, 5, k],
                     (1, (i, j, k)): -iv[1][i, j, k], (1, (i - 1, j, k)): iv[1][i - 1, j, k]})
    # at the last rho line the forward neighbour is the cell itself: no H_alpha there from ez
    i = 4
    op, _, h = _impulse_step(CLOSED, 2, (i, 3, k), "e")
    _expect_only(h, {(0, (i, 3, k)): iv[0][i, 3, k], (0, (i, 2, k)): -iv[0][i, 2, k],
                     (1, (i - 1, 3, k)): iv[1][i - 1, 3, k]})


def test_axis_rules():
    g = CylindricalGrid([i * 0.001 for i in range(5)], [j * 2 * math.pi / 6 for j in range(7)],
                        [k * 0.002 for k in range(5)])
    assert g.r0_included
    # hz at the axis: E_rho and E_z curls are zero for i = 0, E_alpha(0) is forced to 0
    op, e, _ = _impulse_step(g, 2, (0, 3, 2), "h")
    vi = op.vi()
    _expect_only(e, {(1, (1, 3, 2)): vi[1][1, 3, 2]})
    # ha at i = 1: E_z(1) gains +vi and E_z(2) -vi (ha(i) - ha(i - 1)), and
    # E_z(0) is then set to E_z(1) / 2
    op, e, _ = _impulse_step(g, 1, (1, 3, 2), "h")
    ez1 = vi[2][1, 3, 2]
    _expect_only(e, {(0, (1, 3, 2)): -vi[0][1, 3, 2], (0, (1, 3, 3)): vi[0][1, 3, 3],
                     (2, (1, 3, 2)): ez1, (2, (2, 3, 2)): -vi[2][2, 3, 2],
                     (2, (0, 3, 2)): np.float32(ez1 * np.float32(0.5))})
