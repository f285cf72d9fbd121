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
