"""Cylindrical FDTD engine (src/fdtd/cylindrical.rs:393-638) on the GPU
against the oracle, bit for bit: closed and open alpha meshes, a mesh
through R = 0, counters, field write/read and reset, and the reference's
own engine tests.

The reference's update is not stable at its own calculate_timestep(): its
coefficients make vi * iv several hundred per cell, and the fields overflow
to NaN within a few dozen steps.  Parity is therefore checked bit for bit at
a hundredth of that step, where the fields stay finite, and at the full step
with NaN-aware equality (finite values bit-equal, the same cells
non-finite: the device's NaN payload differs from numpy's)."""
import math

import numpy as np
import pytest

from oracle import cylindrical_ref as ref
from openems_b200.cylindrical import CylindricalEngine, CylindricalGrid, CylindricalOperator

pytestmark = pytest.mark.gpu

GRIDS = {
    "closed": (list(np.linspace(0.005, 0.015, 25)), [j * 2 * math.pi / 32 for j in range(33)],
               list(np.linspace(0.0, 0.02, 41))),
    "r0": ([i * 0.0005 for i in range(21)], [j * math.pi / 12 for j in range(25)], [k * 0.0005 for k in range(31)]),
    "open": (list(0.01 + 0.0004 * np.arange(17) ** 1.2), [0.0, 0.1, 0.25, 0.4, 0.5, 0.62, 0.8],
             [0.0, 0.001, 0.003, 0.004, 0.006, 0.0065, 0.008]),
    # z rows of 128 cells or more take the row-tiled kernels (130: a ragged tail block)
    "rows": (list(np.linspace(0.005, 0.013, 9)), [j * 2 * math.pi / 12 for j in range(13)],
             list(np.linspace(0.0, 0.032, 161))),
    "rows_r0_open": ([i * 0.0005 for i in range(9)], [0.0, 0.2, 0.4, 0.6, 0.8, 1.0, 1.2],
                     list(np.linspace(0.0, 0.026, 131))),
}


def _bits(a):
    return np.ascontiguousarray(a, dtype=np.float32).view(np.uint32)


def _same(a, b):
    a, b = np.asarray(a, np.float32), np.asarray(b, np.float32)
    na, nb = np.isnan(a), np.isnan(b)
    return np.array_equal(na, nb) and np.array_equal(_bits(a[~na]), _bits(b[~nb]))


@pytest.mark.parametrize("scale", [0.01, 1.0])
@pytest.mark.parametrize("name", sorted(GRIDS))
def test_engine_matches_oracle(name, scale):
    rho, alpha, z = GRIDS[name]
    g = CylindricalGrid(rho, alpha, z)
    op = CylindricalOperator(g, CylindricalOperator(g, 1.0).calculate_timestep() * scale)
    rng = np.random.default_rng(11)
    shape = g.dimensions()
    e0 = [rng.standard_normal(shape).astype(np.float32) for _ in range(3)]
    h0 = [(rng.standard_normal(shape) * 1e-3).astype(np.float32) for _ in range(3)]
    e, h = [a.copy() for a in e0], [a.copy() for a in h0]
    with CylindricalEngine(op) as eng:
        eng.write_fields(e0, h0)
        with np.errstate(all="ignore"):
            for chunk in (1, 7, 32, 160):
                eng.step(chunk)
                ref.step(e, h, op.vi(), op.iv(), g.closed_alpha, g.r0_included, steps=chunk)
                ge, gh = eng.read_fields()
                for c in range(3):
                    assert _same(ge[c], e[c]), (name, scale, chunk, "E", c)
                    assert _same(gh[c], h[c]), (name, scale, chunk, "H", c)
                if scale < 1.0:
                    assert all(np.isfinite(a).all() for a in ge + gh)
        assert eng.timestep() == 200
        t = 0.0
        for _ in range(200):
            t += op.dt()
        assert eng.time() == t


def test_reference_engine_step_and_reset():
    """test_engine_step / test_engine_reset (src/fdtd/cylindrical.rs:701-735)."""
    g = CylindricalGrid.uniform(0.005, 0.015, 5, 8, 0.0, 0.01, 5)
    op = CylindricalOperator(g, 1e-12)
    with CylindricalEngine(op) as eng:
        assert eng.timestep() == 0 and eng.time() == 0.0
        ez = np.zeros(g.dimensions(), np.float32)
        ez[2, 4, 2] = 1.0
        eng.write_fields(e=[np.zeros_like(ez), np.zeros_like(ez), ez])
        eng.step(10)
        assert eng.timestep() == 10 and eng.time() > 0.0
        e = [np.zeros_like(ez), np.zeros_like(ez), ez.copy()]
        h = [np.zeros_like(ez) for _ in range(3)]
        ref.step(e, h, op.vi(), op.iv(), True, False, steps=10)
        ge, gh = eng.read_fields()
        assert all(np.array_equal(_bits(a), _bits(b)) for a, b in zip(ge + gh, e + h))
        eng.write_fields(e=[np.ones_like(ez)] * 3)
        eng.step()
        eng.reset()
        assert eng.timestep() == 0 and eng.time() == 0.0
        ge, gh = eng.read_fields()
        assert ge[2][2, 2, 2] == 0.0 and all(not a.any() for a in ge + gh)
