"""CPU tests of the C ABI library and the C++ host mirror (no GPU calls).

- the library loads and exports every function include/*.h declares;
- the C++ Operator reproduces the oracle's coefficients bit for bit
  (two independent restatements of src/fdtd/operator.rs:82-263);
- excitation sampling matches the oracle (src/fdtd/batch.rs:110-129);
- without a GPU, engine creation fails loudly with NoDeviceError.
"""
import ctypes
import os
import re

import numpy as np
import pytest

import oracle
import openems_b200 as oe
from openems_b200 import _native as N

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_functions():
    names = set()
    for h in ("include/oems.h", "include/oems_host.h", "include/oems_predictor.h"):
        src = open(os.path.join(ROOT, h)).read()
        names |= set(re.findall(r"OEMS_API\s+[\w\s\*]+?\b(oems_\w+)\s*\(", src))
    return names


def test_library_exports_every_declared_symbol():
    names = declared_functions()
    assert len(names) >= 35
    lib = ctypes.CDLL(N.LIB_PATH)
    missing = [n for n in sorted(names) if not hasattr(lib, n)]
    assert not missing, f"not exported: {missing}"
    # every declared function has a ctypes signature in the binding
    assert names <= set(N.SIGNATURES), sorted(names - set(N.SIGNATURES))


def test_abi_version_and_status_strings():
    assert N.lib().oems_abi_version() == 1
    assert N.lib().oems_status_string(N.ERR_NUMERICAL) == b"numerical error"


@pytest.mark.parametrize("dims,delta,mats,pecs", [
    ((5, 5, 5), 1e-3, [(4.0, 1.0, 0.0, 0.0, (1, 3, 1, 3, 1, 3))], []),
    ((7, 6, 9), 0.37e-3, [(2.0, 1.0, 0.01, 0.0, (0, 7, 2, 5, 1, 8)),
                          (1.0, 4.0, 0.0, 1e6, (3, 6, 0, 6, 0, 4)),
                          (100.0, 10.0, 0.3, 50.0, (2, 4, 2, 4, 2, 4))], [(1, 2, 1, 5, 3, 9)]),
])
def test_operator_matches_oracle_bitwise(dims, delta, mats, pecs):
    op = oe.Operator(oe.Grid.uniform(*dims, delta), oe.BoundaryConditions.all_pec())
    lines = [oracle.uniform_lines(n, delta) for n in dims]
    dt, d3 = oracle.grid_timestep(*lines)
    assert op.timestep() == dt
    assert op.cell_size() == pytest.approx(d3, rel=0, abs=0)
    s = oracle.OracleSim(*dims, dt, d3)
    for m in mats:
        op.set_material(*m)
        s.set_material(*m)
    for r in pecs:
        op.set_pec(r)
        s.set_pec(r)
    assert np.array_equal(op.coefficients(), s.coefficients())


def test_nonuniform_grid_timestep():
    """Operator::calculate_timestep on an anisotropic grid (operator.rs:481-501)."""
    g = oe.Grid([0.0, 0.001, 0.002, 0.003], [0.0, 0.002, 0.004, 0.006], [0.0, 0.0005, 0.001])
    op = oe.Operator(g, oe.BoundaryConditions.all_pec())
    dt_max = 1.0 / (oe.C0 * np.sqrt(1 / 0.001**2 + 1 / 0.002**2 + 1 / 0.0005**2))
    assert dt_max * 0.9 < op.timestep() < dt_max
    assert op.dimensions() == (3, 3, 2)
    dt, _ = oracle.grid_timestep(g.x_lines, g.y_lines, g.z_lines)
    assert op.timestep() == dt


def test_excitation_samples_match_oracle():
    dt = 1.9065748695310057e-12
    cases = [oe.Excitation.gaussian(1e9, 0.5, 2, (1, 1, 1)),
             oe.Excitation.gaussian_modulated(3.5e9, 0.8, 0, (1, 1, 1)),
             oe.Excitation.sinusoidal(3e9, 1, (1, 1, 1)),
             oe.Excitation.dirac(2.0, 2, (1, 1, 1))]
    for x in cases:
        got = x.sample(37, 500, dt)
        ref = np.array([np.float32(oracle.excitation_eval(int(x.excitation_type), list(x.params),
                                                          x.amplitude, (37 + s) * dt))
                        for s in range(500)], dtype=np.float32)
        assert np.array_equal(got, ref)


def test_region_clipping_and_validation():
    op = oe.Operator(oe.Grid.uniform(4, 4, 4, 1e-3), oe.BoundaryConditions.all_pec())
    op.set_material(2.0, 1.0, 0.0, 0.0, (2, 100, 0, 100, 0, 100))  # clipped, no error
    with pytest.raises(oe.MaterialError):
        op.set_material(-1.0, 1.0, 0.0, 0.0, (0, 1, 0, 1, 0, 1))
    # non-finite parameters would put NaN / inf into the coefficients: refused
    before = op.coefficients().copy()
    for bad in ((np.nan, 1.0, 0.0, 0.0), (np.inf, 1.0, 0.0, 0.0), (2.0, np.inf, 0.0, 0.0),
                (2.0, 1.0, np.nan, 0.0), (2.0, 1.0, np.inf, 0.0), (2.0, 1.0, 0.0, np.nan)):
        with pytest.raises(oe.MaterialError):
            op.set_material(*bad, (0, 2, 0, 2, 0, 2))
        with pytest.raises(oe.MaterialError):
            op.set_material_cells(*bad, [(1, 1, 1)])
    assert np.array_equal(op.coefficients(), before)
    with pytest.raises(oe.GridError):
        oe.Operator(oe.Grid([0.0, 1.0, 0.5], [0.0, 1.0], [0.0, 1.0]))


def test_engine_without_gpu_fails_loudly():
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    op = oe.Operator(oe.Grid.uniform(4, 4, 4, 1e-3), oe.BoundaryConditions.all_pec())
    with pytest.raises(oe.NoDeviceError):
        oe.Engine(op)


def test_interface_entry_points_refuse_null_arguments():
    """oems_engine_sample / _integral / _eval_terms / _set_cells check their
    arguments on the host before any device work."""
    L = N.lib()
    d = N.SampleDescC()
    out = N.c_f64()
    three = (N.c_f64 * 3)(0.0, 0.0, 0.0)
    assert L.oems_engine_sample(None, ctypes.byref(d), None, None, 1, None, None) == N.ERR_INVALID_ARGUMENT
    assert L.oems_engine_integral(None, ctypes.byref(d), 0, three, three, 0, ctypes.byref(out)) \
        == N.ERR_INVALID_ARGUMENT
    assert L.oems_engine_eval_terms(None, None, 0, 0, ctypes.byref(out)) == N.ERR_INVALID_ARGUMENT
    assert L.oems_engine_set_cells(None, 0, None, None, 1, 0) == N.ERR_INVALID_ARGUMENT
