"""Field dumps from an engine's device buffers into the binary container and
VTK, read back exactly."""
import numpy as np
import pytest

import openems_b200 as oe
from openems_b200 import field_io as F

pytestmark = pytest.mark.gpu


def _engine():
    op = oe.Operator(oe.Grid.uniform(12, 10, 14, 1e-3), oe.BoundaryConditions.all_pec())
    eng = oe.Engine(op, kernels="register")
    exc = oe.Excitation.gaussian_modulated(20e9, 0.5, 2, (6, 5, 7))
    dt = op.timestep()
    return op, eng, exc, dt


def test_dump_fields_roundtrip(tmp_path):
    op, eng, exc, dt = _engine()
    eng.run_batch(oe.EngineBatch(num_steps=60, excitations=[oe.ScheduledExcitation.from_excitation(exc, 0, 60, dt)]))
    e, h = eng.read_fields()
    assert np.abs(e).max() > 0
    F.dump_fields(eng, op.grid, tmp_path / "snap.oems", timestep=60 * dt)
    r = F.Hdf5Reader.open(tmp_path / "snap.oems")
    assert r.dimensions() == (12, 10, 14) and list(r.timesteps) == [60 * dt]
    for k, c in enumerate(r.vector_fields["E-Field"]):
        assert np.array_equal(c, e[k].ravel())
    for k, c in enumerate(r.vector_fields["H-Field"]):
        assert np.array_equal(c, h[k].ravel())
    F.dump_fields(eng, op.grid, tmp_path / "snap", fmt="vtk")
    lines = (tmp_path / "snap_E.vtk").read_text().splitlines()
    vals = np.array([[np.float32(v) for v in s.split()] for s in lines[lines.index("VECTORS E-Field float") + 1:]])
    assert np.array_equal(vals.T, e.reshape(3, -1))


def test_dump_field_dft(tmp_path):
    op, eng, exc, dt = _engine()
    freqs = [15e9, 20e9]
    d = eng.add_field_dft((2, 10, 2, 8, 3, 11), freqs, components="E")
    eng.run_batch(oe.EngineBatch(num_steps=80, excitations=[oe.ScheduledExcitation.from_excitation(exc, 0, 80, dt)]))
    F.dump_field_dft(eng, d, freqs, (0, 1, 2), tmp_path / "fd.oems")
    r = F.Hdf5Reader.open(tmp_path / "fd.oems")
    assert list(r.frequencies) == freqs
    for fi in range(2):
        for c, name in enumerate(("Ex", "Ey", "Ez")):
            assert np.array_equal(r.complex_fields[f"{name}_f{fi}"], eng.field_dft(d, fi, c).ravel())
    assert np.abs(r.complex_fields["Ez_f1"]).max() > 0
