"""The reference's probe tests (src/processing/probes.rs tests module)
replayed on the CUDA engine through `openems_b200.processing`, and the
per-step recording against sampling on demand."""
import numpy as np
import pytest

import openems_b200 as oe
from openems_b200.processing import CurrentProbe, FieldProbe, Processing, VoltageProbe

pytestmark = pytest.mark.gpu


def _engine(nx, ny, nz):
    op = oe.Operator(oe.Grid.uniform(nx, ny, nz, 1e-3), oe.BoundaryConditions.all_pec())
    return op, oe.Engine(op)


def _write(eng, fill):
    e = np.zeros((3,) + tuple(eng.dims), np.float32)
    h = np.zeros_like(e)
    fill(e, h)
    eng.write_fields(e, h)


def test_voltage_probes():
    """test_voltage_probe, _x_direction, _y_direction, _multiple_samples,
    _z_direction_single_point."""
    op, eng = _engine(10, 10, 20)
    p = VoltageProbe("test", (5, 5, 0), (5, 5, 10), 2)
    _write(eng, lambda e, h: e[2].fill(1.0))
    p.sample(eng, 0.0)
    assert p.times == [0.0] and p.values == [11.0]
    eng.close()
    op, eng = _engine(10, 10, 10)
    px = VoltageProbe("test_x", (0, 5, 5), (9, 5, 5), 0)
    py = VoltageProbe("test_y", (5, 0, 5), (5, 9, 5), 1)
    _write(eng, lambda e, h: (e[0].fill(2.0), e[1].fill(3.0)))
    px.sample(eng, 1.0e-9)
    py.sample(eng, 2.0e-9)
    assert px.times == [1.0e-9] and px.values == [20.0]
    assert py.times == [2.0e-9] and py.values == [30.0]
    pm = VoltageProbe("test_multi", (5, 5, 0), (5, 5, 4), 2)
    for t, v in ((0.0, 1.0), (1e-9, 2.0), (2e-9, 0.5)):
        _write(eng, lambda e, h: e[2].fill(v))
        pm.sample(eng, t)
    assert pm.values == [5.0, 10.0, 2.5] and len(pm.times) == 3
    ps = VoltageProbe("test_single", (5, 5, 5), (5, 5, 5), 2)
    _write(eng, lambda e, h: e[2].__setitem__((5, 5, 5), 2.5))
    ps.sample(eng, 0.0)
    assert ps.values == [2.5]
    eng.close()


def test_current_probes():
    """test_current_probe, _y_normal, _z_normal, _invalid_direction."""
    op, eng = _engine(10, 20, 20)
    p = CurrentProbe("test_current", (5, 0, 0), (5, 10, 10), 0)
    _write(eng, lambda e, h: h[1].fill(1.0))
    p.sample(eng, 0.0)
    assert p.values == [121.0]
    eng.close()
    op, eng = _engine(10, 10, 10)
    py = CurrentProbe("test_y_normal", (0, 5, 0), (9, 5, 9), 1)
    _write(eng, lambda e, h: (h[2].fill(1.0), h[0].fill(0.5)))
    py.sample(eng, 0.0)
    assert py.values == [50.0]
    pz = CurrentProbe("test_z_normal", (0, 0, 5), (9, 9, 5), 2)
    _write(eng, lambda e, h: (h[0].fill(2.0), h[1].fill(1.0)))
    pz.sample(eng, 0.0)
    assert pz.values == [100.0]
    pi = CurrentProbe("test_invalid", (5, 0, 0), (5, 4, 4), 10)
    _write(eng, lambda e, h: h[1].fill(1.0))
    pi.sample(eng, 0.0)
    assert pi.times == [0.0] and pi.values == [0.0]
    eng.close()


def test_field_probes():
    """test_field_probe, test_field_probe_all_components, test_field_probe_multiple_samples."""
    op, eng = _engine(10, 10, 10)
    p = FieldProbe("test_all", (3, 4, 5))

    def fill(e, h):
        e[:, 3, 4, 5] = [1.0, 2.0, 3.0]
        h[:, 3, 4, 5] = [0.1, 0.2, 0.3]
    _write(eng, fill)
    p.sample(eng, 1e-9)
    assert p.e_values == [(1.0, 2.0, 3.0)]
    assert p.h_values == [tuple(float(np.float32(v)) for v in (0.1, 0.2, 0.3))]
    eng.close()
    op, eng = _engine(5, 5, 5)
    pm = FieldProbe("test_multi", (2, 2, 2))
    for t, (ev, hv) in ((0.0, (1.0, 0.1)), (1e-9, (2.0, 0.2))):
        _write(eng, lambda e, h: (e[0].__setitem__((2, 2, 2), ev), h[0].__setitem__((2, 2, 2), hv)))
        pm.sample(eng, t)
    assert len(pm.times) == 2 and [v[0] for v in pm.e_values] == [1.0, 2.0]
    assert [v[0] for v in pm.h_values] == [float(np.float32(0.1)), float(np.float32(0.2))]
    eng.close()


def test_recorded_steps_match_sampling_on_demand():
    """record / collect: a source drives a 24^3 box for 60 steps; each probe's
    recorded trace ends with the value sampled on the fields after the batch,
    and its times are the step counts times dt."""
    op, eng = _engine(24, 24, 24)
    proc = Processing()
    proc.add_voltage_probe(VoltageProbe("v", (12, 12, 4), (12, 12, 20), 2))
    proc.add_current_probe(CurrentProbe("i", (4, 4, 12), (20, 20, 12), 2))
    proc.add_field_probe(FieldProbe("f", (13, 11, 12)))
    proc.record(eng)
    exc = oe.Excitation.gaussian(6e9, 0.5, 2, (12, 12, 12))
    steps = 60
    eng.run_batch(oe.EngineBatch(num_steps=steps,
                                 excitations=[oe.ScheduledExcitation.from_excitation(exc, 0, steps, op.timestep())]))
    assert proc.collect(eng) == steps
    live = Processing()
    live.add_voltage_probe(VoltageProbe("v", (12, 12, 4), (12, 12, 20), 2))
    live.add_current_probe(CurrentProbe("i", (4, 4, 12), (20, 20, 12), 2))
    live.add_field_probe(FieldProbe("f", (13, 11, 12)))
    live.process(eng, steps * eng.dt)
    for rec, now in ((proc.voltage_probes[0], live.voltage_probes[0]), (proc.current_probes[0], live.current_probes[0])):
        assert len(rec.values) == steps and rec.values[-1] == now.values[0]
        assert rec.times[0] == eng.dt and rec.times[-1] == steps * eng.dt
        assert any(v != 0.0 for v in rec.values)
    f, g = proc.field_probes[0], live.field_probes[0]
    assert f.e_values[-1] == g.e_values[0] and f.h_values[-1] == g.h_values[0]
    eng.close()
