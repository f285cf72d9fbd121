"""Checkpoint / resume on the engine: a run saved after its first batch and
loaded into a freshly built engine (or into the same engine after a reset)
continues bit for bit -- fields and probe traces -- with CPML, dispersive
media, Mur, lumped RLC, a TF/SF source and 2-byte field storage; a
checkpoint refused by an engine built differently leaves it untouched."""
import numpy as np
import pytest

import openems_b200 as oe
from scenarios import dispersive_scenarios, make_operator

pytestmark = pytest.mark.gpu


def _engine(sc, **kw):
    """The engine of a scenario, extensions attached in run_engine's order."""
    op = make_operator(sc)
    eng = oe.Engine(op, kernels="register", **kw)
    if sc.cpml is not None:
        eng.add_cpml(sc.cpml)
    if sc.mur is not None:
        eng.add_mur(sc.mur)
    for mat, cells in sc.dispersive:
        eng.add_dispersive(mat, cells)
    if sc.rlc:
        eng.add_lumped_rlc(sc.rlc)
    for comp, pos in sc.probes:
        eng.add_point_probe(comp, pos)
    return eng, op.timestep()


def _batch(eng, sc, dt, start, n):
    sched = [oe.ScheduledExcitation.from_excitation(x, start, n, dt) for x in sc.excitations]
    eng.run_batch(oe.EngineBatch(num_steps=n, excitations=sched))
    e, h = eng.read_fields()
    return np.concatenate([e, h]), (eng.probe_traces() if sc.probes else None)


def _same(a, b):
    fa, ta = a
    fb, tb = b
    assert np.array_equal(fa, fb)
    assert (ta is None and tb is None) or np.array_equal(ta, tb)


@pytest.mark.parametrize("name", ["drude_debye_cpml", "lumped_rlc"])
def test_resume_in_fresh_engine_and_after_reset(name):
    sc = {s.name: s for s in dispersive_scenarios()}[name]
    a, dt = _engine(sc)
    _batch(a, sc, dt, 0, 60)
    blob = a.save_state()
    kinds = [k for k, _, _ in a.state_sections()]
    assert kinds[0] == 1  # the fields come first
    assert (2 in kinds) == (sc.cpml is not None) and (3 in kinds) == (sc.mur is not None)
    assert kinds.count(5) == len(sc.dispersive) and (6 in kinds) == bool(sc.rlc)
    want = _batch(a, sc, dt, 60, 70)
    b, _ = _engine(sc)
    b.load_state(blob)
    assert b.current_timestep() == 60
    _same(_batch(b, sc, dt, 60, 70), want)
    a.reset()
    a.load_state(blob)
    _same(_batch(a, sc, dt, 60, 70), want)
    assert a.current_timestep() == 130


def test_resume_tfsf_with_cpml():
    cfg = oe.TfsfConfig(oe.PropagationDirection.XPlus, 9e9, 2.0, polarization=oe.Polarization.Transverse1,
                        boundary_layer=9, corrected=True)

    def build():
        op = oe.Operator(oe.Grid.uniform(20, 16, 24, 1e-3), oe.BoundaryConditions.all_pec())
        op.set_material(3.0, 1.0, 0.01, 0.0, (8, 14, 6, 12, 5, 13))
        eng = oe.Engine(op, kernels="register")
        eng.add_cpml(oe.CpmlBoundaries(layers=(4, 4, 3, 5, 4, 4)))
        eng.add_tfsf(cfg)
        return eng

    def fields(eng):
        e, h = eng.read_fields()
        return np.concatenate([e, h])

    a = build()
    a.run_batch(oe.EngineBatch(num_steps=50))
    blob = a.save_state()
    assert [k for k, _, _ in a.state_sections()][-2:] == [10, 11]
    a.run_batch(oe.EngineBatch(num_steps=40))
    want = fields(a)
    assert np.abs(want).max() > 0
    b = build()
    b.load_state(blob)
    b.run_batch(oe.EngineBatch(num_steps=40))
    assert np.array_equal(fields(b), want)


def test_resume_half_storage():
    sc = {s.name: s for s in dispersive_scenarios()}["drude_debye_cpml"]
    sc.dispersive, sc.probes = [], []
    a, dt = _engine(sc, storage="f16")
    _batch(a, sc, dt, 0, 80)
    blob = a.save_state()
    want = _batch(a, sc, dt, 80, 60)
    b, _ = _engine(sc, storage="f16")
    b.load_state(blob)
    _same(_batch(b, sc, dt, 80, 60), want)
    c, _ = _engine(sc)  # float storage: fields section twice the size
    before = _batch(c, sc, dt, 0, 5)[0]
    with pytest.raises(oe.ConfigError):
        c.load_state(blob)
    e, h = c.read_fields()
    assert np.array_equal(np.concatenate([e, h]), before) and c.current_timestep() == 5
    # bfloat16 fields have the half section's size: the storage variant
    # refuses the snapshot, in the blob check and in the C entry point
    d, _ = _engine(sc, storage="bf16")
    before = _batch(d, sc, dt, 0, 5)[0]
    assert d.state_sections()[0][:2] == b.state_sections()[0][:2]
    assert (d.state_sections()[0][2], b.state_sections()[0][2]) == (2, 1)
    with pytest.raises(oe.ConfigError, match="variant"):
        d.load_state(blob)
    from openems_b200 import checkpoint
    fields_bytes = checkpoint.parse(blob).sections[0][1]
    with pytest.raises(oe.ConfigError):
        d.write_state(0, fields_bytes, variant=1)
    e, h = d.read_fields()
    assert np.array_equal(np.concatenate([e, h]), before) and d.current_timestep() == 5
