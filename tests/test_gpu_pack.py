"""Packs: several engines stepped by shared launches (oems_pack_*) give each
engine the bits it gets from oems_engine_run_batch on its own, and a packed
sweep equals the per-engine sweep instance by instance."""
import numpy as np
import pytest

import openems_b200 as oe
from openems_b200.sweep import Sweep
from scenarios import cpml_scenarios, make_operator, odd_scenarios, reference_scenarios
from test_gpu_sweep import FREQS, instances

pytestmark = pytest.mark.gpu


def _engine(sc, storage="f32"):
    op = make_operator(sc)
    eng = oe.Engine(op, storage=storage)
    if sc.cpml is not None:
        eng.add_cpml(sc.cpml)
    for comp, pos in sc.probes:
        eng.add_point_probe(comp, pos)
    return op, eng


def _batch(sc, op, start, n, decay=None):
    dt = op.timestep()
    return oe.EngineBatch(num_steps=n,
                          excitations=[oe.ScheduledExcitation.from_excitation(x, start, n, dt)
                                       for x in sc.excitations],
                          termination=oe.TerminationConfig(max_timesteps=n, check_interval=100,
                                                           energy_decay_db=decay),
                          energy_monitoring=oe.EnergyMonitorConfig(sample_interval=50, track_peak=True))


def _mixed():
    """Grids with and without CPML, odd sizes, nz not a multiple of 4."""
    scs = [cpml_scenarios()[0], cpml_scenarios()[1], cpml_scenarios()[2], odd_scenarios()[4],
           reference_scenarios()[2]]
    for sc in scs:
        sc.num_steps = 240
    return scs


@pytest.mark.parametrize("storage", ["f32", "f16"])
def test_pack_equals_separate_engines(storage):
    scs = _mixed()
    alone = [_engine(sc, storage) for sc in scs]
    packed = [_engine(sc, storage) for sc in scs]
    pack = oe.Pack([e for _, e in packed])
    for start, n in ((0, 130), (130, 110)):
        want = [eng.run_batch(_batch(sc, op, start, n)) for sc, (op, eng) in zip(scs, alone)]
        got = pack.run_batch([_batch(sc, op, start, n) for sc, (op, _) in zip(scs, packed)])
        for w, g in zip(want, got):
            assert g.timesteps_executed == w.timesteps_executed
            assert [(s.timestep, s.e_energy, s.h_energy) for s in g.energy_samples] == \
                   [(s.timestep, s.e_energy, s.h_energy) for s in w.energy_samples]
            assert g.peak_energy == w.peak_energy
    for (_, a), (_, b) in zip(alone, packed):
        fa, fb = a.read_fields(), b.read_fields()
        assert np.array_equal(np.concatenate(fa), np.concatenate(fb))
        assert a.current_timestep() == b.current_timestep() == 240
        if a.probe_traces().size:
            assert np.array_equal(a.probe_traces(), b.probe_traces())
    pack.close()


def _decaying():
    """CPML on all faces, on some faces, only on z, and none: with a
    modulated Gaussian each falls 20 dB below its peak at another step."""
    scs = cpml_scenarios()[:3] + [reference_scenarios()[2]]
    for sc in scs:
        sc.excitations = [oe.Excitation.gaussian_modulated(15e9, 0.5, 2, tuple(n // 2 for n in sc.dims))]
    return scs


def test_pack_skips_engines_and_stops_each_at_its_decay():
    """An engine given no batch stays untouched; engines end at their own
    decay checks within one pack batch, as they do alone."""
    scs = _decaying()
    alone = [_engine(sc) for sc in scs]
    packed = [_engine(sc) for sc in scs]
    pack = oe.Pack([e for _, e in packed])
    want = [eng.run_batch(_batch(sc, op, 0, 1500, decay=20.0)) for sc, (op, eng) in zip(scs, alone)]
    got = pack.run_batch([_batch(sc, op, 0, 1500, decay=20.0) for sc, (op, _) in zip(scs, packed)])
    assert len({w.timesteps_executed for w in want}) > 1  # they end at different steps
    for w, g in zip(want, got):
        assert (g.timesteps_executed, g.termination_reason, g.final_decay_db) == \
               (w.timesteps_executed, w.termination_reason, w.final_decay_db)
    for (_, a), (_, b) in zip(alone, packed):
        assert np.array_equal(np.concatenate(a.read_fields()), np.concatenate(b.read_fields()))
    pack.close()
    # an engine given no batch sits it out untouched
    fresh = [_engine(sc) for sc in scs]
    pack = oe.Pack([e for _, e in fresh])
    res = pack.run_batch([_batch(scs[0], fresh[0][0], 0, 50), None, _batch(scs[2], fresh[2][0], 0, 50),
                          _batch(scs[3], fresh[3][0], 0, 50)])
    assert res[1] is None and res[0].timesteps_executed == res[2].timesteps_executed == 50
    assert fresh[1][1].current_timestep() == 0
    assert not np.any(np.concatenate(fresh[1][1].read_fields()))
    pack.close()


@pytest.mark.parametrize("shape", [(128, 2, 0), (512, 16, 0), (256, 4, 1), (128, 8, 1), (128, 4, 2), (256, 2, 3),
                                   None])
def test_pack_shapes_give_the_same_bits(shape):
    """Every launch shape (set, or tuned on the first batch over saved
    state) gives each engine the bits of its own run."""
    scs = _mixed()
    alone = [_engine(sc) for sc in scs]
    packed = [_engine(sc) for sc in scs]
    pack = oe.Pack([e for _, e in packed])
    if shape:
        pack.set_shape(*shape)
    want = [eng.run_batch(_batch(sc, op, 0, 150)) for sc, (op, eng) in zip(scs, alone)]
    got = pack.run_batch([_batch(sc, op, 0, 150) for sc, (op, _) in zip(scs, packed)])
    if shape:
        assert pack.shape() == shape
    else:
        assert pack.shape()[:2] in [(t, c) for t in (128, 256, 512) for c in (2, 4, 8, 16)]
    for w, g in zip(want, got):
        assert [(s.timestep, s.e_energy, s.h_energy) for s in g.energy_samples] == \
               [(s.timestep, s.e_energy, s.h_energy) for s in w.energy_samples]
    for (_, a), (_, b) in zip(alone, packed):
        assert np.array_equal(np.concatenate(a.read_fields()), np.concatenate(b.read_fields()))
        if a.probe_traces().size:
            assert np.array_equal(a.probe_traces(), b.probe_traces())
    with pytest.raises(oe.ConfigError):
        pack.set_shape(100, 4)
    pack.close()


def test_pack_refuses_unsupported_engines():
    sc = cpml_scenarios()[0]
    op = make_operator(sc)
    e = oe.Engine(op, compressed=True)
    with pytest.raises(oe.ConfigError):
        oe.Pack([e])
    f = oe.Engine(op)
    f.add_mur(oe.MurAbcConfig.all(1))
    with pytest.raises(oe.ConfigError):
        oe.Pack([f])
    g = oe.Engine(op)
    with pytest.raises(oe.ConfigError):
        oe.Pack([g, g])


@pytest.mark.parametrize("cap", [None, 1500])
def test_packed_sweep_equals_sweep(cap):
    def run(packed):
        sw = Sweep(FREQS, concurrency=2, packed=packed)
        sw.set_trace_steps(900)
        ids = [sw.add(i) for i in instances()]
        if cap:
            sw.run_until(cap, batch_steps=700)
        else:
            sw.run(batch_steps=700)
        return sw, [sw.result(i) for i in ids], [sw.trace(i) for i in ids]

    _, a, ta = run(False)
    sw, b, tb = run(True)
    for ra, rb, xa, xb in zip(a, b, ta, tb):
        for k in ("timesteps", "termination_reason", "final_decay_db", "paused"):
            assert ra[k] == rb[k], k
        assert np.array_equal(ra["uf"], rb["uf"]) and np.array_equal(ra["if"], rb["if"])
        assert np.array_equal(xa, xb)
    wall, cell_steps = sw.stats()
    assert wall > 0 and cell_steps == sum(r["cells"] * r["timesteps"] for r in b)
    if cap:
        # the paused packed sweep continues to the results of an
        # uninterrupted per-engine sweep
        sw.run(batch_steps=700)
        ref = Sweep(FREQS, concurrency=2)
        rids = [ref.add(i) for i in instances()]
        ref.run(batch_steps=700)
        for iid, rid in zip(range(len(rids)), rids):
            r, f = sw.result(iid), ref.result(rid)
            assert r["timesteps"] == f["timesteps"] and not r["paused"]
            assert np.array_equal(r["uf"], f["uf"]) and np.array_equal(r["if"], f["if"])
