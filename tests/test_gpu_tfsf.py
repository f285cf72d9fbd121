"""TF/SF plane source (src/extensions/tfsf.rs) on the engine against the
oracle, bit for bit: the reference's update (kind 0, whose 1D grid grows
exponentially, so compared over short runs) and the corrected source
(kind 1) with batching, early termination (the host-side 1D grid is
replayed to the executed step), CPML and both polarizations."""
import numpy as np
import pytest

import oracle
import openems_b200 as oe

pytestmark = pytest.mark.gpu


def _pair(dims, cfg, cpml=None):
    lines = [oracle.uniform_lines(n, 1e-3) for n in dims]
    dt, d3 = oracle.grid_timestep(*lines)
    op = oe.Operator(oe.Grid.uniform(*dims, 1e-3), oe.BoundaryConditions.all_pec())
    op.set_material(3.0, 1.0, 0.01, 0.0, (8, 14, 6, 12, 5, 13))
    eng = oe.Engine(op, kernels="register")
    s = oracle.OracleSim(*dims, dt, d3)
    s.set_material(3.0, 1.0, 0.01, 0.0, (8, 14, 6, 12, 5, 13))
    if cpml:
        eng.add_cpml(oe.CpmlBoundaries(layers=cpml))
        s.enable_cpml(cpml)
    eng.add_tfsf(cfg)
    s.enable_tfsf(int(cfg.direction), int(cfg.polarization), cfg.frequency, cfg.amplitude, cfg.boundary_layer,
                  cfg.phase_velocity or 0.0, kind=1 if cfg.corrected else 0)
    return eng, s


def _fields(eng):
    e, h = eng.read_fields()
    return np.concatenate([e, h])


def test_reference_update_two_batches():
    """Kind 0 grows by ~1e5 per 10 steps (as the reference): 2 x 15 steps."""
    cfg = oe.TfsfConfig(oe.PropagationDirection.XPlus, 12e9, 1.0, boundary_layer=5)
    eng, s = _pair((22, 18, 20), cfg)
    for n in (15, 15):
        eng.run_batch(oe.EngineBatch(num_steps=n))
        s.run_batch(n)
    ref = s.fields()
    assert np.all(np.isfinite(ref)) and np.abs(ref).max() > 0
    assert np.array_equal(_fields(eng), ref)


@pytest.mark.parametrize("direction,polarization", [(oe.PropagationDirection.XPlus, oe.Polarization.Transverse1),
                                                    (oe.PropagationDirection.ZPlus, oe.Polarization.Transverse2)])
def test_corrected_source_with_cpml_batches_and_early_stop(direction, polarization):
    cfg = oe.TfsfConfig(direction, 9e9, 2.0, polarization=polarization, boundary_layer=9, corrected=True)
    eng, s = _pair((20, 16, 24), cfg, cpml=(4, 4, 3, 5, 4, 4))
    # a tiny decay threshold ends the first batch at the first check below the peak
    r = eng.run_batch(oe.EngineBatch(num_steps=900, termination=oe.TerminationConfig(
        max_timesteps=900, energy_decay_db=1e-4, check_interval=100),
        energy_monitoring=oe.EnergyMonitorConfig(sample_interval=100, track_peak=True)))
    o = s.run_batch(900, sample_interval=100, track_peak=True, check_interval=100, energy_decay_db=1e-4)
    assert r.timesteps_executed == o["timesteps_executed"]
    print("first batch ended after", r.timesteps_executed, "steps")
    assert np.array_equal(_fields(eng), s.fields())
    for n in (120, 37):
        eng.run_batch(oe.EngineBatch(num_steps=n))
        s.run_batch(n)
    ref = s.fields()
    assert np.all(np.isfinite(ref)) and np.abs(ref).max() > 0.1
    assert np.array_equal(_fields(eng), ref)


def test_tfsf_refusals():
    op = oe.Operator(oe.Grid.uniform(12, 12, 12, 1e-3), oe.BoundaryConditions.all_pec())
    eng = oe.Engine(op)
    with pytest.raises(oe.ConfigError):
        eng.add_tfsf(oe.TfsfConfig(oe.PropagationDirection.YPlus, 1e9, 1.0, boundary_layer=12))
    eng.add_tfsf(oe.TfsfConfig(oe.PropagationDirection.YPlus, 1e9, 1.0, boundary_layer=3))
    with pytest.raises(oe.ConfigError):
        eng.add_tfsf(oe.TfsfConfig(oe.PropagationDirection.YPlus, 1e9, 1.0, boundary_layer=3))
    with pytest.raises(oe.ConfigError):  # the corrected source: positive directions only
        oe.Engine(op).add_tfsf(oe.TfsfConfig(oe.PropagationDirection.YMinus, 1e9, 1.0, boundary_layer=3,
                                             corrected=True))
    half = oe.Engine(op, storage="f16")
    with pytest.raises(oe.ConfigError):
        half.add_tfsf(oe.TfsfConfig(oe.PropagationDirection.YPlus, 1e9, 1.0))
