"""CUDA engine vs the oracle (BasicEngine semantics), through the C ABI.

The kernels round every product and sum separately in the reference's order,
so FP32 results must be bit-identical to the FP32 oracle.  The stated gate of
the hot path is a relative L2 error <= 1e-5 per field array (and per probe
trace) after the full step count; the tests assert both, and report the FP32
error against the FP64 accuracy oracle.
"""
import numpy as np
import pytest

import openems_b200 as oe
from conftest import rel_l2
from scenarios import (config1_scenario, cpml_scenarios, mur_scenarios, odd_scenarios, probe_scenario,
                       reference_scenarios, run_engine, run_oracle)

pytestmark = pytest.mark.gpu

REL_L2_GATE = 1e-5
FIELD_NAMES = ("Ex", "Ey", "Ez", "Hx", "Hy", "Hz")


def assert_parity(got, ref, bit_exact=True):
    g, r = got["fields"], ref["fields"]
    assert g.shape == r.shape
    for c in range(6):
        err = rel_l2(g[c], r[c])
        assert err <= REL_L2_GATE, f"{FIELD_NAMES[c]} rel-L2 {err:.3e}"
        if bit_exact:
            diff = np.abs(g[c].astype(np.float64) - r[c].astype(np.float64)).max()
            assert diff == 0.0, f"{FIELD_NAMES[c]} differs from the oracle by {diff:.3e}"
    assert got["timestep"] == ref["timestep"]
    if ref["traces"] is not None:
        assert got["traces"].shape == ref["traces"].shape
        for p in range(ref["traces"].shape[1]):
            assert rel_l2(got["traces"][:, p], ref["traces"][:, p]) <= REL_L2_GATE
        if bit_exact:
            assert np.array_equal(got["traces"], ref["traces"])
    assert len(got["energy"]) == len(ref["energy"])
    for (t1, e1, h1, _), (t2, e2, h2, _) in zip(got["energy"], ref["energy"]):
        assert t1 == t2
        assert e1 == pytest.approx(e2, rel=1e-10, abs=1e-300)
        assert h1 == pytest.approx(h2, rel=1e-10, abs=1e-300)


@pytest.mark.parametrize("kernels", ("auto", "register", "staged"))
def test_config1_64_pec_2000_steps(kernels):
    """64^3 PEC, 2000 steps, soft Gaussian Ez, 4 Ez/Hy probes (bit-exact)."""
    sc = config1_scenario(2000)
    got = run_engine(sc, kernels=kernels)
    ref = run_oracle(sc, precision=32, threads=8)
    assert_parity(got, ref)
    # accuracy against the FP64 oracle, reported and bounded
    ref64 = run_oracle(sc, precision=64, threads=8)
    errs = [rel_l2(got["fields"][c], ref64["fields"][c]) for c in range(6)]
    print("config1 FP32 vs FP64 rel-L2:", ["%.2e" % e for e in errs])
    # per vector field (Hz of an Ez source is ~0 by symmetry: its own relative
    # error is rounding noise)
    assert rel_l2(got["fields"][:3], ref64["fields"][:3]) < 1e-4
    assert rel_l2(got["fields"][3:], ref64["fields"][3:]) < 1e-4


KERNELS = ("register", "staged", "split", "zsplit", "pipe")


@pytest.mark.parametrize("kernels", KERNELS)
@pytest.mark.parametrize("sc", reference_scenarios(), ids=lambda s: s.name)
def test_reference_scenarios(sc, kernels):
    assert_parity(run_engine(sc, kernels=kernels), run_oracle(sc))


@pytest.mark.parametrize("kernels", KERNELS)
@pytest.mark.parametrize("sc", odd_scenarios(), ids=lambda s: s.name)
def test_odd_sizes(sc, kernels):
    assert_parity(run_engine(sc, kernels=kernels), run_oracle(sc))


@pytest.mark.parametrize("kernels", KERNELS)
@pytest.mark.parametrize("sc", cpml_scenarios(), ids=lambda s: s.name)
def test_cpml(sc, kernels):
    assert_parity(run_engine(sc, kernels=kernels), run_oracle(sc))


@pytest.mark.parametrize("kernels", KERNELS)
@pytest.mark.parametrize("sc", mur_scenarios(), ids=lambda s: s.name)
def test_mur(sc, kernels):
    assert_parity(run_engine(sc, kernels=kernels), run_oracle(sc))


@pytest.mark.parametrize("sc", cpml_scenarios() + odd_scenarios()[3:5], ids=lambda s: s.name)
def test_small_grid_default_shape(sc):
    """Without the tuner a small grid gets shorter x-runs (and narrower CTAs)
    so that every SM has a work item; the results stay bit-exact."""
    got = run_engine(sc, autotune=False, kernels="register")
    info = got["engine"].launch_info()
    assert info["ichunk"] < 8 or info["threads"] < 256, info
    assert_parity(got, run_oracle(sc))


# the grids whose CPML leaves a CPML-free box (the thin-z one has none)
@pytest.mark.parametrize("sc", cpml_scenarios()[:3] + [probe_scenario()], ids=lambda s: s.name)
def test_zsplit_forked_default_shape(sc):
    """The untuned z-split forks its CPML slab launch onto a second stream
    beside the plain interior launch (joined by events, inside the graphs
    and in direct launches alike); the results stay bit-exact."""
    got = run_engine(sc, autotune=False, kernels="zsplit")
    assert got["engine"].launch_info()["staged"] == 3
    ref = run_oracle(sc)
    assert_parity(got, ref)
    direct = run_engine(sc, autotune=False, kernels="zsplit", graphs=False)
    assert np.array_equal(direct["fields"], got["fields"])


def test_staged_kernels_are_used_when_requested():
    sc = cpml_scenarios()[0]
    r = run_engine(sc, kernels="staged")
    info = r["engine"].launch_info()
    assert info["staged"] == 1 and info["stages"] >= 2, info


@pytest.mark.parametrize("sc", [reference_scenarios()[2], odd_scenarios()[4], cpml_scenarios()[1]],
                         ids=lambda s: s.name)
def test_compressed_coefficients(sc):
    """Material-id + table storage gives the same bits as the full arrays."""
    assert_parity(run_engine(sc, compressed=True), run_oracle(sc))


def test_graphs_and_direct_launch_agree():
    sc = odd_scenarios()[4]
    a = run_engine(sc, graphs=True)
    b = run_engine(sc, graphs=False, autotune=False)
    assert np.array_equal(a["fields"], b["fields"])
    assert np.array_equal(a["traces"], b["traces"])


def test_reset_and_rerun_is_identical():
    sc = reference_scenarios()[1]
    r = run_engine(sc)
    eng = r["engine"]
    eng.reset()
    assert eng.current_timestep() == 0
    e, h = eng.read_fields()
    assert not e.any() and not h.any()
    dt = r["operator"].timestep()
    sched = [oe.ScheduledExcitation.from_excitation(x, 0, sc.num_steps, dt) for x in sc.excitations]
    eng.run_batch(oe.EngineBatch(num_steps=sc.num_steps, excitations=sched))
    e2, h2 = eng.read_fields()
    assert np.array_equal(np.concatenate([e2, h2]), r["fields"])


def test_write_read_fields_roundtrip_and_continue():
    """write_fields / read_fields round trip, then continuing from injected
    state matches the oracle started from the same state."""
    sc = odd_scenarios()[0]
    rng = np.random.default_rng(7)
    init = rng.standard_normal((6,) + sc.dims).astype(np.float32)
    from scenarios import make_operator
    op = make_operator(sc)
    eng = oe.Engine(op)
    eng.write_fields(init[:3], init[3:])
    e, h = eng.read_fields()
    assert np.array_equal(np.concatenate([e, h]), init)
    eng.run_batch(oe.EngineBatch(num_steps=25))
    e, h = eng.read_fields()
    import oracle
    lines = [oracle.uniform_lines(n, sc.delta) for n in sc.dims]
    dt, delta = oracle.grid_timestep(*lines)
    s = oracle.OracleSim(*sc.dims, dt, delta)
    s.set_fields(init)
    s.run_batch(25)
    assert np.array_equal(np.concatenate([e, h]), s.fields())


def test_energy_decay_termination_matches_oracle():
    """EnergyDecay stop: same step, same decay in dB (basic_engine.rs:117-141)."""
    tau = 1.0 / (np.pi * 20e9)
    sc_cpml = oe.CpmlBoundaries.uniform(6)
    from scenarios import Scenario, make_operator
    sc = Scenario("decay", (24, 24, 24), 1e-3,
                  excitations=[oe.Excitation.gaussian_modulated(10e9, 0.3, 2, (12, 12, 12))],
                  num_steps=3000, cpml=sc_cpml)
    op = make_operator(sc)
    eng = oe.Engine(op)
    eng.add_cpml(sc_cpml)
    dt = op.timestep()
    sched = [oe.ScheduledExcitation.from_excitation(x, 0, 3000, dt) for x in sc.excitations]
    res = eng.run_batch(oe.EngineBatch(
        num_steps=3000, excitations=sched,
        termination=oe.TerminationConfig(max_timesteps=3000, energy_decay_db=30.0, check_interval=50),
        energy_monitoring=oe.EnergyMonitorConfig(sample_interval=10, track_peak=True)))
    import oracle
    lines = [oracle.uniform_lines(n, sc.delta) for n in sc.dims]
    dt_o, delta = oracle.grid_timestep(*lines)
    s = oracle.OracleSim(*sc.dims, dt_o, delta)
    s.enable_cpml((6,) * 6)
    x = sc.excitations[0]
    s.add_excitation_analytic(x.position, 2, True, int(x.excitation_type), list(x.params), 1.0, 0, 3000)
    r = s.run_batch(3000, sample_interval=10, track_peak=True, check_interval=50, energy_decay_db=30.0)
    assert r["termination_reason"] == 1
    assert res.termination_reason == oe.TerminationReason.EnergyDecay
    assert res.timesteps_executed == r["timesteps_executed"] < 3000
    assert res.final_decay_db == pytest.approx(r["final_decay_db"], rel=1e-9)
    assert res.final_decay_db < -30.0
    assert len(res.energy_samples) == len(r["energy_samples"])


def test_nan_is_reported_as_numerical_error():
    """A NaN seeded on the host surfaces as Error::Numerical at the next energy
    sample; nothing on the GPU faults."""
    from scenarios import make_operator
    sc = odd_scenarios()[0]
    eng = oe.Engine(make_operator(sc))
    e = np.zeros((3,) + sc.dims, np.float32)
    h = np.zeros_like(e)
    e[2, 2, 3, 4] = np.nan
    eng.write_fields(e, h)
    with pytest.raises(oe.NumericalError):
        eng.run_batch(oe.EngineBatch(num_steps=10, energy_monitoring=oe.EnergyMonitorConfig(
            sample_interval=5, track_peak=True)))


def test_invalid_configurations_are_rejected():
    from scenarios import make_operator
    sc = odd_scenarios()[0]
    eng = oe.Engine(make_operator(sc))
    with pytest.raises(oe.ConfigError):
        eng.add_point_probe(7, (0, 0, 0))
    with pytest.raises(oe.ConfigError):
        eng.add_point_probe(0, (5, 0, 0))
    bad = oe.ScheduledExcitation((9, 0, 0), 2, True, np.ones(3, np.float32))
    with pytest.raises(oe.ConfigError):
        eng.run_batch(oe.EngineBatch(num_steps=3, excitations=[bad]))
    with pytest.raises(oe.ConfigError):
        eng.add_cpml(oe.CpmlBoundaries(layers=(3, 3, 0, 0, 0, 0)))  # 3 + 3 > nx = 5


def test_simulation_run_api():
    """Simulation::new/run through the C++ host mirror (1000-step batches)."""
    g = oe.Grid.uniform(32, 32, 32, 1e-3)
    sim = oe.Simulation(g, oe.BoundaryConditions.all_pec())
    sim.add_excitation(oe.Excitation.gaussian(5e9, 0.5, 2, (16, 16, 16)))
    sim.set_end_condition(oe.EndCondition.timesteps(2500)).set_verbose(0).set_show_progress(False)
    assert sim.state() is oe.SimulationState.Created
    st = sim.run()
    assert sim.state() is oe.SimulationState.Finished
    with pytest.raises(oe.ConfigError):  # a second run, as in the reference
        sim.run()
    assert st.timesteps == 2500
    assert st.speed_mcells_per_sec > 0
    assert np.isfinite(st.final_energy) and st.final_energy > 0
    # same run on the oracle: final energy agrees
    import oracle
    lines = [oracle.uniform_lines(32, 1e-3)] * 3
    dt, delta = oracle.grid_timestep(*lines)
    s = oracle.OracleSim(32, 32, 32, dt, delta, threads=8)
    x = sim.excitations[0]
    for start in (0, 1000, 2000):
        n = min(1000, 2500 - start)
        s.clear_excitations()
        s.add_excitation_analytic(x.position, 2, True, 0, list(x.params), 1.0, start, n)
        s.run_batch(n, sample_interval=100, track_peak=True)
    e, h = s.energy()
    assert st.final_energy == pytest.approx(e + h, rel=1e-10)


def test_simulation_basic():
    """test_simulation_basic (src/fdtd/simulation.rs tests): 20^3, 100 steps
    of a 1 GHz Gaussian."""
    sim = oe.Simulation(oe.Grid.uniform(20, 20, 20, 1e-3))
    sim.set_end_condition(oe.EndCondition.timesteps(100)).set_verbose(0).set_show_progress(False)
    sim.add_excitation(oe.Excitation.gaussian(1e9, 0.5, 2, (10, 10, 10)))
    sim.setup()
    assert sim.state() is oe.SimulationState.Ready
    st = sim.run()
    assert st.timesteps == 100 and st.speed_mcells_per_sec > 0.0


def test_energy_decay_end_condition_stops_simulation():
    g = oe.Grid.uniform(24, 24, 24, 1e-3)
    sim = oe.Simulation(g, oe.BoundaryConditions.all_pml(6))
    tau = 1.0 / (np.pi * 20e9)
    sim.add_excitation(oe.Excitation.gaussian_modulated(10e9, 0.3, 2, (12, 12, 12)))
    sim.set_end_condition(oe.EndCondition.energy_decay(40.0))
    st = sim.run()
    assert 100 < st.timesteps < 1_000_000
    assert st.final_energy < st.peak_energy * 1e-4


def _all_probes(op):
    return [oe.voltage_probe((3, 9, 12), (17, 9, 12), 0),
            oe.voltage_probe((10, 9, 6), (10, 9, 18), 2),
            oe.current_probe((10, 5, 8), (10, 12, 16), 0),
            oe.current_probe((5, 9, 5), (15, 9, 18), 1),
            oe.voltage_integral(op, (4, 5, 6), (14, 12, 18)),
            oe.current_integral(op, (6, 4, 12), (14, 13, 12), 2),
            oe.port_probe(op, (10, 9, 12), 2, 0),
            oe.port_probe(op, (10, 9, 12), 2, 1),
            oe.port_probe(op, (12, 6, 15), 0, 1)]


@pytest.mark.parametrize("kernels", KERNELS)
def test_probes_and_dft_match_oracle(kernels):
    """f32 probe sums and f64 integrals bit-exact; DFT to 1e-12 (sincos)."""
    from scenarios import probe_scenario, make_operator
    import oracle
    sc = probe_scenario()
    freqs = np.linspace(1e9, 12e9, 23)
    op = make_operator(sc)
    eng = oe.Engine(op, kernels=kernels)
    eng.add_cpml(sc.cpml)
    probes = _all_probes(op)
    pids = [eng.add_probe(p) for p in probes]
    dfts = [eng.add_probe_dft(p, freqs) for p in pids]
    lines = [oracle.uniform_lines(n, sc.delta) for n in sc.dims]
    dt, delta = oracle.grid_timestep(*lines)
    s = oracle.OracleSim(*sc.dims, dt, delta)
    for m in sc.materials:
        s.set_material(*m)
    s.enable_cpml(sc.cpml.layers)
    opids = [s.add_probe(p.terms, p.mode) for p in probes]
    odfts = [s.add_probe_dft(p, freqs) for p in opids]
    start = 0
    for n in sc.batch_sizes():
        sched = [oe.ScheduledExcitation.from_excitation(x, start, n, dt) for x in sc.excitations]
        eng.run_batch(oe.EngineBatch(num_steps=n, excitations=sched))
        s.clear_excitations()
        for x in sc.excitations:
            s.add_excitation_analytic(x.position, x.direction, True, int(x.excitation_type),
                                      list(x.params), 1.0, start, n)
        s.run_batch(n)
        got, ref = eng.probe_traces(), s.probe_traces()
        assert got.shape == ref.shape == (n, len(probes))
        assert np.array_equal(got, ref)
        start += n
    for d, od in zip(dfts, odfts):
        g, r = eng.probe_dft(d), s.probe_dft(od)
        assert np.abs(g - r).max() <= 1e-12 * np.abs(r).max() + 1e-300


def test_corrupted_coefficient_is_reported_as_numerical_error():
    """Fault injection on the host: one coefficient of the operator set to
    NaN before the engine copies it.  The run's energy check sees the
    non-finite energy and the batch ends with NumericalError (no clamping,
    no device fault); the same engine resets and runs on cleanly after the
    field is written again."""
    import ctypes
    from openems_b200 import _native as N
    op = oe.Operator(oe.Grid.uniform(16, 16, 16, 1e-3), oe.BoundaryConditions.all_pec())
    ptrs = (N.PF * 12)()
    N.check(N.lib().oems_operator_coefficients(op.handle, ptrs))
    ca0 = ctypes.cast(ptrs[0], ctypes.POINTER(ctypes.c_float))
    ca0[(8 * 16 + 8) * 16 + 8] = float("nan")  # Ca_x of cell (8, 8, 8)
    eng = oe.Engine(op)
    e = np.zeros((3, 16, 16, 16), np.float32)
    e[0, 8, 8, 8] = 1.0
    eng.write_fields(e, np.zeros_like(e))
    with pytest.raises(oe.NumericalError):
        eng.run_batch(oe.EngineBatch(num_steps=200, excitations=[],
                                     energy_monitoring=oe.EnergyMonitorConfig(sample_interval=10)))
    eng.reset()
    assert eng.current_timestep() == 0 and not np.any(np.concatenate(eng.read_fields()))
    eng.close()
