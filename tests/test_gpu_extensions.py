"""Dispersive ADE materials, lumped RLC elements and the lumped port on the
CUDA engine against the oracle (bit-exact, through the C ABI)."""
import numpy as np
import pytest

import oracle
import openems_b200 as oe
from scenarios import dispersive_scenarios, run_engine, run_oracle, upml_scenarios
from test_gpu_parity import KERNELS, assert_parity

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("kernels", KERNELS)
@pytest.mark.parametrize("sc", dispersive_scenarios(), ids=lambda s: s.name)
def test_extension_scenarios(sc, kernels):
    assert_parity(run_engine(sc, kernels=kernels), run_oracle(sc))


@pytest.mark.parametrize("kernels", KERNELS)
@pytest.mark.parametrize("sc", upml_scenarios(), ids=lambda s: s.name)
def test_upml_scenarios(sc, kernels):
    """The reference's UPML, bit-exact over short runs (it diverges later)."""
    assert_parity(run_engine(sc, kernels=kernels), run_oracle(sc))


def test_upml_reset_and_graphs():
    sc = upml_scenarios()[0]
    a, b = run_engine(sc, graphs=True), run_engine(sc, graphs=False)
    assert np.array_equal(a["fields"], b["fields"])
    eng = a["engine"]
    eng.reset()
    dt = a["operator"].timestep()
    sched = [oe.ScheduledExcitation.from_excitation(x, 0, sc.num_steps, dt) for x in sc.excitations]
    eng.run_batch(oe.EngineBatch(num_steps=sc.num_steps, excitations=sched))
    e, h = eng.read_fields()
    assert np.array_equal(np.concatenate([e, h]), a["fields"])


def test_compressed_with_dispersive():
    sc = dispersive_scenarios()[0]
    assert_parity(run_engine(sc, compressed=True), run_oracle(sc))


def test_extension_state_resets():
    """Engine.reset clears the ADE and integrator state: a second run from
    zero repeats the first bit for bit."""
    sc = dispersive_scenarios()[3]
    sc.dispersive = dispersive_scenarios()[0].dispersive[:1]
    r = run_engine(sc)
    eng = r["engine"]
    eng.reset()
    dt = r["operator"].timestep()
    sched = [oe.ScheduledExcitation.from_excitation(x, 0, sc.num_steps, dt) for x in sc.excitations]
    eng.run_batch(oe.EngineBatch(num_steps=sc.num_steps, excitations=sched))
    e, h = eng.read_fields()
    assert np.array_equal(np.concatenate([e, h]), r["fields"])


def test_dispersive_graphs_and_direct_agree():
    sc = dispersive_scenarios()[1]
    a, b = run_engine(sc, graphs=True), run_engine(sc, graphs=False)
    assert np.array_equal(a["fields"], b["fields"])


def test_invalid_extension_configs():
    op = oe.Operator(oe.Grid.uniform(8, 8, 8, 1e-3))
    eng = oe.Engine(op)
    with pytest.raises(oe.MaterialError):
        eng.add_dispersive(oe.DrudeMaterial(1e10, 0.0), [(8, 0, 0)])
    with pytest.raises(oe.MaterialError):
        eng.add_dispersive(oe.DrudeMaterial(1e10, 0.0, eps_inf=0.0), [(1, 1, 1)])
    with pytest.raises(oe.ConfigError):
        eng.add_lumped_rlc([oe.RlcElement.resistor((1, 1, 1), 3, 50.0)])
    with pytest.raises(oe.ConfigError):
        eng.add_lumped_rlc([oe.RlcElement.resistor((1, 1, 1), 0, 50.0),
                            oe.RlcElement.resistor((1, 9, 1), 0, 50.0)])
    with pytest.raises(oe.ConfigError):
        op.set_lumped((1, 1, 8), 2, resistance=50.0)


def _port_run(kernels):
    """Lumped 50 ohm port (gaussian-modulated 2-14 GHz) feeding a short
    dipole-like gap in a CPML box; returns engine, port, oracle sim, ids."""
    dims, delta = (24, 24, 30), 1e-3
    pos, d = (12, 12, 15), 2
    freqs = np.linspace(2e9, 14e9, 25)
    op = oe.Operator(oe.Grid.uniform(*dims, delta), oe.BoundaryConditions.all_pec())
    # two short PEC arms on the port's axis
    op.set_pec((12, 13, 12, 13, 9, 15))
    op.set_pec((12, 13, 12, 13, 16, 22))
    port = oe.LumpedPort(1, 50.0, pos, d, excite=1.0).apply(op)
    eng = oe.Engine(op, kernels=kernels)
    eng.add_cpml(oe.CpmlBoundaries.uniform(6))
    port.add_probes(eng, freqs)
    wave = oe.Excitation.gaussian_modulated(8e9, 0.75, d, pos)
    exc = port.excitation(wave)

    lines = [oracle.uniform_lines(n, delta) for n in dims]
    dt, dl = oracle.grid_timestep(*lines)
    s = oracle.OracleSim(*dims, dt, dl)
    s.set_pec((12, 13, 12, 13, 9, 15))
    s.set_pec((12, 13, 12, 13, 16, 22))
    scale = s.set_lumped(pos, d, 50.0, 0.0, 1.0, 0.0)
    assert scale == pytest.approx(port.source_scale, rel=1e-15)
    s.enable_cpml((6,) * 6)
    u = oe.port_probe(op, pos, d, 0)
    i = oe.port_probe(op, pos, d, 1)
    ou = s.add_probe([(c, q, -w) for c, q, w in u.terms], u.mode)
    oi = s.add_probe([(c, q, -w) for c, q, w in i.terms], i.mode)
    du, di = s.add_probe_dft(ou, freqs), s.add_probe_dft(oi, freqs)
    start = 0
    for n in (600, 900):
        eng.run_batch(oe.EngineBatch(num_steps=n, excitations=[
            oe.ScheduledExcitation.from_excitation(exc, start, n, dt)]))
        s.clear_excitations()
        s.add_excitation_analytic(pos, d, True, int(exc.excitation_type), list(exc.params),
                                  exc.amplitude, start, n)
        s.run_batch(n)
        assert np.array_equal(eng.probe_traces(), s.probe_traces())
        start += n
    return eng, port, s, (du, di), freqs


@pytest.mark.parametrize("kernels", KERNELS)
def test_lumped_port_s11(kernels):
    eng, port, s, (du, di), freqs = _port_run(kernels)
    port.calc_port(eng)
    # oracle's DFTs through the same CalcPort arithmetic
    uf, if_ = s.probe_dft(du), s.probe_dft(di)
    assert np.abs(port.uf_tot - uf).max() <= 1e-12 * np.abs(uf).max()
    assert np.abs(port.if_tot - if_).max() <= 1e-12 * np.abs(if_).max()
    s11 = port.s11()
    assert np.all(port.P_inc > 0)
    # passive structure: no more power reflected than incident
    assert np.all(np.abs(s11) <= 1.0 + 1e-3), np.abs(s11)
    assert np.all(port.P_acc >= -1e-6 * port.P_inc)
    # the PEC arms radiate: some power is accepted in band
    assert np.abs(s11).min() < 0.99
    print("|S11| dB:", np.round(20 * np.log10(np.abs(s11)), 2))
