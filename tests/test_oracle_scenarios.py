"""The reference's scenario physics checks (src/fdtd/engine_testing.rs:782-1700)
replayed on the oracle, plus self-consistency of the oracle (CPU).

- the numpy restatement agrees with the C++ oracle bit for bit;
- the OpenMP restatement of the parallel engine gives identical bits;
- FP32 stays close to the FP64 accuracy oracle;
- splitting a run into batches does not change the result.
"""
import numpy as np
import pytest

import oracle
from oracle import numpy_ref
from conftest import rel_l2
from scenarios import make_operator, reference_scenarios, odd_scenarios, run_oracle

SC = {s.name: s for s in reference_scenarios()}


def energies(r):
    return [e[3] for e in r["energy"]]


def test_pec_cavity_energy_conserved():
    r = run_oracle(SC["pec_cavity"])
    e = energies(r)
    assert all(np.isfinite(e))
    assert abs(e[-1] - e[0]) / e[0] < 0.30


def test_free_propagation_wave_grows():
    e = energies(run_oracle(SC["free_propagation"]))
    assert max(e) > 2.0 * e[0] and all(np.isfinite(e))


def test_dielectric_slab_propagates():
    r = run_oracle(SC["dielectric_slab"])
    e = energies(r)
    assert max(e) > 1.5 * e[0]
    assert np.isfinite(r["fields"]).all()


def test_resonant_cavity_builds_up():
    e = energies(run_oracle(SC["resonant_cavity"]))
    assert e[-1] > 3.0 * e[0]


def test_small_grid_stable():
    e = energies(run_oracle(SC["small_grid"]))
    assert all(np.isfinite(e)) and min(e) >= 0.0


def test_multi_direction_excites_all_components():
    f = run_oracle(SC["multi_direction"])["fields"]
    assert all((f[c].astype(np.float64) ** 2).sum() > 0 for c in range(3))


def test_hard_soft_sources():
    r = run_oracle(SC["hard_soft_source"])
    assert (r["fields"][:3].astype(np.float64) ** 2).sum() > 0


def test_zero_excitation_stays_zero():
    r = run_oracle(SC["zero_excitation"])
    assert not r["fields"].any()
    assert all(e == 0.0 for e in energies(r))


def test_batch_consistency():
    """Three batches (50+70+80 steps) equal one 200-step batch."""
    sc = SC["batch_consistency"]
    split = run_oracle(sc)
    import copy
    one = copy.copy(sc)
    one.batches = ()
    single = run_oracle(one)
    assert np.array_equal(split["fields"], single["fields"])
    assert split["timestep"] == single["timestep"] == 200


@pytest.mark.parametrize("name", ["high_permittivity", "extreme_permittivity", "magnetic_material"])
def test_material_scenarios_finite_and_energetic(name):
    r = run_oracle(SC[name])
    tot = (r["fields"].astype(np.float64) ** 2).sum()
    assert np.isfinite(tot) and tot > 0


def test_lossy_material_bounded():
    e = energies(run_oracle(SC["lossy_material"]))
    assert all(np.isfinite(e)) and max(e) < 1e10


def test_very_long_simulation_10k_steps():
    """VeryLongSimulationScenario: 12^3, Dirac Ey, 10000 steps, drift < 50%."""
    from scenarios import Scenario
    import openems_b200 as oe
    sc = Scenario("very_long", (12, 12, 12), 1e-3, excitations=[oe.Excitation.dirac(1.0, 1, (6, 6, 6))],
                  num_steps=10_000, sample_interval=100, track_peak=True)
    r = run_oracle(sc)
    e = energies(r)
    assert r["timestep"] == 10_000 and all(np.isfinite(e))
    assert abs(e[-1] - e[0]) / e[0] < 0.50


# ---- oracle self-consistency --------------------------------------------------

@pytest.mark.parametrize("sc", [SC["dielectric_slab"], SC["hard_soft_source"], SC["magnetic_material"],
                                odd_scenarios()[0], odd_scenarios()[4]], ids=lambda s: s.name)
def test_numpy_restatement_agrees_bitwise(sc):
    ref = run_oracle(sc)
    lines = [oracle.uniform_lines(n, sc.delta) for n in sc.dims]
    dt, delta = oracle.grid_timestep(*lines)
    s = oracle.OracleSim(*sc.dims, dt, delta)
    for m in sc.materials:
        s.set_material(*m)
    for p in sc.pec:
        s.set_pec(p)
    exc = []
    for x in sc.excitations:
        samples = np.array([oracle.excitation_eval(int(x.excitation_type), list(x.params), x.amplitude,
                                                   st * dt) for st in range(sc.num_steps)], dtype=np.float32)
        exc.append((x.position, x.direction, x.soft_source, samples))
    got = numpy_ref.run(s.coefficients(), np.zeros((6,) + sc.dims, np.float32), sc.num_steps, exc)
    assert np.array_equal(got, ref["fields"])


def test_parallel_restatement_is_bit_identical():
    sc = SC["dielectric_slab"]
    assert np.array_equal(run_oracle(sc, threads=1)["fields"], run_oracle(sc, threads=4)["fields"])


@pytest.mark.parametrize("name", ["free_propagation", "dielectric_slab", "lossy_material"])
def test_fp32_close_to_fp64(name):
    sc = SC[name]
    a = run_oracle(sc, precision=32)["fields"]
    b = run_oracle(sc, precision=64)["fields"]
    # per vector field: a component that is ~0 by symmetry (Hz of an Ez
    # dipole) is pure rounding noise relative to its own norm
    assert rel_l2(a[:3], b[:3]) < 1e-5
    assert rel_l2(a[3:], b[3:]) < 1e-5
