"""The reference's uniaxial PML on the oracle (CPU): its unit tests
(src/extensions/pml.rs:860-990) and the instability its cross-engine tests
record (src/fdtd/engine_testing.rs:2322-2330)."""
import numpy as np
import pytest

import oracle
from scenarios import Scenario, run_oracle, upml_scenarios
import openems_b200 as oe


def sim(n=50, d=1e-3, dt=1e-12):
    return oracle.OracleSim(n, n, n, dt, (d, d, d))


def test_upml_regions():
    """test_upml_creation / test_upml_disabled_boundary (pml.rs:889-925)."""
    assert sim().enable_upml((8,) * 6) == 6
    assert sim().enable_upml((0, 0, 8, 8, 8, 8)) == 4
    assert sim().enable_upml((0,) * 6) == 0
    # a face with layers >= n is not built, but its layer count still trims
    # the other faces' extent (pml.rs:244-250), which leaves nothing here
    assert sim(n=8).enable_upml((8, 8, 2, 2, 2, 2)) == 0
    assert sim(n=8).enable_upml((0, 0, 2, 2, 8, 2)) == 3


def test_pml_config_sigma_max():
    """test_pml_config (pml.rs:864-871): sigma_max = -(m+1) ln R / (2 eta d) > 0."""
    d = 8 * 1e-3
    smax = -(3.0 + 1.0) * np.log(1e-6) / (2.0 * 376.730313668 * d)
    assert smax > 0


def test_kappa_grading():
    """test_kappa_grading (pml.rs:927-951)."""
    s = sim()
    kv, ki = s.upml_kappa(0, 0, (25, 25, 25), True, 8, 0.008, 1000.0, 3.0)
    assert kv == 0.0 and ki == 0.0
    kv, ki = s.upml_kappa(0, 0, (4, 25, 25), True, 8, 0.008, 1000.0, 3.0)
    assert kv == pytest.approx(125.0, abs=1e-6)
    # current grading half a cell shallower along the PML direction, deeper across
    assert ki == pytest.approx(1000.0 * (3.5 / 8) ** 3, rel=1e-12)
    _, ki1 = s.upml_kappa(1, 0, (4, 25, 25), True, 8, 0.008, 1000.0, 3.0)
    assert ki1 == pytest.approx(1000.0 * (4.5 / 8) ** 3, rel=1e-12)
    kv, _ = s.upml_kappa(0, 0, (45, 25, 25), False, 8, 0.008, 1000.0, 3.0)  # max side: 45 - 41
    assert kv == pytest.approx(1000.0 * (4 / 8) ** 3, rel=1e-12)


def test_center_unaffected_by_pml():
    """test_upml_field_update (pml.rs:953-988): away from the regions the
    fields evolve exactly as without the PML until the PML's influence
    arrives (one cell per half step)."""
    E = oe.Excitation
    base = Scenario("c", (20, 20, 20), 1e-3, excitations=[E.dirac(1.0, 2, (10, 10, 10))], num_steps=3)
    with_pml = Scenario("p", (20, 20, 20), 1e-3, excitations=[E.dirac(1.0, 2, (10, 10, 10))], num_steps=3,
                        upml=oe.PmlBoundaries.uniform(4))
    a, b = run_oracle(base)["fields"], run_oracle(with_pml)["fields"]
    core = (slice(None), slice(7, 14), slice(7, 14), slice(7, 14))
    assert np.array_equal(a[core], b[core])
    assert a[2, 10, 10, 10] == b[2, 10, 10, 10] != 0


def test_reference_upml_grows_without_bound():
    """PmlAbsorbingScenario (engine_testing.rs:1712-1760): 60^3, 0.5 mm,
    8-layer PML; the reference's coefficients amplify instead of absorb,
    about 1e20 per 30 steps as its note says (the same run without the PML
    reaches 7e-5 at step 120)."""
    E = oe.Excitation
    sc = Scenario("pml60", (60, 60, 60), 0.5e-3, excitations=[E.gaussian(3e9, 0.5, 2, (30, 30, 30))],
                  num_steps=150, sample_interval=30, track_peak=True, upml=oe.PmlBoundaries.uniform(8))
    e = [x[3] for x in run_oracle(sc, threads=8)["energy"]]
    assert len(e) == 5  # steps 0, 30, ..., 120
    assert e[3] > 1e10 and e[4] > 1e30


def test_corrected_upml_absorbs_in_the_reference_scenario():
    """The reference's PmlAbsorbingScenario (src/fdtd/engine_testing.rs:
    1703-1768: 60^3, 0.5 mm, Gaussian Ez at the centre, 8-layer PML, energy
    every 30 steps) with the corrected UPML, run to 1500 steps so that the
    pulse (t0 = 357 steps) has passed: the reference's own check (final
    energy below the peak) cannot hold at its 300 steps, where the pulse is
    still rising.  The Gaussian has a DC part, which leaves a static charge
    at the source whose field no absorber removes, so the run is compared
    with the same run terminated by the CPML: equal energies at every sample
    to 1e-3 (the radiated part leaves through both), bounded throughout."""
    sc = upml_scenarios()[0]
    assert sc.upml.kind == 1
    sc.num_steps, sc.sample_interval, sc.probes = 1500, 100, []
    r = run_oracle(sc, threads=4, zline=True)
    sc.upml, sc.cpml = None, oe.CpmlBoundaries.uniform(8)
    c = run_oracle(sc, threads=4, zline=True)
    tu = np.array([e[3] for e in r["energy"]])
    tc = np.array([e[3] for e in c["energy"]])
    assert np.all(np.isfinite(tu)) and tu[-1] <= tu.max()
    assert np.allclose(tu, tc, rtol=1e-3, atol=0.0)


def test_reference_upml_in_its_scenario_grows():
    """The same scenario with the reference's coefficients (kind 0) does not
    settle: the energy ends above its early peak (the instability)."""
    sc = upml_scenarios()[0]
    sc.upml = oe.PmlBoundaries.uniform(8, kind=0)
    sc.num_steps = 150
    r = run_oracle(sc, threads=4, zline=True)
    tot = np.array([e[3] for e in r["energy"]])
    assert not np.isfinite(tot[-1]) or tot[-1] > tot[:3].max()
