"""Scenario descriptions run identically on the CUDA engine and on the oracle.

A Scenario mirrors the reference's SimulationSetup
(src/fdtd/engine_testing.rs:38-66): grid, material boxes, PEC boxes,
excitations, steps, energy monitoring, plus CPML and point probes.
"""
from __future__ import annotations

from dataclasses import dataclass, field
from typing import List, Optional, Sequence, Tuple

import numpy as np

import oracle
import openems_b200 as oe


@dataclass
class Scenario:
    name: str
    dims: Tuple[int, int, int]
    delta: float
    materials: List[Tuple] = field(default_factory=list)  # (eps_r, mu_r, sig_e, sig_m, region6)
    pec: List[Tuple] = field(default_factory=list)        # region6
    excitations: List[oe.Excitation] = field(default_factory=list)
    num_steps: int = 100
    sample_interval: int = 0
    track_peak: bool = False
    cpml: Optional[oe.CpmlBoundaries] = None
    mur: Optional[oe.MurAbcConfig] = None
    probes: List[Tuple[int, Tuple[int, int, int]]] = field(default_factory=list)
    batches: Sequence[int] = ()  # split num_steps into these batch sizes (default: one batch)
    dispersive: List[Tuple] = field(default_factory=list)  # (material, cells (n, 3))
    rlc: List[oe.RlcElement] = field(default_factory=list)
    lumped: List[Tuple] = field(default_factory=list)      # (pos, dir, R, C, eps_r, sigma)
    upml: Optional[oe.PmlBoundaries] = None

    def batch_sizes(self):
        return list(self.batches) if self.batches else [self.num_steps]


def make_operator(sc: Scenario) -> oe.Operator:
    grid = oe.Grid.uniform(*sc.dims, sc.delta)
    op = oe.Operator(grid, oe.BoundaryConditions.all_pec())
    for eps_r, mu_r, se, sm, reg in sc.materials:
        op.set_material(eps_r, mu_r, se, sm, reg)
    for reg in sc.pec:
        op.set_pec(reg)
    for pos, d, r, c, eps_r, sig in sc.lumped:
        op.set_lumped(pos, d, r, c, eps_r, sig)
    return op


def run_engine(sc: Scenario, compressed=False, graphs=True, autotune=True, kernels="auto", storage="f32"):
    """Runs the scenario on the CUDA engine; returns dict of results."""
    op = make_operator(sc)
    eng = oe.Engine(op, compressed=compressed, graphs=graphs, autotune=autotune, kernels=kernels,
                    storage=storage)
    if sc.cpml is not None:
        eng.add_cpml(sc.cpml)
    if sc.mur is not None:
        eng.add_mur(sc.mur)
    if sc.upml is not None:
        eng.add_upml(sc.upml)
    for mat, cells in sc.dispersive:
        eng.add_dispersive(mat, cells)
    if sc.rlc:
        eng.add_lumped_rlc(sc.rlc)
    for comp, pos in sc.probes:
        eng.add_point_probe(comp, pos)
    dt = op.timestep()
    energy, traces, start = [], [], 0
    for n in sc.batch_sizes():
        sched = [oe.ScheduledExcitation.from_excitation(x, start, n, dt) for x in sc.excitations]
        res = eng.run_batch(oe.EngineBatch(
            num_steps=n, excitations=sched,
            termination=oe.TerminationConfig(max_timesteps=n, check_interval=100),
            energy_monitoring=oe.EnergyMonitorConfig(sample_interval=sc.sample_interval,
                                                     track_peak=sc.track_peak)))
        energy += [(s.timestep, s.e_energy, s.h_energy, s.total_energy) for s in res.energy_samples]
        if sc.probes:
            traces.append(eng.probe_traces())
        start += n
    e, h = eng.read_fields()
    return {"fields": np.concatenate([e, h]), "energy": energy,
            "traces": np.concatenate(traces) if traces else None,
            "timestep": eng.current_timestep(), "engine": eng, "operator": op}


def run_oracle(sc: Scenario, precision=32, threads=1, zline=False):
    """Runs the scenario on the oracle (BasicEngine semantics); zline picks
    the SIMD engine's loop form (same bits, faster on large grids)."""
    lines = [oracle.uniform_lines(n, sc.delta) for n in sc.dims]
    dt, delta = oracle.grid_timestep(*lines)
    s = oracle.OracleSim(*sc.dims, dt, delta, precision=precision, threads=threads, zline=zline)
    for eps_r, mu_r, se, sm, reg in sc.materials:
        s.set_material(eps_r, mu_r, se, sm, reg)
    for reg in sc.pec:
        s.set_pec(reg)
    if sc.cpml is not None:
        c = sc.cpml
        s.enable_cpml(c.layers, c.grading_order, c.reflection_coeff, c.alpha_max, c.kappa_max)
    if sc.mur is not None:
        s.enable_mur(sc.mur.enabled, sc.mur.order, sc.mur.phase_velocity or 0.0)
    for pos, d, r, c, eps_r, sig in sc.lumped:
        s.set_lumped(pos, d, r, c, eps_r, sig)
    if sc.upml is not None:
        s.enable_upml(sc.upml.layers, sc.upml.grading_order, sc.upml.reflection_coeff, sc.upml.kind)
    for mat, cells in sc.dispersive:
        d = mat.to_c()
        s.add_dispersive(d.kind, list(d.params), cells, d.eps_inf)
    for e in sc.rlc:
        s.add_lumped_rlc(e.position, e.direction, int(e.rlc_type), e.resistance, e.inductance,
                         e.capacitance)
    for comp, pos in sc.probes:
        s.add_point_probe(comp, pos)
    energy, traces, start = [], [], 0
    for n in sc.batch_sizes():
        s.clear_excitations()
        for x in sc.excitations:
            s.add_excitation_analytic(x.position, x.direction, x.soft_source,
                                      int(x.excitation_type), list(x.params), x.amplitude, start, n)
        r = s.run_batch(n, sample_interval=sc.sample_interval, track_peak=sc.track_peak,
                        check_interval=100)
        energy += r["energy_samples"]
        if sc.probes:
            traces.append(s.probe_traces())
        start += n
    return {"fields": s.fields(), "energy": energy,
            "traces": np.concatenate(traces) if traces else None,
            "timestep": s.timestep, "sim": s}


def config1_scenario(num_steps=2000) -> Scenario:
    """64^3, 1 mm, vacuum, PEC faces, soft Gaussian Ez at the centre
    (tau = 1/(pi*20 GHz), t0 = 4 tau), Ez/Hy probes at 4 fixed cells."""
    tau = 1.0 / (np.pi * 20e9)
    exc = oe.Excitation.gaussian_pulse(tau, 4.0 * tau, 2, (32, 32, 32))
    cells = [(16, 16, 16), (48, 16, 32), (32, 48, 16), (40, 40, 48)]
    probes = [(2, c) for c in cells] + [(4, c) for c in cells]
    return Scenario("config1_64_pec", (64, 64, 64), 1e-3, excitations=[exc], num_steps=num_steps,
                    sample_interval=100, track_peak=True, probes=probes)


def reference_scenarios() -> List[Scenario]:
    """The reference's physics scenarios (src/fdtd/engine_testing.rs:782-1700)
    with their grids, materials, sources and step counts."""
    E = oe.Excitation
    return [
        Scenario("pec_cavity", (20, 20, 20), 0.5e-3, excitations=[E.dirac(1.0, 2, (10, 10, 10))],
                 num_steps=200, sample_interval=10, track_peak=True),
        Scenario("free_propagation", (40, 40, 60), 0.5e-3,
                 excitations=[E.gaussian(5e9, 0.5, 2, (20, 20, 10))], num_steps=150,
                 sample_interval=20, track_peak=True),
        Scenario("dielectric_slab", (30, 30, 60), 0.3e-3,
                 materials=[(4.0, 1.0, 0.0, 0.0, (0, 30, 0, 30, 25, 35))],
                 excitations=[E.gaussian(3e9, 0.5, 2, (15, 15, 10))], num_steps=200,
                 sample_interval=20, track_peak=True),
        Scenario("resonant_cavity", (20, 20, 40), 0.5e-3,
                 excitations=[E.sinusoidal(3e9, 2, (10, 10, 20))], num_steps=300,
                 sample_interval=20, track_peak=True),
        Scenario("small_grid", (10, 10, 10), 1.0e-3,
                 excitations=[E.gaussian(2e9, 0.5, 0, (5, 5, 5))], num_steps=100,
                 sample_interval=10, track_peak=True),
        Scenario("multi_direction", (25, 25, 25), 0.5e-3,
                 excitations=[E.gaussian(3e9, 0.5, 0, (12, 12, 12)),
                              E.gaussian(3e9, 0.5, 1, (13, 13, 13)),
                              E.gaussian(3e9, 0.5, 2, (14, 14, 14))],
                 num_steps=150, sample_interval=15, track_peak=True),
        Scenario("hard_soft_source", (30, 30, 30), 0.5e-3,
                 excitations=[E.gaussian(3e9, 0.5, 2, (15, 15, 15)),
                              E.gaussian(3e9, 0.5, 0, (20, 20, 20)).hard_source()],
                 num_steps=100, sample_interval=10, track_peak=True),
        Scenario("long_simulation", (15, 15, 15), 1.0e-3,
                 excitations=[E.dirac(1.0, 1, (7, 7, 7))], num_steps=1000, sample_interval=100,
                 track_peak=True),
        Scenario("zero_excitation", (20, 20, 20), 0.5e-3, num_steps=100, sample_interval=10,
                 track_peak=True),
        Scenario("batch_consistency", (15, 15, 15), 0.8e-3,
                 excitations=[E.gaussian(4e9, 0.5, 2, (7, 7, 7))], num_steps=200,
                 sample_interval=10, track_peak=True, batches=(50, 70, 80)),
        Scenario("high_permittivity", (30, 30, 60), 0.3e-3,
                 materials=[(100.0, 1.0, 0.0, 0.0, (0, 30, 0, 30, 25, 35))],
                 excitations=[E.gaussian(1e9, 0.5, 2, (15, 15, 10))], num_steps=300,
                 sample_interval=20, track_peak=True),
        Scenario("extreme_permittivity", (25, 25, 50), 0.4e-3,
                 materials=[(1000.0, 1.0, 0.0, 0.0, (0, 25, 0, 25, 20, 30))],
                 excitations=[E.gaussian(0.5e9, 0.5, 2, (12, 12, 8))], num_steps=400,
                 sample_interval=20, track_peak=True),
        Scenario("lossy_material", (30, 30, 60), 0.3e-3,
                 materials=[(4.0, 1.0, 0.1, 0.0, (0, 30, 0, 30, 20, 40))],
                 excitations=[E.gaussian(3e9, 0.5, 2, (15, 15, 10))], num_steps=300,
                 sample_interval=20, track_peak=True),
        Scenario("magnetic_material", (25, 25, 50), 0.4e-3,
                 materials=[(1.0, 10.0, 0.0, 0.0, (0, 25, 0, 25, 18, 32))],
                 excitations=[E.gaussian(2e9, 0.5, 2, (12, 12, 8))], num_steps=300,
                 sample_interval=20, track_peak=True),
    ]


def odd_scenarios() -> List[Scenario]:
    """Bounds cases: odd sizes, nz not a multiple of 4, one-cell-thick grids,
    sources on faces, overlapping material / PEC boxes."""
    E = oe.Excitation
    tau = 1.0 / (np.pi * 30e9)
    g = lambda d, p: E.gaussian_pulse(tau, 4 * tau, d, p)  # noqa: E731
    return [
        Scenario("odd_5x7x9", (5, 7, 9), 1e-3, excitations=[g(2, (2, 3, 4)), g(0, (4, 6, 8))],
                 num_steps=60, sample_interval=7, track_peak=True,
                 probes=[(0, (4, 6, 8)), (5, (0, 0, 0)), (3, (2, 3, 4))]),
        Scenario("nz1", (6, 5, 1), 1e-3, excitations=[g(2, (3, 2, 0))], num_steps=40),
        Scenario("nx1", (1, 9, 10), 1e-3, excitations=[g(1, (0, 4, 5))], num_steps=40),
        Scenario("ny1", (7, 1, 6), 1e-3, excitations=[g(0, (3, 0, 3))], num_steps=40),
        Scenario("nz_odd_33", (11, 13, 33), 0.7e-3,
                 materials=[(3.0, 1.5, 0.02, 0.0, (2, 9, 0, 13, 5, 30)),
                            (6.0, 1.0, 0.0, 2e2, (4, 11, 3, 8, 0, 12))],
                 pec=[(5, 7, 5, 7, 10, 20)],
                 excitations=[g(2, (5, 6, 16)), g(1, (10, 12, 32)).hard_source(),
                              g(0, (0, 0, 0))],
                 num_steps=120, sample_interval=10, track_peak=True,
                 probes=[(2, (5, 6, 16)), (1, (10, 12, 32)), (4, (3, 3, 31))]),
        Scenario("wide_z_130", (6, 9, 130), 1e-3, excitations=[g(2, (3, 4, 65))], num_steps=80,
                 probes=[(2, (3, 4, 64)), (3, (1, 1, 129))]),
    ]


def cpml_scenarios() -> List[Scenario]:
    E = oe.Excitation
    tau = 1.0 / (np.pi * 20e9)
    return [
        Scenario("cpml_cube_24", (24, 24, 24), 1e-3,
                 excitations=[E.gaussian_pulse(tau, 4 * tau, 2, (12, 12, 12))], num_steps=200,
                 sample_interval=20, track_peak=True, cpml=oe.CpmlBoundaries.uniform(6),
                 probes=[(2, (12, 12, 12)), (2, (2, 12, 12))]),
        Scenario("cpml_odd_asym", (19, 23, 29), 0.8e-3,
                 materials=[(4.0, 1.0, 0.05, 0.0, (5, 14, 6, 17, 8, 21))],
                 excitations=[E.gaussian_pulse(tau, 4 * tau, 1, (9, 11, 14)),
                              E.gaussian_pulse(tau, 4 * tau, 0, (10, 12, 15))],
                 num_steps=150, sample_interval=25, track_peak=True,
                 cpml=oe.CpmlBoundaries(layers=(4, 5, 0, 6, 7, 3), grading_order=4.0,
                                        reflection_coeff=1e-5, alpha_max=0.05, kappa_max=3.0),
                 probes=[(1, (9, 11, 14)), (5, (1, 1, 1))]),
        # z slabs only, nz not a multiple of 4, a row of 12 chunks: the
        # CPML-free box of a z-split has partial rows that end inside warps
        Scenario("cpml_z_only_45", (14, 26, 45), 1e-3,
                 materials=[(2.0, 1.0, 0.01, 0.0, (3, 11, 4, 20, 2, 43))],
                 excitations=[E.gaussian_pulse(tau, 4 * tau, 2, (7, 13, 22)),
                              E.gaussian_pulse(tau, 4 * tau, 0, (5, 9, 5))],
                 num_steps=160, sample_interval=20, track_peak=True,
                 cpml=oe.CpmlBoundaries(layers=(0, 0, 0, 0, 5, 6)),
                 probes=[(2, (7, 13, 22)), (0, (5, 9, 2)), (4, (7, 13, 41))]),
        # z slabs that meet (5 + 5 layers on nz = 10): the float4 chunk of
        # k = 4..7 lies in both, so its update stretches with both z faces
        Scenario("cpml_z_thin_10", (16, 18, 10), 1e-3,
                 excitations=[E.gaussian_pulse(tau, 4 * tau, 2, (8, 9, 5)),
                              E.gaussian_pulse(tau, 4 * tau, 1, (6, 10, 4))],
                 num_steps=120, sample_interval=20, track_peak=True,
                 cpml=oe.CpmlBoundaries(layers=(3, 3, 0, 2, 5, 5)),
                 probes=[(2, (8, 9, 5)), (1, (6, 10, 7))]),
    ]


def mur_scenarios() -> List[Scenario]:
    E = oe.Excitation
    f0 = 10e9
    x = E.gaussian_modulated(f0, 0.5, 2, (12, 11, 13))
    return [
        Scenario("mur1_all", (25, 22, 27), 1e-3, excitations=[x], num_steps=300, sample_interval=25,
                 track_peak=True, mur=oe.MurAbcConfig.all(1), probes=[(2, (1, 11, 13)), (1, (24, 5, 5))]),
        Scenario("mur2_all", (25, 22, 27), 1e-3, excitations=[x], num_steps=300, sample_interval=25,
                 track_peak=True, mur=oe.MurAbcConfig.all(2), probes=[(2, (1, 11, 13)), (1, (24, 5, 5))]),
        Scenario("mur1_partial_phase", (18, 9, 14), 0.8e-3,
                 materials=[(3.0, 1.0, 0.01, 0.0, (0, 18, 0, 9, 0, 7))],
                 excitations=[E.gaussian_modulated(8e9, 0.5, 1, (9, 4, 7))], num_steps=200,
                 mur=oe.MurAbcConfig(enabled=(1, 0, 1, 1, 0, 1), phase_velocity=2.0e8, order=1)),
        Scenario("mur2_partial", (18, 9, 14), 0.8e-3,
                 excitations=[E.gaussian_modulated(8e9, 0.5, 0, (9, 4, 7))], num_steps=200,
                 mur=oe.MurAbcConfig(enabled=(0, 1, 1, 0, 1, 1), order=2)),
    ]


def probe_scenario() -> Scenario:
    """Lossy box with CPML, two sources and every probe kind."""
    E = oe.Excitation
    return Scenario("probes", (21, 18, 24), 1e-3,
                    materials=[(2.5, 1.0, 0.02, 0.0, (4, 16, 3, 15, 5, 19))],
                    excitations=[E.gaussian_modulated(9e9, 0.5, 2, (10, 9, 12)),
                                 E.gaussian_modulated(6e9, 0.4, 0, (12, 6, 15))],
                    num_steps=260, cpml=oe.CpmlBoundaries(layers=(4, 4, 4, 4, 4, 4)),
                    batches=(100, 160))


def _box_cells(i0, i1, j0, j1, k0, k1):
    g = np.mgrid[i0:i1, j0:j1, k0:k1].reshape(3, -1).T
    return np.ascontiguousarray(g, dtype=np.int64)


def dispersive_scenarios() -> List[Scenario]:
    """Drude, Debye and second-order Lorentz blocks with sources and CPML;
    the reference's first-order Lorentz for a few steps (it diverges);
    lumped RLC elements of both types; a lumped resistor port."""
    E = oe.Excitation
    x = E.gaussian_modulated(12e9, 0.5, 2, (8, 9, 10))
    drude = oe.DrudeMaterial(2 * np.pi * 20e9, 1e10)
    debye = oe.DebyeMaterial(1e-11, 3.0, eps_inf=2.0)
    lorentz2 = oe.LorentzMaterial(2 * np.pi * 15e9, 2e9, 2.0, eps_inf=1.5, second_order=True)
    lorentz = oe.LorentzMaterial(2 * np.pi * 15e9, 2e9, 2.0)
    rlc = [oe.RlcElement((5, 5, 5), 2, oe.RlcType.Parallel, 50.0, 1e-9, 1e-12),
           oe.RlcElement((11, 4, 12), 0, oe.RlcType.Parallel, 0.0, 2e-9, 0.0),
           oe.RlcElement((6, 12, 7), 1, oe.RlcType.Series, 10.0, 1e-9, 0.5e-12),
           oe.RlcElement((5, 5, 5), 2, oe.RlcType.Parallel, 100.0, 0.0, 0.0)]
    return [
        Scenario("drude_debye_cpml", (17, 19, 21), 1e-3, excitations=[x], num_steps=220,
                 sample_interval=20, track_peak=True, cpml=oe.CpmlBoundaries.uniform(4),
                 dispersive=[(drude, _box_cells(10, 14, 3, 9, 12, 18)),
                             (debye, _box_cells(2, 7, 11, 16, 2, 19))],
                 probes=[(2, (11, 5, 14)), (0, (4, 13, 10))]),
        Scenario("lorentz2_overlap", (14, 13, 22), 1e-3, excitations=[x], num_steps=200,
                 dispersive=[(lorentz2, _box_cells(3, 12, 2, 11, 12, 20)),
                             (drude, _box_cells(6, 9, 5, 8, 14, 17)),
                             (oe.DrudeMaterial(2 * np.pi * 30e9, 0.0, eps_inf=1.5, second_order=True),
                              _box_cells(2, 5, 2, 5, 3, 9))],
                 probes=[(2, (7, 6, 15)), (1, (3, 3, 5))]),
        Scenario("lorentz_reference_short", (10, 11, 12), 1e-3,
                 excitations=[E.gaussian_modulated(12e9, 0.5, 1, (5, 5, 6))], num_steps=30,
                 dispersive=[(lorentz, _box_cells(2, 8, 2, 9, 3, 10))]),
        Scenario("lumped_rlc", (16, 15, 18), 1e-3,
                 excitations=[E.gaussian_modulated(10e9, 0.5, 2, (8, 7, 9))], num_steps=250,
                 sample_interval=25, track_peak=True, rlc=rlc, mur=oe.MurAbcConfig.all(1),
                 probes=[(2, (5, 5, 5)), (0, (11, 4, 12)), (1, (6, 12, 7))]),
        Scenario("lumped_port_r", (16, 16, 20), 1e-3,
                 excitations=[E.gaussian_modulated(10e9, 0.5, 2, (8, 8, 10)).with_amplitude(7.0)],
                 num_steps=200, lumped=[((8, 8, 10), 2, 50.0, 0.0, 1.0, 0.0),
                                        ((4, 9, 6), 0, 0.0, 2e-13, 2.0, 0.01)],
                 cpml=oe.CpmlBoundaries.uniform(4), probes=[(2, (8, 8, 10)), (0, (4, 9, 6))]),
    ]


def upml_scenarios() -> List[Scenario]:
    """The reference's UPML: short runs (it grows without bound), all faces
    and partial faces, with a dielectric and Mur on other faces; the
    corrected UPML (kind 1): the reference's PML scenario for its full 300
    steps, and partial faces with a lossy dielectric and a PEC block that
    reach into the PML."""
    E = oe.Excitation
    return [
        Scenario("upml_fixed_reference_scenario", (60, 60, 60), 0.5e-3,
                 excitations=[E.gaussian(3e9, 0.5, 2, (30, 30, 30))], num_steps=300, sample_interval=30,
                 track_peak=True, upml=oe.PmlBoundaries.uniform(8, kind=1),
                 probes=[(2, (30, 30, 30)), (2, (3, 30, 30)), (4, (55, 5, 57))]),
        Scenario("upml_fixed_partial", (19, 15, 26), 0.5e-3,
                 materials=[(3.0, 1.0, 0.02, 0.0, (2, 17, 3, 12, 4, 24))],
                 pec=[(8, 10, 0, 4, 10, 14)],
                 excitations=[E.gaussian(4e9, 0.5, 1, (9, 7, 13)), E.gaussian(5e9, 0.5, 0, (12, 9, 15))],
                 num_steps=160, sample_interval=20, track_peak=True,
                 upml=oe.PmlBoundaries(layers=(4, 0, 3, 5, 0, 6), grading_order=4.0, reflection_coeff=1e-5,
                                       kind=1),
                 mur=oe.MurAbcConfig(enabled=(0, 1, 0, 0, 1, 0)),
                 probes=[(1, (9, 7, 13)), (3, (1, 1, 1)), (0, (17, 13, 24))]),
        Scenario("upml_all_20", (20, 21, 22), 0.5e-3,
                 excitations=[E.gaussian(3e9, 0.5, 2, (10, 10, 11))], num_steps=40, sample_interval=5,
                 track_peak=True, upml=oe.PmlBoundaries.uniform(4),
                 probes=[(2, (10, 10, 11)), (2, (2, 3, 4)), (4, (18, 18, 19))]),
        Scenario("upml_partial", (17, 13, 23), 0.5e-3,
                 materials=[(3.0, 1.0, 0.0, 0.0, (3, 14, 2, 11, 5, 18))],
                 excitations=[E.gaussian(4e9, 0.5, 1, (8, 6, 11))], num_steps=35,
                 upml=oe.PmlBoundaries(layers=(3, 0, 5, 4, 0, 6), grading_order=4.0, reflection_coeff=1e-5),
                 mur=oe.MurAbcConfig(enabled=(0, 1, 0, 0, 1, 0)),
                 probes=[(1, (8, 6, 11)), (3, (1, 1, 1))]),
    ]
