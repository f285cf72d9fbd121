"""The reference's known-answer unit tests, applied to the oracle (CPU).

These pin the oracle to every known answer the Rust reference's own tests
hold for this path; the reference ships no golden field arrays.
"""
import math

import numpy as np
import pytest

import oracle

C0 = 299792458.0


def op5(delta=0.001, dt=None, precision=32):
    """create_test_grid (src/fdtd/operator.rs:278-285): 5 cells of 1 mm per axis."""
    lines = oracle.uniform_lines(5, delta)
    dt0, d3 = oracle.grid_timestep(lines, lines, lines)
    return oracle.OracleSim(5, 5, 5, dt if dt else dt0, d3, precision=precision), dt0


# ---- src/fdtd/operator.rs:287-501 -----------------------------------------

def test_timestep_below_cfl():
    lines = oracle.uniform_lines(2, 0.001)
    dt, _ = oracle.grid_timestep(lines, lines, lines)
    assert 0 < dt < 1.0 / (C0 * math.sqrt(3.0) / 0.001)


def test_vacuum_coefficients():
    s, _ = op5()
    c = s.coefficients()
    ca, cb, da, db = c[0:3], c[3:6], c[6:9], c[9:12]
    assert np.all(np.abs(ca[:, 2, 2, 2] - 1.0) < 1e-6) and np.all(cb[:, 2, 2, 2] > 0)
    assert np.all(np.abs(da[:, 2, 2, 2] - 1.0) < 1e-6) and np.all(db[:, 2, 2, 2] < 0)


def test_set_material_eps4_ratio_quarter():
    s, _ = op5()
    s.set_material(4.0, 1.0, 0.0, 0.0, (1, 3, 1, 3, 1, 3))
    c = s.coefficients()
    assert abs(c[0, 2, 2, 2] - 1.0) < 1e-6
    assert abs(c[3, 2, 2, 2] / c[3, 0, 0, 0] - 0.25) < 1e-5
    assert abs(c[6, 2, 2, 2] - 1.0) < 1e-6


def test_set_material_lossy():
    s, _ = op5()
    s.set_material(2.0, 1.0, 0.01, 0.0, (1, 3, 1, 3, 1, 3))
    ca = s.coefficients()[0, 2, 2, 2]
    assert 0.0 < ca < 1.0


def test_set_material_magnetic():
    s, _ = op5()
    s.set_material(1.0, 4.0, 0.0, 1e6, (1, 3, 1, 3, 1, 3))
    c = s.coefficients()
    assert 0.0 < c[6, 2, 2, 2] < 1.0
    assert abs(c[9, 2, 2, 2]) < abs(c[9, 0, 0, 0])


def test_set_pec():
    s, _ = op5()
    s.set_pec((1, 3, 1, 3, 1, 3))
    c = s.coefficients()
    assert np.all(np.abs(c[0:6, 2, 2, 2]) < 1e-10)
    assert abs(c[0, 0, 0, 0] - 1.0) < 1e-6 and c[3, 0, 0, 0] > 0


def test_anisotropic_timestep():
    dt, _ = oracle.grid_timestep([0, 0.001, 0.002, 0.003], [0, 0.002, 0.004, 0.006], [0, 0.0005, 0.001])
    dt_max = 1.0 / (C0 * math.sqrt(1 / 0.001 ** 2 + 1 / 0.002 ** 2 + 1 / 0.0005 ** 2))
    assert 0.9 * dt_max < dt < dt_max


# ---- src/fdtd/excitation.rs:258-400 -----------------------------------------

def gaussian_params(fc, bw):
    f_max = fc * (1.0 + 0.5 * bw)
    tau = 1.0 / (math.pi * f_max)
    return [4.0 * tau, tau]


def test_gaussian():
    p = gaussian_params(1e9, 0.5)
    assert abs(oracle.excitation_eval(oracle.EXC_GAUSSIAN, p, 1.0, p[0]) - 1.0) < 1e-10
    assert oracle.excitation_eval(oracle.EXC_GAUSSIAN, p, 1.0, 0.0) < 0.01
    assert abs(oracle.excitation_eval(oracle.EXC_GAUSSIAN, p, 2.5, p[0]) - 2.5) < 1e-10


def test_sinusoidal():
    f = 1e9
    v1 = oracle.excitation_eval(oracle.EXC_SINUSOIDAL, [f], 1.0, 0.0)
    v2 = oracle.excitation_eval(oracle.EXC_SINUSOIDAL, [f], 1.0, 1.0 / f)
    assert abs(v1 - v2) < 1e-10
    assert abs(oracle.excitation_eval(oracle.EXC_SINUSOIDAL, [f], 1.0, 0.25 / f) - 1.0) < 1e-10


def test_gaussian_modulated():
    fc, bw = 1e9, 0.5
    tau = 1.0 / (math.pi * fc * bw)
    p = [fc, 4 * tau, tau]
    assert abs(oracle.excitation_eval(oracle.EXC_GAUSSIAN_MODULATED, p, 1.0, 0.0)) < 0.01
    v1 = oracle.excitation_eval(oracle.EXC_GAUSSIAN_MODULATED, p, 1.0, p[1])
    v2 = oracle.excitation_eval(oracle.EXC_GAUSSIAN_MODULATED, p, 1.0, p[1] + 0.5 / fc)
    assert v1 * v2 <= 0.0 or abs(v1) < 0.1 or abs(v2) < 0.1


def test_dirac_and_step():
    assert abs(oracle.excitation_eval(oracle.EXC_DIRAC, [], 1.0, 0.0) - 1.0) < 1e-10
    assert abs(oracle.excitation_eval(oracle.EXC_DIRAC, [], 1.0, 1e-9)) < 1e-10
    assert abs(oracle.excitation_eval(oracle.EXC_DIRAC, [], 1.0, -1e-9)) < 1e-10
    assert abs(oracle.excitation_eval(oracle.EXC_STEP, [], 3.0, 0.0) - 3.0) < 1e-10
    assert abs(oracle.excitation_eval(oracle.EXC_STEP, [], 3.0, 1e-9) - 3.0) < 1e-10
    assert abs(oracle.excitation_eval(oracle.EXC_STEP, [], 3.0, -1e-9)) < 1e-10


# ---- src/fdtd/batch.rs:235-294 ----------------------------------------------

def test_batch_config_defaults():
    """test_termination_config_default / test_energy_monitor_config_default:
    no step cap, no decay threshold, checks every 100 steps; no sampling,
    no peak tracking, no threshold (the Python mirror's defaults, which the
    C structs take over)."""
    import openems_b200 as oe
    t = oe.TerminationConfig()
    assert t.max_timesteps is None and t.energy_decay_db is None and t.check_interval == 100
    m = oe.EnergyMonitorConfig()
    assert m.sample_interval == 0 and not m.track_peak and m.decay_threshold is None


def test_scheduled_samples_match_evaluate():
    """ScheduledExcitation::from_excitation: samples[i] == (f32) evaluate(i*dt)."""
    p = gaussian_params(1e9, 0.5)
    s, _ = op5(dt=1e-12)
    s.add_excitation_analytic((2, 2, 2), 2, True, oracle.EXC_GAUSSIAN, p, 1.0, 0, 100)
    s.add_point_probe(2, (2, 2, 2))
    s.run_batch(1)
    # soft source into a zero field: after step 0 (E update of zero fields is zero)
    # the cell holds exactly samples[0]
    got = s.probe_traces()[0, 0]
    assert abs(got - np.float32(oracle.excitation_eval(oracle.EXC_GAUSSIAN, p, 1.0, 0.0))) < 1e-6


def test_energy_sample_arithmetic():
    s, _ = op5()
    f = np.zeros((6, 5, 5, 5), np.float32)
    f[0, 2, 2, 2] = 1.0
    f[4, 2, 2, 2] = 2.0
    s.set_fields(f)
    e, h = s.energy()
    assert e == 1.0 and h == 4.0


# ---- src/extensions/cpml.rs:744-804 ------------------------------------------

def test_cpml_coefficient_ranges():
    """sigma_max > 0; 0 <= b <= 1; a >= 0 (the reference's a is -c*kappa)."""
    lines = oracle.uniform_lines(50, 0.001)
    _, d3 = oracle.grid_timestep(lines, lines, lines)
    s = oracle.OracleSim(50, 50, 50, 1e-12, d3)
    s.enable_cpml((8,) * 6)
    for f in range(6):
        prof = s.cpml_profile(f)
        assert len(prof["b_e"]) == 8
        for k in ("b_e", "b_h"):
            assert np.all((prof[k] >= 0) & (prof[k] <= 1))
        for k in ("c_e", "c_h"):
            assert np.all(-prof[k] >= 0)
        # graded: deeper layers absorb more (smaller b)
        b = prof["b_e"] if f % 2 else prof["b_e"][::-1]
        assert np.all(np.diff(b) <= 0)


def test_cpml_regions_count():
    """Cpml::new with uniform(8) on 50^3 has 6 active regions (cpml.rs:744-759);
    a face with layers >= n is inactive (cpml.rs:262, 283)."""
    lines = oracle.uniform_lines(50, 0.001)
    _, d3 = oracle.grid_timestep(lines, lines, lines)
    s = oracle.OracleSim(50, 50, 50, 1e-12, d3)
    s.enable_cpml((8,) * 6)
    assert sum(1 for f in range(6) if len(s.cpml_profile(f)["b_e"])) == 6
    s2 = oracle.OracleSim(6, 50, 50, 1e-12, d3)
    s2.enable_cpml((6, 6, 8, 8, 8, 8))
    assert [len(s2.cpml_profile(f)["b_e"]) for f in range(6)] == [0, 0, 8, 8, 8, 8]


# ---- src/processing/probes.rs:388-503 (probe sums, via the C++ term builders) --

def _probe_value(terms, fields_fn, dims=(10, 10, 10)):
    lines = oracle.uniform_lines(dims[0], 1e-3)
    dt, d3 = oracle.grid_timestep(lines, lines, lines)
    s = oracle.OracleSim(*dims, dt, d3)
    f = np.zeros((6,) + dims, np.float32)
    fields_fn(f)
    s.set_fields(f)
    s.add_probe(terms.terms, terms.mode)
    return s.eval_probes()[0]


def test_voltage_probe_sums():
    import openems_b200 as oe
    assert abs(_probe_value(oe.voltage_probe((0, 5, 5), (9, 5, 5), 0),
                            lambda f: f[0].fill(2.0)) - 20.0) < 1e-6
    assert abs(_probe_value(oe.voltage_probe((5, 0, 5), (5, 9, 5), 1),
                            lambda f: f[1].fill(3.0)) - 30.0) < 1e-6
    for val, want in ((1.0, 5.0), (2.0, 10.0), (0.5, 2.5)):
        assert abs(_probe_value(oe.voltage_probe((5, 5, 0), (5, 5, 4), 2),
                                lambda f, v=val: f[2].fill(v)) - want) < 1e-6

    def single(f):
        f[2, 5, 5, 5] = 2.5
    assert abs(_probe_value(oe.voltage_probe((5, 5, 5), (5, 5, 5), 2), single) - 2.5) < 1e-5


def test_current_probe_sums():
    import openems_b200 as oe

    def yfill(f):
        f[5].fill(1.0)
        f[3].fill(0.5)
    assert abs(_probe_value(oe.current_probe((0, 5, 0), (9, 5, 9), 1), yfill) - 50.0) < 1e-5

    def zfill(f):
        f[3].fill(2.0)
        f[4].fill(1.0)
    assert abs(_probe_value(oe.current_probe((0, 0, 5), (9, 9, 5), 2), zfill) - 100.0) < 1e-5
    t = oe.current_probe((5, 0, 0), (5, 4, 4), 10)
    assert t.terms == [] and abs(_probe_value(t, lambda f: f[4].fill(1.0))) < 1e-10


def test_engine_interface_integrals():
    """test_voltage_integral / test_current_integral_{y,z}_normal
    (src/fdtd/engine_interface.rs tests module): E_x = 100 V/m over 5 cells
    of 1 mm integrates to -0.5 V (V = -sum E dl); uniform H through a y- or
    z-normal surface gives a non-zero current."""
    import openems_b200 as oe
    op = oe.Operator(oe.Grid.uniform(10, 10, 10, 1e-3), oe.BoundaryConditions.all_pec())
    v = _probe_value(oe.voltage_integral(op, (0, 5, 5), (5, 5, 5)), lambda f: f[0].fill(100.0))
    assert v < 0.0 and abs(v - (-0.5)) < 1e-12

    def yfill(f):
        f[3].fill(1.0)
        f[5].fill(0.5)

    def zfill(f):
        f[3].fill(1.0)
        f[4].fill(0.5)
    assert abs(_probe_value(oe.current_integral(op, (0, 5, 0), (5, 5, 5), 1), yfill)) > 0.0
    assert abs(_probe_value(oe.current_integral(op, (0, 0, 5), (5, 5, 5), 2), zfill)) > 0.0


def test_constants():
    """src/constants.rs tests: Z0 = MU0 C0, C0 = 1 / sqrt(EPS0 MU0), and a
    1 GHz wavelength of 0.299792458 m."""
    from openems_b200.constants import C0, EPS0, MU0, Z0
    assert abs(Z0 - MU0 * C0) < 1e-6
    assert abs(C0 - 1.0 / np.sqrt(EPS0 * MU0)) < 1.0
    assert abs(C0 / 1e9 - 0.299792458) < 1e-6


def test_voltage_integral_weights_and_sign():
    """V = -sum E . dl (src/fdtd/engine_interface.rs:206-247)."""
    import openems_b200 as oe
    op = oe.Operator(oe.Grid.uniform(10, 10, 10, 1e-3), oe.BoundaryConditions.all_pec())
    t = oe.voltage_integral(op, (2, 3, 4), (2, 3, 9))
    assert len(t.terms) == 5 and all(c == 2 and abs(w + 1e-3) < 1e-15 for c, _, w in t.terms)
    assert abs(_probe_value(t, lambda f: f[2].fill(4.0)) - (-5 * 4.0 * 1e-3)) < 1e-15


def test_storage_rounding_restatement():
    """2-byte storage in the numpy restatement: bfloat16 rounds to nearest
    even on the 16 dropped bits, half as numpy's float16; the f32 "storage"
    run is the plain update."""
    from oracle.numpy_ref import round_to_storage, run, run_stored
    v = np.array([1.0, 1.0 + 2 ** -8, 1.0 + 3 * 2 ** -8, -2.5, 3.0e38], dtype=np.float32)
    assert list(round_to_storage(v, "bf16")[:4]) == [1.0, 1.0, 1.0 + 2 ** -6, -2.5]
    assert round_to_storage(np.float32(1 + 2 ** -11), "f16") == 1.0
    rng = np.random.default_rng(0)
    co = [np.full((6, 5, 7), x, np.float32) for x in (1.0, 1.0, 1.0, 0.4, 0.4, 0.4, 1.0, 1.0, 1.0,
                                                         -0.3, -0.3, -0.3)]
    f = rng.standard_normal((6, 6, 5, 7)).astype(np.float32)
    assert np.array_equal(run_stored(co, f, 5, store="f32", h_scale=1.0), run(co, f, 5))
    # half storage of the same update stays within a few half ulps per step
    a = run_stored(co, f, 5, store="f16")
    assert np.abs(a - run(co, f, 5)).max() < 5 * 2 ** -11 * np.abs(f).max() * 8


def _tfsf_samples(n_steps, length, pos, dt, dx, freq, amp, v=299792458.0):
    """The reference's TF/SF 1D auxiliary grid (src/extensions/tfsf.rs:204-238)
    restated in numpy float32: (e_inc, h_inc) at `pos` after each step."""
    EPS0, MU0 = 8.854187817e-12, 1.256637062e-6
    e, h = np.zeros(length, np.float32), np.zeros(length, np.float32)
    db, cb = np.float32(-(dt / (MU0 * dx))), np.float32(dt / (EPS0 * dx))
    coeff = np.float32((v * dt - dx) / (v * dt + dx))
    eta = np.sqrt(MU0 / EPS0)
    out = []
    for t in range(n_steps):
        for i in range(length - 1):
            h[i] = h[i] + db * (e[i + 1] - e[i])
        h[0] = np.float32((amp / eta) * np.sin(2.0 * np.pi * freq * (t * dt)))
        for i in range(1, length):
            e[i] = e[i] + cb * (h[i] - h[i - 1])
        e[length - 1] = coeff * e[length - 2]
        out.append((e[pos], h[pos]))
    return out


@pytest.mark.parametrize("precision", [32, 64])
def test_tfsf_plane_injection_known_answer(precision):
    """With Ca = Da = 1 and Cb = Db = 0 the Yee update leaves the fields as
    they are, so after n steps plane `pos` of the H component holds
    -sum db e_inc and that of the E component sum cb h_inc (f32 steps of the
    numpy restatement of the 1D grid); nothing else changes."""
    n = (9, 7, 12)
    dt, dx = 1e-12, 1e-3
    s = oracle.OracleSim(*n, dt, (dx,) * 3, precision=precision)
    co = np.zeros((12,) + n)
    co[0:3] = 1.0
    co[6:9] = 1.0
    s.set_coefficients(co.astype(np.float32 if precision == 32 else np.float64))
    s.enable_tfsf(4, 0, 20e9, 2.0, boundary_layer=5)  # +z, E along x, H along y
    s.run_batch(40)
    f = s.fields()
    samples = _tfsf_samples(40, n[2] + 1, 5, dt, dx, 20e9, 2.0)
    T = np.float32 if precision == 32 else np.float64
    db, cb = T(np.float32(-(dt / (1.256637062e-6 * dx)))), T(np.float32(dt / (8.854187817e-12 * dx)))
    hy, ex = T(0), T(0)
    for e_inc, h_inc in samples:
        hy = hy - db * T(e_inc)
        ex = ex + cb * T(h_inc)
    assert np.all(f[4][:, :, 5] == hy) and np.all(f[0][:, :, 5] == ex) and hy != 0 and ex != 0
    rest = f.copy()
    rest[4][:, :, 5] = 0
    rest[0][:, :, 5] = 0
    assert np.all(rest == 0)
    with pytest.raises(ValueError):
        oracle.OracleSim(*n, dt, (dx,) * 3).enable_tfsf(0, 0, 1e9, 1.0, boundary_layer=9)


@pytest.mark.parametrize("polarization,e_axis", [(0, 1), (1, 2)])
def test_corrected_tfsf_separates_total_and_scattered_fields(polarization, e_axis):
    """The corrected TF/SF source (kind 1) on a grid with CPML on every face,
    so that a plane wave uniform across y and z is an exact solution: before
    any wave comes back from the domain's ends, the scattered region (x <
    boundary) stays below 1e-3 of the amplitude and the total region carries
    the wave at the amplitude (numerical dispersion and switch-on within 20%)."""
    nx, ny, nz = 120, 24, 24
    lines = [oracle.uniform_lines(n, 1e-3) for n in (nx, ny, nz)]
    dt, d3 = oracle.grid_timestep(*lines)
    s = oracle.OracleSim(nx, ny, nz, dt, d3, threads=8)
    s.enable_cpml((6,) * 6)
    s.enable_tfsf(0, polarization, 15e9, 1.0, boundary_layer=20, kind=1)
    worst_scattered, total = 0.0, []
    for _ in range(5):
        s.run_batch(60)
        e = s.fields()[e_axis][:, ny // 2, nz // 2]
        worst_scattered = max(worst_scattered, float(np.abs(e[8:19]).max()))
        total.append(float(np.abs(e[25:100]).max()))
    assert worst_scattered < 1e-3
    assert 0.9 < max(total[1:]) < 1.2
    with pytest.raises(ValueError):  # the corrected source needs a positive direction
        oracle.OracleSim(nx, ny, nz, dt, d3).enable_tfsf(1, 0, 15e9, 1.0, boundary_layer=20, kind=1)
