"""Dispersive ADE materials and lumped RLC elements on the oracle (CPU).

A 1 x 1 x 1 grid isolates the per-cell extension: E is updated only at
i, j, k >= 1 and the H update sees zero forward differences at the max faces,
so the single cell's E changes only through post_update_e.  That makes the
oracle's traces comparable bit for bit with the independent numpy
restatement (oracle/numpy_ref.py), and lets the continuous-time physics of
each model be checked on the oracle:

- Drude (no damping): E oscillates at omega_p / sqrt(eps_inf);
- second-order Lorentz (no damping): at omega_0 sqrt(1 + delta_eps / eps_inf);
- Debye: E relaxes to E0 eps_inf / (eps_inf + delta_eps);
- the reference's first-order Lorentz update grows without bound.

The reference's own unit tests for these types
(src/extensions/dispersive.rs:657-755, src/extensions/lumped_rlc.rs:319-416)
assert only that state builds up and resets; they are replayed here too.
"""
import numpy as np
import pytest

import oracle
from oracle import numpy_ref as nr

DT = 1.9e-12


def one_cell(dt=DT, e0=(1.0, 1.0, 1.0)):
    s = oracle.OracleSim(1, 1, 1, dt, (1e-3, 1e-3, 1e-3))
    f = np.zeros((6, 1, 1, 1), dtype=np.float32)
    f[:3, 0, 0, 0] = e0
    s.set_fields(f)
    for c in range(3):
        s.add_point_probe(c, (0, 0, 0))
    return s


def restated_trace(kind, params, eps_inf, steps, dt=DT, e0=(1.0, 1.0, 1.0)):
    co = nr.dispersive_coeffs(kind, params, dt, eps_inf)
    out = np.zeros((steps, 3), dtype=np.float32)
    for c in range(3):
        e, st, pv = np.float32(e0[c]), np.float32(0), np.float32(0)
        for n in range(steps):
            e, st, pv = nr.dispersive_step(kind, co, e, st, pv, dt)
            out[n, c] = e
    return out


CASES = [
    (0, (2 * np.pi * 20e9, 1e10), 1.0),
    (0, (2 * np.pi * 35e9, 0.0), 2.5),
    (1, (2 * np.pi * 15e9, 2e9, 2.0), 1.0),
    (2, (1e-11, 3.0), 2.0),
    (2, (4e-12, 10.0), 1.0),  # explicit update unstable here (b / eps0 > 2): diverges alike
    (3, (2 * np.pi * 15e9, 2e9, 2.0), 1.5),
    (4, (2 * np.pi * 20e9, 1e10), 1.0),
    (4, (2 * np.pi * 35e9, 0.0), 2.5),
]


@pytest.mark.parametrize("kind,params,eps_inf", CASES)
def test_dispersive_matches_numpy_restatement_bitwise(kind, params, eps_inf):
    steps = 40 if kind == 1 else 400
    s = one_cell(e0=(1.0, -0.5, 0.25))
    s.add_dispersive(kind, params, [(0, 0, 0)], eps_inf)
    s.run_batch(steps)
    got = s.probe_traces().astype(np.float32)
    with np.errstate(all="ignore"):
        want = restated_trace(kind, params, eps_inf, steps, e0=(1.0, -0.5, 0.25))
    assert np.array_equal(got, want, equal_nan=True)


def dominant_frequency(x, dt):
    x = np.asarray(x, dtype=np.float64)
    x = x - x.mean()
    n = 1 << 16
    spec = np.abs(np.fft.rfft(x * np.hanning(len(x)), n))
    return np.fft.rfftfreq(n, dt)[np.argmax(spec)]


def test_drude_plasma_oscillation_frequency():
    wp, eps_inf = 2 * np.pi * 25e9, 2.0
    s = one_cell()
    s.add_dispersive(0, (wp, 0.0), [(0, 0, 0)], eps_inf)
    s.run_batch(4000)
    f = dominant_frequency(s.probe_traces()[:, 2], DT)
    assert f == pytest.approx(wp / np.sqrt(eps_inf) / (2 * np.pi), rel=0.01)


def test_second_order_drude_plasma_frequency():
    wp, eps_inf = 2 * np.pi * 25e9, 2.0
    s = one_cell()
    s.add_dispersive(4, (wp, 0.0), [(0, 0, 0)], eps_inf)
    s.run_batch(4000)
    f = dominant_frequency(s.probe_traces()[:, 2], DT)
    assert f == pytest.approx(wp / np.sqrt(eps_inf) / (2 * np.pi), rel=0.01)


@pytest.mark.parametrize("kind,params,eps_inf,bounded", [
    (0, (2 * np.pi * 5e9, 0.0), 1.0, False),          # the reference's Drude grows
    (4, (2 * np.pi * 5e9, 0.0), 1.0, True),
    (3, (2 * np.pi * 4e9, 0.0, 3.0), 2.0, True),
])
def test_lossless_dispersive_block_in_a_closed_box(kind, params, eps_inf, bounded):
    """16^3 block of a lossless dispersive medium in a 32^3 PEC box, driven
    by a zero-mean pulse: the total E + H energy must not keep growing (it
    fluctuates: the polarisation holds part of the energy).  The reference's
    Drude update, whose current is driven by the field after the curl
    update, grows without bound here."""
    n = 32
    lines = [oracle.uniform_lines(n, 1e-3) for _ in range(3)]
    dt, delta = oracle.grid_timestep(*lines)
    s = oracle.OracleSim(n, n, n, dt, delta, threads=8)
    if eps_inf != 1.0:
        s.set_material(eps_inf, 1.0, 0.0, 0.0, (8, 24, 8, 24, 8, 24))
    s.add_dispersive(kind, params, np.mgrid[8:24, 8:24, 8:24].reshape(3, -1).T.astype(np.int64), eps_inf)
    tau = 4e-11
    t = np.arange(4000) * dt - 5 * tau
    s.add_excitation_sampled((4, 16, 16), 2, True,
                             (-(t / tau) * np.exp(-(t / tau) ** 2)).astype(np.float32))
    e = [x[3] for x in s.run_batch(4000, sample_interval=400)["energy_samples"]]
    growth = max(e[-3:]) / max(e[1:4])
    assert (growth < 3.0) == bounded, e


def test_lorentz_second_order_longitudinal_frequency():
    w0, de, eps_inf = 2 * np.pi * 12e9, 3.0, 1.5
    s = one_cell()
    s.add_dispersive(3, (w0, 0.0, de), [(0, 0, 0)], eps_inf)
    s.run_batch(4000)
    tr = s.probe_traces()[:, 0]
    assert np.isfinite(tr).all() and np.abs(tr).max() < 1.5
    f = dominant_frequency(tr, DT)
    assert f == pytest.approx(w0 * np.sqrt(1 + de / eps_inf) / (2 * np.pi), rel=0.01)


def test_debye_relaxes_to_static_ratio():
    tau, de, eps_inf = 1e-11, 3.0, 2.0
    s = one_cell()
    s.add_dispersive(2, (tau, de), [(0, 0, 0)], eps_inf)
    s.run_batch(2000)
    tr = s.probe_traces()[:, 1]
    assert tr[-1] == pytest.approx(eps_inf / (eps_inf + de), rel=1e-3)
    assert np.all(np.diff(tr) <= 0)  # monotone relaxation


def test_reference_first_order_lorentz_grows():
    """LorentzMaterial::post_update_e (dispersive.rs:171-196) drops P^{n-1};
    with a ~ 2 the field grows geometrically (about 1.25x per step here)."""
    s = one_cell()
    s.add_dispersive(1, (2 * np.pi * 15e9, 2e9, 2.0), [(0, 0, 0)], 1.0)
    s.run_batch(120)
    tr = np.abs(s.probe_traces()[:, 0])
    assert tr[-1] > 1e6 * tr[0]


def test_reference_lorentz_current_builds_up():
    """test_lorentz_material (dispersive.rs:671-698): 100 updates with Ex
    reset to 1 after each; the auxiliary current is then non-zero, seen as an
    Ex that leaves 1 on the next free update."""
    dt = 1e-15
    w0, g = 2 * np.pi * 1e14, 2 * np.pi * 1e13
    s = one_cell(dt=dt, e0=(1.0, 0.0, 0.0))
    s.add_dispersive(1, (w0, g, 1.0), [(0, 0, 0)], 1.0)
    s.add_excitation_sampled((0, 0, 0), 0, False, np.ones(100, dtype=np.float32))
    s.run_batch(100)
    assert s.probe_traces()[-1, 0] == 1.0
    s.clear_excitations()
    s.run_batch(1)
    assert s.probe_traces()[-1, 0] != 1.0


def test_reference_drude_modifies_field():
    """test_drude_material (dispersive.rs:700-721)."""
    dt = 1e-16
    s = one_cell(dt=dt, e0=(0.0, 0.0, 1.0))
    s.add_dispersive(0, (2 * np.pi * 2e15, 2 * np.pi * 1e13), [(0, 0, 0)], 1.0)
    s.run_batch(1)
    assert s.probe_traces()[0, 2] != 1.0


def test_dispersive_reset_clears_state():
    """test_material_reset (dispersive.rs:742-755): after reset the same run
    repeats bit for bit."""
    s = one_cell()
    s.add_dispersive(0, (2 * np.pi * 20e9, 1e10), [(0, 0, 0)], 1.0)
    s.run_batch(50)
    a = s.probe_traces().copy()
    s.reset()
    f = np.zeros((6, 1, 1, 1), dtype=np.float32)
    f[:3] = 1.0
    s.set_fields(f)
    s.run_batch(50)
    assert np.array_equal(a, s.probe_traces())


RLC_CASES = [
    (0, 50.0, 0.0, 0.0),
    (0, 50.0, 1e-9, 1e-12),
    (0, 0.0, 2e-9, 0.0),
    (0, 0.0, 0.0, 1e-12),
    (1, 10.0, 1e-9, 0.5e-12),
    (1, 0.0, 0.0, 1e-12),
]


@pytest.mark.parametrize("rtype,r,l,c", RLC_CASES)
@pytest.mark.parametrize("direction", [0, 2])
def test_rlc_matches_numpy_restatement_bitwise(rtype, r, l, c, direction):
    s = one_cell(e0=(0.75, -0.5, 0.25))
    s.add_lumped_rlc((0, 0, 0), direction, rtype, r, l, c)
    s.run_batch(300)
    got = s.probe_traces().astype(np.float32)
    co = nr.rlc_coeffs(rtype, r, l, c, 1e-3, DT)
    e, ii = np.float32([0.75, -0.5, 0.25][direction]), np.float32(0)
    want = np.zeros(300, dtype=np.float32)
    for n in range(300):
        e, ii = nr.rlc_step(co, e, ii, DT)
        want[n] = e
    assert np.array_equal(got[:, direction], want)
    others = [a for a in range(3) if a != direction]
    assert np.all(got[:, others] == np.float32([0.75, -0.5, 0.25])[others])


def test_parallel_resistor_decays_field():
    """test_rlc_update (lumped_rlc.rs:353-376): a 50 ohm resistor modifies Ex;
    for a parallel R alone |v_vv| < 1 so Ex decays geometrically."""
    s = one_cell(e0=(1.0, 0.0, 0.0))
    s.add_lumped_rlc((0, 0, 0), 0, 0, 50.0, 0.0, 0.0)
    s.run_batch(20)
    tr = s.probe_traces()[:, 0]
    assert tr[0] != 1.0 and np.all(np.diff(np.abs(tr)) < 0)


def test_two_elements_on_one_edge_compose_in_order():
    s = one_cell(e0=(0.0, 0.0, 1.0))
    s.add_lumped_rlc((0, 0, 0), 2, 0, 50.0, 1e-9, 0.0)
    s.add_lumped_rlc((0, 0, 0), 2, 0, 100.0, 0.0, 0.0)
    s.run_batch(50)
    c1, c2 = nr.rlc_coeffs(0, 50.0, 1e-9, 0.0, 1e-3, DT), nr.rlc_coeffs(0, 100.0, 0.0, 0.0, 1e-3, DT)
    e, i1, i2 = np.float32(1), np.float32(0), np.float32(0)
    for n in range(50):
        e, i1 = nr.rlc_step(c1, e, i1, DT)
        e, i2 = nr.rlc_step(c2, e, i2, DT)
    assert s.probe_traces()[-1, 2] == np.float32(e)


def test_lumped_resistor_coefficients():
    """set_lumped: eps = eps_r eps0 + C dl / A, sigma += dl / (R A)."""
    s = oracle.OracleSim(4, 4, 4, DT, (1e-3, 2e-3, 0.5e-3))
    scale = s.set_lumped((2, 1, 3), 1, 50.0, 1e-13, 2.0, 0.01)
    ca, cb = s.coefficients()[1][2, 1, 3], s.coefficients()[4][2, 1, 3]
    dl, area = 2e-3, 1e-3 * 0.5e-3
    eps = 2.0 * nr.EPS0 + 1e-13 * dl / area
    sig = 0.01 + dl / (50.0 * area)
    loss = sig * DT / (2 * eps)
    assert ca == np.float32((1 - loss) / (1 + loss))
    assert cb == np.float32((DT / eps) / (1 + loss) / dl)
    assert scale == pytest.approx((DT / eps) / (1 + loss) / (50.0 * area), rel=1e-15)


def test_lumped_port_dipole_on_oracle():
    """50 ohm lumped port in the gap of a 13 mm PEC wire dipole (1 mm cells,
    CPML): passive (|S11| <= 1, Re Z_in > 0) with a resonance dip below
    -10 dB between 8 and 11 GHz, the half-wave band of that length.  The
    S-parameter arithmetic is Port.CalcPort (python/openEMS/ports.py:136-138)."""
    import openems_b200 as oe
    dims, delta, pos, d = (24, 24, 30), 1e-3, (12, 12, 15), 2
    freqs = np.linspace(2e9, 14e9, 25)
    op = oe.Operator(oe.Grid.uniform(*dims, delta))
    arms = [(12, 13, 12, 13, 9, 15), (12, 13, 12, 13, 16, 22)]
    for a in arms:
        op.set_pec(a)
    port = oe.LumpedPort(1, 50.0, pos, d, excite=1.0).apply(op)
    exc = port.excitation(oe.Excitation.gaussian_modulated(8e9, 0.75, d, pos))
    dt, dl = oracle.grid_timestep(*[oracle.uniform_lines(n, delta) for n in dims])
    s = oracle.OracleSim(*dims, dt, dl, threads=4)
    for a in arms:
        s.set_pec(a)
    assert s.set_lumped(pos, d, 50.0, 0.0, 1.0, 0.0) == pytest.approx(port.source_scale, rel=1e-15)
    s.enable_cpml((6,) * 6)
    ids = []
    for kind in (0, 1):
        t = oe.port_probe(op, pos, d, kind)
        ids.append(s.add_probe_dft(s.add_probe([(c, q, -w) for c, q, w in t.terms], t.mode), freqs))
    s.add_excitation_analytic(pos, d, True, int(exc.excitation_type), list(exc.params), exc.amplitude,
                              0, 1500)
    s.run_batch(1500)
    uf, if_ = s.probe_dft(ids[0]), s.probe_dft(ids[1])
    uinc = 0.5 * (uf + if_ * 50.0)
    s11 = (uf - uinc) / uinc
    assert np.all(np.abs(s11) <= 1.0 + 1e-3)
    assert np.all(np.real(uf / if_) > 0)
    band = (freqs >= 8e9) & (freqs <= 11e9)
    assert 20 * np.log10(np.abs(s11[band]).min()) < -10.0
