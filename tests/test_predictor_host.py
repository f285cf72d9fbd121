"""Host side of early termination (no GPU): the closed-form tail DFT, the
pole-grid fit, the matrix-pencil continuation on known damped sinusoids,
and the seeded patch family."""
import numpy as np
import pytest

from openems_b200 import predictor as P

DT = P.grid_dt()
FREQS = P.FREQS[::4]


def damped(n, modes, dt=DT, start=0):
    """sum_m a_m exp(-alpha_m t) cos(omega_m t + phi_m) at t = (start + k) dt."""
    t = (start + np.arange(n)) * dt
    return sum(a * np.exp(-al * t) * np.cos(w * t + ph) for a, al, w, ph in modes)


MODES = [(1.0, 2.0e8, 2 * np.pi * 3.1e9, 0.3), (0.4, 6.0e8, 2 * np.pi * 7.7e9, -1.1),
         (0.15, 1.0e8, 2 * np.pi * 1.3e9, 2.0)]


def test_tail_dft_closed_form_matches_direct_sum():
    poles = P.PoleGrid(nf=6, qs=(10.0,)).poles()
    c = np.random.default_rng(0).normal(size=6) + 1j * np.random.default_rng(1).normal(size=6)
    n, t0 = 3000, 123.5 * DT
    x = (np.exp(np.outer(np.arange(n) * DT, poles)) @ c).real
    want = 2 * DT * (np.exp(-2j * np.pi * np.outer(FREQS, t0 + np.arange(n) * DT)) @ x)
    got = P.tail_dft(c, poles, t0, DT, FREQS, n)
    assert np.abs(got - want).max() < 1e-10 * np.abs(want).max()


def test_head_dft_is_the_engine_probe_dft():
    x = np.random.default_rng(2).normal(size=50)
    got = P.head_dft(x, 1, DT, FREQS, half=0.5)
    want = [2 * DT * sum(x[k] * np.exp(-2j * np.pi * f * (k + 1 - 0.5) * DT) for k in range(50)) for f in FREQS]
    assert np.allclose(got, want, rtol=1e-12, atol=0)


def test_tail_matrix_matches_tail_dft():
    poles = P.PoleGrid().poles()
    T = P.tail_matrix(poles, 2048, DT, FREQS, 0.5, 6000)
    c = np.random.default_rng(0).normal(size=64) + 1j * np.random.default_rng(1).normal(size=64)
    x = P.tail_dft(c, poles, (2048 + 1 - 0.5) * DT, DT, FREQS, 6000 - 2048)
    y = T @ np.concatenate([c.real, c.imag])
    F = len(FREQS)
    assert np.abs(y[:F] - x.real).max() < 1e-12 * np.abs(x).max()
    assert np.abs(y[F:] - x.imag).max() < 1e-12 * np.abs(x).max()


def test_fit_tail_recovers_grid_coefficients():
    poles = P.PoleGrid(nf=8, qs=(8.0,)).poles()
    c = np.random.default_rng(3).normal(size=8) + 1j * np.random.default_rng(4).normal(size=8)
    tail = (np.exp(np.outer(np.arange(4000) * DT, poles)) @ c).real
    got = P.fit_tail(tail, poles, DT, ridge=0.0)
    assert np.abs(got - c).max() < 1e-6 * np.abs(c).max()
    assert np.all(P.fit_tail(np.zeros(0), poles, DT) == 0)


def test_matrix_pencil_finds_damped_modes():
    y = damped(400, MODES)
    z, r = P.matrix_pencil(y, 20)
    assert len(z) == 6
    k = np.arange(400)
    assert np.abs((np.power.outer(z, k).T @ r).real - y).max() < 1e-9
    got = np.sort(np.abs(np.angle(z)) / DT / (2 * np.pi))
    want = np.sort(np.repeat([m[2] / (2 * np.pi) for m in MODES], 2))
    assert np.allclose(got, want, rtol=1e-8)
    # growing or silent input: nothing to continue
    assert len(P.matrix_pencil(np.zeros(64), 8)[0]) == 0
    assert len(P.matrix_pencil(1.01 ** np.arange(64), 8)[0]) == 0


@pytest.mark.parametrize("half", [0.0, 0.5])
def test_pencil_continuation_of_known_signal(half):
    """The continuation of a sum of damped sinusoids from a 1536-sample
    window is the exact DFT of its remaining samples."""
    K, horizon = 2048, 12000
    x = damped(horizon, MODES)
    got = P.pencil_tail_dft(x[:K], K, DT, FREQS, half, horizon)
    want = P.head_dft(x[K:], K + 1, DT, FREQS, half)
    assert np.abs(got - want).max() < 1e-6 * np.abs(want).max()
    # a signal that has already died away continues as nothing
    assert np.all(P.pencil_tail_dft(np.zeros(K), K, DT, FREQS, half, horizon) == 0)


def test_s11_of_matched_and_open_port():
    uf = np.array([50.0 + 0j, 1.0 + 0j])
    if_ = np.array([1.0 + 0j, 0.0 + 0j])
    assert np.allclose(P.s11(uf, if_), [0.0, 1.0])


def test_family_specs_seeded_and_in_range():
    a, b = P.family_specs(32, seed=5), P.family_specs(32, seed=5)
    assert a == b and a != P.family_specs(32, seed=50)
    for s in a:
        assert all(40 <= n <= 80 for n in s.dims)
        assert 2.2 <= s.eps_r <= 10.2 and 2 <= s.h_cells <= 6
        margin = s.layers + 4
        assert s.x0 >= margin - 1 and s.x0 + s.W <= s.dims[0] - margin + 1
        assert s.y0 >= margin - 1 and s.y0 + s.L <= s.dims[1] - margin + 1
        assert s.x0 <= s.fx < s.x0 + s.W and s.y0 <= s.fy < s.y0 + s.L
        assert s.k_patch + 1 < s.dims[2] - s.layers


def test_s11_db_error_clips_at_floor():
    from openems_b200 import early_stop as E
    a = np.array([1e-3, 0.5, 0.9])
    b = np.array([1e-4, 0.5 * 10 ** (0.2 / 20), 0.9])
    band = np.array([True, True, True])
    # -60 dB vs -80 dB both clip at -30 dB: no error there
    assert E.s11_db_error(a, b, band) == pytest.approx(0.2, rel=1e-9)
    assert E.s11_db_error(a, b, np.array([True, False, True])) == 0.0


@pytest.mark.parametrize("lag", [0, 256])
def test_pencil_s11_of_known_ringdown(lag):
    """Port traces made of damped sinusoids: the prediction at K (from the
    window ending at K - lag) equals the S11 of the whole traces."""
    from openems_b200 import early_stop as E
    K, H = 2048, 12000
    u = damped(H, MODES)
    i = 0.02 * damped(H, [(1.0, 2.0e8, 2 * np.pi * 3.1e9, 0.7), (0.3, 6.0e8, 2 * np.pi * 7.7e9, 0.1)])
    tr = np.stack([u, i], 1)
    uf, if_ = P.head_dft(u[:K], 1, DT, FREQS, 0.0), P.head_dft(i[:K], 1, DT, FREQS, 0.5)
    full = P.s11(P.head_dft(u, 1, DT, FREQS, 0.0), P.head_dft(i, 1, DT, FREQS, 0.5))
    got = E.pencil_s11(tr, uf, if_, K, DT, FREQS, H, lag)
    assert E.s11_db_error(got, full, FREQS >= 0.5e9) < 1e-6


def test_staged_rule_on_calibration_records():
    from openems_b200 import early_stop as E
    nan = np.nan
    cal = {"check_db": np.array([[0.5, 0.05, 0.01], [0.01, 0.2, 0.3], [nan, nan, nan], [0.4, nan, nan],
                                 [0.3, 0.3, 0.3]]),
           "error_db": np.array([[2.0, 0.3, 0.1], [0.04, 0.5, 0.6], [nan, nan, nan], [1.0, nan, nan],
                                 [1.0, 1.0, 1.0]])}
    sim = E.simulate(cal, 0.1)
    assert list(sim["stop"]) == [1, 0, -1, -1, -1]
    assert np.allclose(sim["error_db"], [0.3, 0.04, 0.0, 0.0, 0.0])


def test_plain_end_of_single_mode_decay():
    """One mode decaying at alpha: the plain run's energy falls 50 dB below
    its peak at ln(1e5) / (2 alpha); the estimate lands on the next 100-step
    check after that."""
    from openems_b200 import early_stop as E
    K, H, alpha = 2048, 40000, 2e8
    u = damped(K, [(1.0, alpha, 2 * np.pi * 3e9, 0.0)])
    level = 10 * np.log10(np.exp(-2 * alpha * K * DT))
    end = E.plain_end(u, K, level, DT, 50.0, H, **E.StagePlan().pencil(K))
    want = np.log(1e5) / (2 * alpha) / DT
    assert want <= end < want + 100
    # already decayed: the end is now; a cap that comes first wins
    assert E.plain_end(u, K, -60.0, DT, 50.0, H, **E.StagePlan().pencil(K)) == K
    assert E.plain_end(u, K, level, DT, 50.0, 20000, **E.StagePlan().pencil(K)) == 20000


def _small_ref(seed=0):
    from oracle.tailnet_ref import TailNetRef
    rng = np.random.default_rng(seed)
    convs = [(rng.normal(0, 0.4, (4, 8 * 2)), rng.normal(0, 0.1, 4)),
             (rng.normal(0, 0.3, (6, 8 * 4)), rng.normal(0, 0.1, 6))]
    # T 64 -> 15 -> 2
    fc1 = (rng.normal(0, 0.3, (10, 2 * 6)), rng.normal(0, 0.1, 10))
    fc2 = (rng.normal(0, 0.3, (8, 10)), rng.normal(0, 0.1, 8))
    spec = rng.normal(0, 0.5, (12, 8))
    return TailNetRef(convs, fc1, fc2, spec), rng.normal(size=(3, 64, 2))


def test_tailnet_oracle_gradients_match_finite_differences():
    """Pins the CPU restatement of the network: its hand-written backward
    equals central differences of its forward (float64, no bf16)."""
    net, x = _small_ref()
    G = np.random.default_rng(9).normal(size=(3, 12))
    net.forward(x)
    grads = net.backward(G)
    params = [p for c in net.convs for p in c] + list(net.fc1) + list(net.fc2)
    flat = [g for pair in grads for g in pair]
    rng = np.random.default_rng(10)
    for p, g in zip(params, flat):
        for _ in range(4):
            idx = tuple(rng.integers(0, n) for n in p.shape)
            old = p[idx]
            p[idx] = old + 1e-6
            up = (net.forward(x) * G).sum()
            p[idx] = old - 1e-6
            dn = (net.forward(x) * G).sum()
            p[idx] = old
            assert g[idx] == pytest.approx((up - dn) / 2e-6, rel=1e-5, abs=1e-8)


def test_tailnet_oracle_im2col_adjoint_and_bf16_rounding():
    from oracle.tailnet_ref import col2im, im2col, round_bf16
    rng = np.random.default_rng(1)
    x, d = rng.normal(size=(2, 37, 3)), rng.normal(size=(2 * 8, 8 * 3))
    assert np.isclose((im2col(x, 8, 4) * d).sum(), (x * col2im(d, 2, 37, 3, 8, 4)).sum(), rtol=1e-12)
    # round to nearest even on the 16 dropped bits
    v = np.array([1.0, 1.0 + 2 ** -8, 1.0 + 3 * 2 ** -8, 1.0 + 2 ** -9, -2.5], dtype=np.float64)
    assert list(round_bf16(v)) == [1.0, 1.0, 1.0 + 2 ** -6, 1.0, -2.5]


def _small_stage_ref():
    from oracle.tailnet_ref import StageNetRef
    rng = np.random.default_rng(21)
    ch, ks = 6, 3
    convs = [(rng.normal(0, 0.4, (ch, ks * 4)), rng.normal(0, 0.1, ch))] + \
            [(rng.normal(0, 0.3, (ch, ks * ch)), rng.normal(0, 0.1, ch)) for _ in range(2)]
    fc1 = (rng.normal(0, 0.3, (9, ch + 3)), rng.normal(0, 0.1, 9))
    fc2 = (rng.normal(0, 0.3, (4, 9)), rng.normal(0, 0.1, 4))
    return StageNetRef(convs, fc1, fc2, ks), rng.normal(size=(3, 40, 4)), rng.normal(size=(3, 3))


def test_stagenet_oracle_gradients_match_finite_differences():
    """Pins the CPU restatement of the acceptance network (causal dilated
    TCN read at the last step, scalars, MLP): its hand-written backward
    equals central differences of its forward (float64)."""
    net, x, s = _small_stage_ref()
    G = np.random.default_rng(22).normal(size=(3, 4))
    net.forward(x, s)
    grads = net.backward(G)
    params = [p for c in net.convs for p in c] + list(net.fc1) + list(net.fc2)
    flat = [g for pair in grads for g in pair]
    rng = np.random.default_rng(23)
    for p, g in zip(params, flat):
        for _ in range(4):
            idx = tuple(rng.integers(0, n) for n in p.shape)
            old = p[idx]
            p[idx] = old + 1e-6
            up = (net.forward(x, s) * G).sum()
            p[idx] = old - 1e-6
            dn = (net.forward(x, s) * G).sum()
            p[idx] = old
            assert g[idx] == pytest.approx((up - dn) / 2e-6, rel=1e-5, abs=1e-8)


def test_causal_im2col_adjoint_and_causality():
    from oracle.tailnet_ref import col2im_causal, im2col_causal
    rng = np.random.default_rng(3)
    x, d = rng.normal(size=(2, 29, 3)), rng.normal(size=(2 * 29, 5 * 3))
    assert np.isclose((im2col_causal(x, 5, 4) * d).sum(), (x * col2im_causal(d, 2, 29, 3, 5, 4)).sum(),
                      rtol=1e-12)
    cols = im2col_causal(x, 5, 4).reshape(2, 29, 5, 3)
    assert np.array_equal(cols[:, 20, 4], x[:, 20]) and np.array_equal(cols[:, 20, 0], x[:, 4])
    assert not cols[:, 3, :4].any()  # before the start


def test_stage_rule_threshold_and_evaluation():
    """first_accept / choose_threshold / evaluate on hand-made records: two
    instances, three stages."""
    from openems_b200 import stage_net as SN
    score = np.array([0.5, -0.2, -0.9, 0.1, -0.5])
    err = np.array([2.0, 0.3, 0.1, 0.9, 0.2])
    stage = np.array([0, 1, 2, 0, 1])
    inst = np.array([0, 0, 0, 1, 1])
    acc, worst = SN.first_accept(score, err, stage, inst, 0.0)
    assert acc == {0: 1, 1: 1} and worst == 0.3
    acc, worst = SN.first_accept(score, err, stage, inst, 0.2)
    assert acc == {0: 1, 1: 0} and worst == 0.9
    thr = SN.choose_threshold(score, err, stage, inst, limit_db=0.5)
    assert SN.first_accept(score, err, stage, inst, thr)[1] <= 0.5 and thr >= -0.2
    r = SN.evaluate(score, 0.0, err, stage, inst, [100, 200, 400], np.array([1000.0, 1000.0]))
    assert r["accepted"] == 2 and r["over_limit"] == 0 and r["step_ratio"] == pytest.approx(2000 / 400)


def test_stage_inputs_window_and_scalars():
    """The acceptance network's inputs: the window ends at K - 1, keeps the
    newest samples, is scaled per channel, and pads short windows at the
    front with zeros."""
    from openems_b200 import stage_net as SN
    t = np.arange(5000, dtype=np.float64)
    trace = np.stack([np.sin(t / 7.0) * (1 + t), np.cos(t / 5.0)], axis=1)
    x = SN.window_input(trace, 4096, 3072)
    assert x.shape == (SN.T_WIN, SN.C_IN) and x.dtype == np.float32
    dec = 3072 // SN.T_WIN
    w = trace[4096 - 3072:4096][::-1][::dec][::-1][-SN.T_WIN:]
    assert np.allclose(x[:, :2], w / np.abs(w).max(axis=0), rtol=1e-6)
    assert not x[:, 2:].any()
    short = SN.window_input(trace, 300, 3072)
    assert not short[:SN.T_WIN - (300 + dec - 1) // dec, :2].any() and np.abs(short[-1, :2]).max() > 0
    s = SN.scalar_input(0.2, 0.05, 0.4, 1.5, -23.0, 4096, 20000)
    assert s.shape == (SN.N_SCALAR,) and s[-1] == 1.0
    assert s[0] == pytest.approx(np.log10(0.21)) and s[3] == pytest.approx(np.log10(1.51))
    assert s[5] == pytest.approx(2.0 / 5.0)
