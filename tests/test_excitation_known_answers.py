"""The rest of the reference's Excitation unit tests
(src/fdtd/excitation.rs:254-636, tests module) on the Python mirror and its
C++ host functions: amplitude, hard source, custom waveforms (evaluation,
interpolation, clamping), durations, activity windows and the TE10 helper.
The analytic waveform values themselves are pinned in
test_oracle_known_answers.py.  CPU only."""
import math

import numpy as np
import pytest

import openems_b200 as oe
from openems_b200.fdtd import ExcitationType

E = oe.Excitation


def _gaussian():
    return E.gaussian(1e9, 0.5, 2, (10, 10, 10))


def test_with_amplitude():
    exc = _gaussian().with_amplitude(2.5)
    assert exc.amplitude == 2.5
    t0 = exc.params[0]
    assert exc.evaluate(t0) == pytest.approx(2.5, abs=1e-10)


def test_hard_source():
    assert not _gaussian().hard_source().soft_source


def test_custom_excitation():
    exc = E.custom([0.0, 1.0, 2.0, 3.0], [0.0, 1.0, 0.5, 0.0], 2, (5, 5, 5))
    for t, v in ((0.0, 0.0), (1.0, 1.0), (2.0, 0.5), (3.0, 0.0), (0.5, 0.5), (1.5, 0.75), (-1.0, 0.0),
                 (5.0, 0.0)):
        assert exc.evaluate(t) == pytest.approx(v, abs=1e-10), t


def test_custom_excitation_with_amplitude():
    exc = E.custom([0.0, 1.0, 2.0], [0.0, 1.0, 0.0], 2, (5, 5, 5), amplitude=5.0)
    assert exc.evaluate(1.0) == pytest.approx(5.0, abs=1e-10)
    assert exc.evaluate(0.5) == pytest.approx(2.5, abs=1e-10)


def test_custom_waveform_samples_like_the_others():
    """sample(start, n, dt) = (f32) evaluate((start + k) dt) for a custom
    waveform, as ScheduledExcitation::from_excitation does for every kind."""
    dt = 1e-12
    exc = E.custom([0.0, 5e-12, 1e-11], [0.0, 2.0, -1.0], 1, (3, 4, 5))
    s = exc.sample(2, 10, dt)
    want = np.array([exc.evaluate((2 + k) * dt) for k in range(10)], dtype=np.float32)
    assert s.dtype == np.float32 and np.array_equal(s, want)
    sched = oe.ScheduledExcitation.from_excitation(exc, 2, 10, dt)
    assert np.array_equal(sched.samples, want) and sched.position == (3, 4, 5)


@pytest.mark.parametrize("kind", ["gaussian", "gaussian_modulated"])
def test_duration_gaussian(kind):
    exc = getattr(E, kind)(1e9, 0.5, 2, (10, 10, 10))
    t0, tau = exc.params[-2], exc.params[-1]
    assert abs(exc.duration() - (t0 + 6.0 * tau)) < 1e-20


def test_duration_infinite_kinds():
    assert math.isinf(E.sinusoidal(1e9, 0, (5, 5, 5)).duration())
    assert math.isinf(E(ExcitationType.Dirac, (), 0, (5, 5, 5)).duration())
    assert math.isinf(E(ExcitationType.Step, (), 0, (5, 5, 5)).duration())


def test_duration_custom():
    assert E.custom([0.0, 1.0, 2.0, 3.0], [0.0, 1.0, 0.5, 0.0], 2, (5, 5, 5)).duration() == 3.0
    assert E.custom([], [], 2, (5, 5, 5)).duration() == 0.0


@pytest.mark.parametrize("kind", ["gaussian", "gaussian_modulated"])
def test_is_active_gaussian(kind):
    exc = getattr(E, kind)(1e9, 0.5, 2, (10, 10, 10))
    t0, tau = exc.params[-2], exc.params[-1]
    end = t0 + 6.0 * tau
    assert exc.is_active(0.0) and exc.is_active(t0) and exc.is_active(end)
    assert not exc.is_active(end + 1.0)


def test_is_active_other_kinds():
    s = E.sinusoidal(1e9, 0, (5, 5, 5))
    assert s.is_active(0.0) and s.is_active(1e10)
    d = E(ExcitationType.Dirac, (), 0, (5, 5, 5))
    assert d.is_active(0.0) and not d.is_active(1e-9) and not d.is_active(-1e-9)
    st = E(ExcitationType.Step, (), 0, (5, 5, 5))
    assert st.is_active(0.0) and st.is_active(1e10)
    c = E.custom([0.0, 1.0, 2.0, 3.0], [0.0, 1.0, 0.5, 0.0], 2, (5, 5, 5))
    assert c.is_active(0.0) and c.is_active(1.5) and c.is_active(3.0) and not c.is_active(4.0)


def test_waveguide_te10_creation():
    exc = oe.waveguide_te10(0.01, 10e9, 5, 20)
    assert exc
    assert all(x.excitation_type == ExcitationType.Sinusoidal and x.direction == 1 and x.position[2] == 5
               for x in exc)
    assert exc[len(exc) // 2].amplitude > exc[0].amplitude


def test_custom_waveform_is_refused_by_the_analytic_host_path():
    with pytest.raises(oe.ConfigError):
        E.custom([0.0, 1.0], [0.0, 1.0], 2, (1, 1, 1)).to_c()
