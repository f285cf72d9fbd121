"""CPML and UPML absorption: how much of a pulse the 8-cell CPML of the
benchmark configuration (m = 3, R0 = 1e-6, kappa 1, alpha 0), and the
corrected UPML with the same grading, reflect.

The reference only checks that its CPML scenario stays finite
(src/fdtd/engine_testing.rs:1780-1864), and its psi is never applied to the
fields (src/extensions/cpml.rs:509-513, :598-602), so there is no reference
number to match.  This test measures the absorber on the oracle, whose CPML
the CUDA kernels reproduce bit for bit: a zero-mean modulated Gaussian
(4-20 GHz, 15-75 cells per wavelength) from the centre of a 72^3 grid with
CPML, probed 20 cells from the source, 8 cells before each slab, against the
same run in a grid 52 cells wider on every side and without CPML, whose own
faces are too far away to be seen in the window.  The difference of the two
probe traces is the reflection; it is referred to the incident peak.
"""
import numpy as np
import pytest

import oracle

N_SMALL, MARGIN, LAYERS, STEPS = 72, 52, 8, 260
F0, BW = 12e9, 8e9


def _traces(n, layers, probes, sources, precision=32, upml=False):
    lines = [oracle.uniform_lines(n, 1e-3)] * 3
    dt, d3 = oracle.grid_timestep(*lines)
    s = oracle.OracleSim(n, n, n, dt, d3, precision=precision, threads=8, zline=True)
    if layers and upml:
        s.enable_upml((layers,) * 6, 3.0, 1e-6, kind=1)
    elif layers:
        s.enable_cpml((layers,) * 6, 3.0, 1e-6, 0.0, 1.0)
    c = n // 2
    tau = 1.0 / (np.pi * BW)
    t0 = np.ceil(4 * tau * 2 * F0) / (2 * F0)  # carrier odd about t0: no DC part
    for comp in sources:
        s.add_excitation_analytic((c, c, c), comp, True, 2, [F0, t0, tau], 1.0, 0, STEPS)
    for comp, off in probes:
        s.add_point_probe(comp, tuple(c + o for o in off))
    s.run_batch(STEPS)
    return s.probe_traces()


# (component, offset from the source): broadside of the Ez source towards
# the x and y faces, of the Ex source towards the z faces
PROBES = [(2, (20, 0, 0)), (2, (-20, 0, 0)), (2, (0, 20, 0)), (2, (0, -20, 0)),
          (0, (0, 0, 20)), (0, (0, 0, -20))]


@pytest.fixture(scope="module")
def reference_traces():
    return _traces(N_SMALL + 2 * MARGIN, 0, PROBES, (2, 0))


def _reflection_db(small, big):
    out = []
    for p in range(big.shape[1]):
        inc = np.abs(big[:, p]).max()
        out.append(20.0 * np.log10(np.abs(small[:, p] - big[:, p]).max() / inc))
    return np.array(out)


def test_cpml_reflection_below_minus_60_db(reference_traces):
    small = _traces(N_SMALL, LAYERS, PROBES, (2, 0))
    refl = _reflection_db(small, reference_traces)
    print("CPML 8 reflection (dB) towards +x -x +y -y +z -z:", np.round(refl, 1))
    assert np.all(refl < -60.0), refl


def test_corrected_upml_reflection_below_minus_60_db(reference_traces):
    """The corrected UPML (kind 1) with the same grading absorbs like the
    CPML; the reference's coefficients (kind 0) grow instead."""
    small = _traces(N_SMALL, LAYERS, PROBES, (2, 0), upml=True)
    refl = _reflection_db(small, reference_traces)
    print("UPML 8 reflection (dB) towards +x -x +y -y +z -z:", np.round(refl, 1))
    assert np.all(refl < -60.0), refl


def test_measurement_sees_an_unterminated_face(reference_traces):
    """Without CPML the same probes see the faces' full reflection: the
    measurement is not blind."""
    small = _traces(N_SMALL, 0, PROBES, (2, 0))
    refl = _reflection_db(small, reference_traces)
    assert np.all(refl > -10.0), refl
