"""Frequency-domain field dumps and the NF2FF transform on the oracle (CPU).

- FrequencyDomainFieldDump known answers (src/processing/fields_fd.rs:
  403-465: accumulation, reset, sub-sampling) with the exact accumulated
  value of a constant field;
- the numpy NF2FF restatement against the exact near fields of a Hertzian
  dipole (far field, directivity 1.5, radiated power);
- an FDTD point source (a Hertzian dipole) in a CPML box recorded by the
  oracle's NF2FF box: directivity 1.5 and a sin(theta) pattern.
"""
import numpy as np
import pytest

import oracle
from oracle import nf2ff_ref as R
import openems_b200 as oe

DT = 1e-12


def test_fd_accumulation_of_constant_field():
    """test_fd_accumulation (fields_fd.rs:414-440): uniform Ex = 1, ten
    samples; each accumulates exp(-j 2 pi f t) 2 dt at t = n dt."""
    s = oracle.OracleSim(5, 5, 5, DT, (1e-3,) * 3)
    d = s.add_field_dft((0, 5, 0, 5, 0, 5), [1e9], comp_mask=0x01)
    f = np.zeros((6, 5, 5, 5), dtype=np.float32)
    f[0] = 1.0
    s.set_fields(f)
    s.run_batch(10)
    t = np.arange(1, 11) * DT
    want = np.sum(2 * DT * np.exp(-2j * np.pi * 1e9 * t))
    got = s.field_dft(d, 0, 0).reshape(5, 5, 5)
    assert np.abs(got[2, 2, 2]) > 0
    assert got[2, 2, 2] == pytest.approx(want, rel=1e-12)


def test_fd_reset():
    """test_fd_reset (fields_fd.rs:442-458)."""
    s = oracle.OracleSim(5, 5, 5, DT, (1e-3,) * 3)
    d = s.add_field_dft((0, 5, 0, 5, 0, 5), [1e9], comp_mask=0x07)
    f = np.zeros((6, 5, 5, 5), dtype=np.float32)
    f[0] = 1.0
    s.set_fields(f)
    s.run_batch(1)
    assert np.abs(s.field_dft(d, 0, 0)).max() > 0
    s.reset()
    assert np.abs(s.field_dft(d, 0, 0)).max() == 0


def test_fd_sub_sampling_and_interval():
    """set_sub_sample (fields_fd.rs:126-128): points every ss cells; with
    interval 3 only multiples of 3 are taken, scaled by 2 dt 3."""
    s = oracle.OracleSim(7, 6, 9, DT, (1e-3,) * 3)
    d = s.add_field_dft((1, 7, 0, 6, 2, 9), [2e9, 5e9], comp_mask=0x24, sub_sample=(2, 4, 3),
                        interval=3)
    assert oracle.lib().orc_field_dft_points(s._h, d) == 3 * 2 * 3
    f = np.zeros((6, 7, 6, 9), dtype=np.float32)
    f[5] = 0.5
    s.set_fields(f)
    s.run_batch(10)
    hz = s.field_dft(d, 1, 5).reshape(3, 2, 3)
    t = (np.array([3, 6, 9]) - 0.5) * DT
    want = np.sum(0.5 * 6 * DT * np.exp(-2j * np.pi * 5e9 * t))
    # Hz stays 0.5 only away from the max faces' zero forward differences
    assert hz[0, 0, 0] == pytest.approx(want, rel=1e-12)


def test_numpy_nf2ff_reproduces_hertzian_dipole():
    f = 3e9
    lam = R.C0 / f
    pts = R.dipole_box_points(0.25 * lam, 40, f, il=1e-3)
    th = np.linspace(0, np.pi, 37)
    ph = np.linspace(0, 2 * np.pi, 73)
    r = R.far_field(pts, f, th, ph, radius=2.0)
    ana = R.dipole_far_field(f, th, 2.0, il=1e-3)
    for j in (0, 17, 50):
        assert np.abs(r["E_theta"][:, j] - ana).max() < 1e-3 * np.abs(ana).max()
    assert np.abs(r["E_phi"]).max() < 1e-3 * np.abs(ana).max()
    assert r["Dmax"] == pytest.approx(1.5, rel=1e-3)
    prad = R.Z0 * np.pi / 3 * (1e-3 / lam) ** 2  # eta pi / 3 (I l / lambda)^2
    assert r["Prad"] == pytest.approx(prad, rel=2e-3)


def fdtd_dipole(n=48, freqs=(6e9, 10e9), steps=900, threads=8):
    lines = [oracle.uniform_lines(n, 1e-3) for _ in range(3)]
    dt, dl = oracle.grid_timestep(*lines)
    s = oracle.OracleSim(n, n, n, dt, dl, threads=threads)
    s.enable_cpml((8,) * 6)
    lo, hi = (13,) * 3, (n - 13,) * 3
    bid = s.add_nf2ff_box(lo, hi, list(freqs))
    c = n // 2
    exc = oe.Excitation.gaussian_modulated(10e9, 0.5, 2, (c, c, c))
    s.add_excitation_analytic((c, c, c), 2, True, int(exc.excitation_type), list(exc.params), 1.0,
                              0, steps)
    s.run_batch(steps)
    return s, bid, lo, hi, [np.asarray(v, dtype=np.float64) for v in lines]


def test_oracle_fdtd_dipole_directivity():
    """A soft Ez point source radiates as a Hertzian dipole: D = 1.5 and
    E_theta ~ sin(theta), E_phi ~ 0, from the recorded box."""
    s, bid, lo, hi, lines = fdtd_dipole()
    th = np.linspace(0, np.pi, 37)
    ph = np.linspace(0, 2 * np.pi, 73)
    for fi, f in enumerate((6e9, 10e9)):
        pts = np.concatenate([R.face_points(lo, hi, face, lines, s.nf2ff_face(bid, face, fi, lo, hi))
                              for face in range(6)])
        r = R.far_field(pts, f, th, ph, 1.0, center=(24e-3, 24e-3, 24.5e-3))
        et = np.abs(r["E_theta"])
        assert r["Dmax"] == pytest.approx(1.5, rel=0.01)
        assert np.abs(r["E_phi"]).max() < 1e-3 * et.max()
        assert np.abs(et[:, 0] / et.max() - np.sin(th)).max() < 0.01
