"""Frequency-domain field dumps, NF2FF box recording and the GPU far-field
transform against the oracle and the numpy restatement."""
import numpy as np
import pytest

import oracle
from oracle import nf2ff_ref as R
import openems_b200 as oe
from scenarios import make_operator, Scenario
from test_gpu_parity import KERNELS

pytestmark = pytest.mark.gpu


def fd_scenario():
    E = oe.Excitation
    return Scenario("fd_cpml", (22, 19, 26), 1e-3,
                    materials=[(3.0, 1.0, 0.02, 0.0, (4, 12, 3, 15, 6, 20))],
                    excitations=[E.gaussian_modulated(9e9, 0.5, 2, (11, 9, 13)),
                                 E.gaussian_modulated(6e9, 0.5, 0, (8, 12, 10))],
                    num_steps=230, cpml=oe.CpmlBoundaries.uniform(4), batches=(100, 130))


DUMPS = [  # region, freqs, mask, sub-sampling, interval
    ((0, 22, 0, 19, 0, 26), [3e9, 9e9], 0x3F, (1, 1, 1), 1),
    ((3, 20, 2, 17, 5, 25), [5e9], 0x05, (2, 3, 4), 3),
    ((10, 11, 0, 19, 0, 26), [4e9, 7e9, 11e9], 0x30, (1, 1, 1), 2),
]
BOX = ((5, 4, 6), (17, 15, 21), [6e9, 9e9], (1, 1, 0, 1, 1, 1), 1)


def run_both(kernels):
    sc = fd_scenario()
    op = make_operator(sc)
    eng = oe.Engine(op, kernels=kernels)
    eng.add_cpml(sc.cpml)
    ids = [eng.add_field_dft(r, f, m, ss, iv) for r, f, m, ss, iv in DUMPS]
    lo, hi, bf, dirs, biv = BOX
    box = oe.Nf2ffBox(eng, lo, hi, bf, directions=dirs, interval=biv)
    lines = [oracle.uniform_lines(n, sc.delta) for n in sc.dims]
    dt, delta = oracle.grid_timestep(*lines)
    s = oracle.OracleSim(*sc.dims, dt, delta)
    for m in sc.materials:
        s.set_material(*m)
    s.enable_cpml(sc.cpml.layers)
    oids = [s.add_field_dft(r, f, m, ss, iv) for r, f, m, ss, iv in DUMPS]
    obox = s.add_nf2ff_box(lo, hi, bf, dirs, biv)
    start = 0
    for n in sc.batch_sizes():
        sched = [oe.ScheduledExcitation.from_excitation(x, start, n, dt) for x in sc.excitations]
        eng.run_batch(oe.EngineBatch(num_steps=n, excitations=sched))
        s.clear_excitations()
        for x in sc.excitations:
            s.add_excitation_analytic(x.position, x.direction, True, int(x.excitation_type),
                                      list(x.params), 1.0, start, n)
        s.run_batch(n)
        start += n
    return eng, ids, box, s, oids, obox, [np.asarray(v, dtype=np.float64) for v in lines]


@pytest.mark.parametrize("kernels", KERNELS)
def test_field_dft_and_box_bit_exact(kernels):
    eng, ids, box, s, oids, obox, _ = run_both(kernels)
    e, h = eng.read_fields()
    assert np.array_equal(np.concatenate([e, h]), s.fields())
    for (r, f, m, ss, iv), d, od in zip(DUMPS, ids, oids):
        for fi in range(len(f)):
            for c in range(6):
                if m >> c & 1:
                    got = eng.field_dft(d, fi, c).reshape(-1)
                    assert np.array_equal(got, s.field_dft(od, fi, c)), (r, fi, c)
    lo, hi, bf, dirs, _ = BOX
    for face in range(6):
        for fi in range(len(bf)):
            ref = s.nf2ff_face(obox, face, fi, lo, hi)
            if not dirs[face]:
                assert ref is None
                with pytest.raises(oe.ConfigError):
                    box.face(face, fi)
                continue
            assert np.array_equal(box.face(face, fi), ref), (face, fi)


def test_far_field_matches_numpy_restatement():
    eng, _, box, s, _, obox, lines = run_both("register")
    lo, hi, bf, dirs, _ = BOX
    th = np.deg2rad(np.arange(0, 181, 5.0))
    ph = np.deg2rad(np.arange(0, 361, 10.0))
    res = box.calc_nf2ff(bf, th, ph, radius=1.5, center=(0.011, 0.009, 0.013), degrees=False)
    for fi, f in enumerate(bf):
        pts = np.concatenate([R.face_points(lo, hi, face, lines, s.nf2ff_face(obox, face, fi, lo, hi))
                              for face in range(6) if dirs[face]])
        ref = R.far_field(pts, f, th, ph, 1.5, center=(0.011, 0.009, 0.013))
        scale = np.abs(ref["E_theta"]).max() + np.abs(ref["E_phi"]).max()
        assert np.abs(res.E_theta[fi] - ref["E_theta"]).max() <= 1e-10 * scale
        assert np.abs(res.E_phi[fi] - ref["E_phi"]).max() <= 1e-10 * scale
        assert res.Prad[fi] == pytest.approx(ref["Prad"], rel=1e-9)
        assert res.Dmax[fi] == pytest.approx(ref["Dmax"], rel=1e-9)
        assert np.allclose(res.P_rad[fi], ref["P_rad"], rtol=1e-9, atol=1e-12 * ref["P_rad"].max())


def test_surface_transform_of_exact_dipole_fields():
    f = 3e9
    lam = R.C0 / f
    pts = R.dipole_box_points(0.25 * lam, 40, f, il=1e-3)
    th = np.linspace(0, np.pi, 37)
    ph = np.linspace(0, 2 * np.pi, 73)
    res = oe.nf2ff_surface(pts, f, th, ph, radius=2.0)
    ref = R.far_field(pts, f, th, ph, radius=2.0)
    scale = np.abs(ref["E_theta"]).max()
    assert np.abs(res.E_theta[0] - ref["E_theta"]).max() <= 1e-10 * scale
    ana = R.dipole_far_field(f, th, 2.0, il=1e-3)
    assert np.abs(res.E_theta[0][:, 0] - ana).max() < 1e-3 * np.abs(ana).max()
    assert res.Dmax[0] == pytest.approx(1.5, rel=1e-3)


def test_fdtd_dipole_directivity_on_gpu():
    """Soft Ez point source in a 64^3 CPML box: the GPU-recorded box gives
    D = 1.5 and a sin(theta) pattern at 5 and 10 GHz.  The source is a
    derivative-of-Gaussian pulse: a waveform with a DC part leaves a static
    charge whose truncated DFT is not a radiating field (the reference's
    modulated Gaussian, whose carrier is not centred on t0, has one)."""
    n = 64
    c = n // 2
    op = oe.Operator(oe.Grid.uniform(n, n, n, 1e-3), oe.BoundaryConditions.all_pec())
    eng = oe.Engine(op)
    eng.add_cpml(oe.CpmlBoundaries.uniform(8))
    box = oe.Nf2ffBox(eng, (14,) * 3, (n - 14,) * 3, [5e9, 10e9])
    dt = op.timestep()
    tau = 4e-11
    t = np.arange(1200) * dt - 5 * tau
    wave = (-(t / tau) * np.exp(-(t / tau) ** 2)).astype(np.float32)
    for start in (0, 600):
        eng.run_batch(oe.EngineBatch(num_steps=600, excitations=[
            oe.ScheduledExcitation((c, c, c), 2, True, wave[start:start + 600])]))
    th = np.arange(0, 181, 5.0)
    ph = np.arange(0, 361, 10.0)
    res = box.calc_nf2ff([5e9, 10e9], th, ph, center=(c * 1e-3, c * 1e-3, (c + 0.5) * 1e-3))
    for fi in range(2):
        et = np.abs(res.E_theta[fi])
        assert res.Dmax[fi] == pytest.approx(1.5, rel=0.01)
        assert np.abs(res.E_phi[fi]).max() < 2e-3 * et.max()
        assert np.abs(et[:, 0] / et.max() - np.sin(np.deg2rad(th))).max() < 0.01


def test_reset_clears_recorders():
    eng, ids, box, *_ = run_both("register")
    eng.reset()
    assert np.abs(eng.field_dft(ids[0], 0, 2)).max() == 0
    assert np.abs(box.face(0, 0)).max() == 0


def test_invalid_recorders():
    op = oe.Operator(oe.Grid.uniform(10, 10, 10, 1e-3), oe.BoundaryConditions.all_pec())
    eng = oe.Engine(op)
    with pytest.raises(oe.ConfigError):
        oe.Nf2ffBox(eng, (0, 2, 2), (8, 8, 8), [1e9])
    with pytest.raises(oe.ConfigError):
        oe.Nf2ffBox(eng, (2, 2, 2), (10, 8, 8), [1e9])
    with pytest.raises(oe.ConfigError):
        eng.add_field_dft((0, 10, 0, 10, 0, 10), [1e9], components=0)
    with pytest.raises(oe.ConfigError):
        eng.add_field_dft((4, 4, 0, 10, 0, 10), [1e9])
    box = oe.Nf2ffBox(eng, (2, 2, 2), (8, 8, 8), [1e9])
    with pytest.raises(oe.ConfigError):
        box.calc_nf2ff(2e9, [0, 90], [0])
