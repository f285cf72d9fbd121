"""The dispersive scattering scene (Drude sphere, Lorentz shell, lumped-port
dipole, CPML, NF2FF box) at a small size against the oracle."""
import numpy as np
import pytest

import oracle
from oracle import nf2ff_ref as R
import openems_b200 as oe
from openems_b200.scene import ScatterScene, run

pytestmark = pytest.mark.gpu


def small():
    return ScatterScene(n=48, layers=4, steps=400, nf2ff_interval=3)


@pytest.mark.parametrize("kernels", ("register", "staged"))
def test_scene_matches_oracle(kernels):
    sc = small()
    op, port, sphere, shell = sc.operator()
    eng = oe.Engine(op, kernels=kernels)
    box = sc.attach(eng, port, sphere, shell)
    exc = port.excitation(sc.waveform())
    dt = op.timestep()

    lines = [oracle.uniform_lines(sc.n, sc.delta) for _ in range(3)]
    odt, delta = oracle.grid_timestep(*lines)
    assert odt == dt
    s = oracle.OracleSim(sc.n, sc.n, sc.n, dt, delta, threads=4)
    s.set_coefficients(op.coefficients())
    s.enable_cpml((sc.layers,) * 6)
    wp, g = sc.drude
    s.add_dispersive(4, (wp, g), sphere.astype(np.int64), 1.0)
    w0, gl, de, ei = sc.lorentz
    s.add_dispersive(3, (w0, gl, de), shell.astype(np.int64), ei)
    dft = []
    for kind in (0, 1):
        t = oe.port_probe(op, sc.port, 2, kind)
        dft.append(s.add_probe_dft(s.add_probe([(c, q, -w) for c, q, w in t.terms], t.mode), list(sc.freqs)))
    lo, hi = sc.box
    obox = s.add_nf2ff_box(lo, hi, list(sc.freqs), interval=sc.nf2ff_interval)
    start = 0
    for n in (150, 250):
        eng.run_batch(oe.EngineBatch(num_steps=n, excitations=[
            oe.ScheduledExcitation.from_excitation(exc, start, n, dt)]))
        s.clear_excitations()
        s.add_excitation_analytic(sc.port, 2, True, int(exc.excitation_type), list(exc.params), exc.amplitude,
                                  start, n)
        s.run_batch(n)
        start += n
    e, h = eng.read_fields()
    f = s.fields()
    assert np.isfinite(f).all() and np.abs(f).max() > 0
    assert np.array_equal(np.concatenate([e, h]), f)
    port.calc_port(eng)
    for got, d in zip((port.uf_tot, port.if_tot), dft):
        ref = s.probe_dft(d)
        assert np.abs(got - ref).max() <= 1e-12 * np.abs(ref).max()
    for face in range(6):
        for fi in range(len(sc.freqs)):
            assert np.array_equal(box.face(face, fi), s.nf2ff_face(obox, face, fi, lo, hi))
    th, ph = np.deg2rad(np.arange(0, 181, 15.0)), np.deg2rad(np.arange(0, 361, 30.0))
    res = box.calc_nf2ff(list(sc.freqs), th, ph, degrees=False)
    L = [np.asarray(v, dtype=np.float64) for v in lines]
    for fi, fr in enumerate(sc.freqs):
        pts = np.concatenate([R.face_points(lo, hi, k, L, s.nf2ff_face(obox, k, fi, lo, hi)) for k in range(6)])
        ref = R.far_field(pts, fr, th, ph)
        scale = np.abs(ref["E_theta"]).max() + np.abs(ref["E_phi"]).max()
        assert np.abs(res.E_theta[fi] - ref["E_theta"]).max() <= 1e-10 * scale
        assert res.Dmax[fi] == pytest.approx(ref["Dmax"], rel=1e-9)


def test_scene_runner_small():
    r = run(ScatterScene(n=64, layers=6, steps=600))
    assert r["steps"] == 600 and r["mcells_per_s_device"] > 0
    assert all(np.isfinite(r["s11_db"])) and all(d > 1.0 for d in r["dmax"])
