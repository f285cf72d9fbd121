"""The oracle's two loop forms give identical bits.

The cell loop restates the reference's parallel engine
(src/fdtd/parallel_engine.rs:108-172, the same arithmetic as
src/fdtd/basic_engine.rs:191-306); the z-line form restates its SIMD engine
(src/fdtd/simd_engine.rs:252-391) with the CPML stretch applied to the row
buffers.  The z-line form is the faster CPU baseline and the one the
full-size GPU parity tests run, so it must not differ in a single bit.
"""
import numpy as np
import pytest

import oracle


def _sim(dims, zline, precision=32, cpml=None, threads=3, mur=False):
    lines = [oracle.uniform_lines(n, 1e-3) for n in dims]
    dt, d3 = oracle.grid_timestep(*lines)
    s = oracle.OracleSim(*dims, dt, d3, precision=precision, threads=threads, zline=zline)
    rng = np.random.default_rng(7)
    for _ in range(4):
        lo = [int(rng.integers(0, n - 3)) for n in dims]
        hi = [lo[a] + int(rng.integers(2, max(3, dims[a] - lo[a]))) for a in range(3)]
        s.set_material(float(rng.uniform(1, 8)), float(rng.uniform(1, 2)), float(rng.uniform(0, 0.2)),
                       float(rng.uniform(0, 50.0)), (lo[0], hi[0], lo[1], hi[1], lo[2], hi[2]))
    s.set_pec((2, 4, 1, dims[1] - 1, 3, 5))
    if cpml is not None:
        s.enable_cpml(cpml)
    if mur:
        s.enable_mur(order=2)
    tau = 1.0 / (np.pi * 40e9)
    c = tuple(n // 2 for n in dims)
    s.add_excitation_analytic(c, 2, True, 0, [tau, 4 * tau], 1.0, 0, 400)
    s.add_excitation_analytic((c[0] - 2, c[1] + 1, c[2] - 3), 0, True, 0, [tau, 4 * tau], 0.5, 0, 400)
    s.add_point_probe(2, c)
    s.add_point_probe(4, (1, 2, 3))
    return s


@pytest.mark.parametrize("dims,cpml,precision", [
    ((17, 13, 11), None, 32),
    ((21, 17, 23), (3, 4, 0, 5, 2, 6), 32),
    ((19, 24, 9), (5, 5, 4, 4, 3, 3), 32),
    ((14, 12, 18), (2, 3, 4, 2, 5, 1), 64),
])
def test_zline_equals_cell_loop(dims, cpml, precision):
    a = _sim(dims, False, precision, cpml)
    b = _sim(dims, True, precision, cpml)
    ra = a.run_batch(90, sample_interval=10, track_peak=True)
    rb = b.run_batch(90, sample_interval=10, track_peak=True)
    fa, fb = a.fields(), b.fields()
    assert np.abs(fa).max() > 0
    assert np.array_equal(fa, fb)
    assert np.array_equal(a.probe_traces(), b.probe_traces())
    assert ra["energy_samples"] == rb["energy_samples"]


def test_zline_with_mur_and_thread_counts():
    a = _sim((16, 15, 13), False, mur=True, threads=1)
    b = _sim((16, 15, 13), True, mur=True, threads=4)
    a.run_batch(70)
    b.run_batch(70)
    assert np.array_equal(a.fields(), b.fields())
