"""The C++ oracle's frequency-domain field dumps against an independent
numpy restatement (oracle/fd_ref.py): accumulators bit for bit over a
driven run, with sub-sampling, an interval, E and H components (their
half-step time offset) and two batches."""
import numpy as np

import oracle
from oracle import fd_ref


def test_field_dft_restatements_agree_bitwise():
    dims = (11, 10, 12)
    lines = [oracle.uniform_lines(n, d) for n, d in zip(dims, (1.0e-3, 0.8e-3, 1.2e-3))]
    dt, delta = oracle.grid_timestep(*lines)
    s = oracle.OracleSim(*dims, dt, delta)
    s.set_material(3.0, 1.0, 0.0, 0.0, (3, 7, 2, 6, 4, 9))
    c12 = s.coefficients()
    steps = 80
    t = (np.arange(steps) - 15.0) / 5.0
    samples = np.exp(-t * t).astype(np.float32)
    exc = [((5, 5, 6), 2, True, samples)]
    dumps = [((1, 10, 0, 9, 2, 11), (2, 3, 1), [0, 2, 4], [3e9, 11e9, 17e9], 1),
             ((0, 11, 0, 10, 0, 12), (1, 1, 1), [1, 3, 5], [6e9], 3)]
    ids = [s.add_field_dft(r, f, sum(1 << c for c in comps), ss, iv) for r, ss, comps, f, iv in dumps]
    half = steps // 2
    s.add_excitation_sampled(*exc[0][:3], samples[:half])
    s.run_batch(half)
    s.clear_excitations()
    s.add_excitation_sampled(*exc[0][:3], samples[half:])
    s.run_batch(steps - half)
    zero = np.zeros((6,) + dims, np.float32)
    fields, acc, _ = fd_ref.run(c12, zero, steps, dt, dumps, exc)
    np.testing.assert_array_equal(fields, np.asarray(s.fields(), np.float32).reshape(fields.shape))
    for did, (region, ss, comps, freqs, iv), a in zip(ids, dumps, acc):
        for fi in range(len(freqs)):
            for ci, comp in enumerate(comps):
                got = s.field_dft(did, fi, comp)
                assert np.abs(got).max() > 0
                np.testing.assert_array_equal(got, a[fi, ci].reshape(-1))


def test_nf2ff_box_restatements_agree_bitwise():
    """All six faces of a recording box (E on the face, H averaged over the
    two half-cells), two frequencies, interval 2."""
    dims = (12, 11, 13)
    lines = [oracle.uniform_lines(n, d) for n, d in zip(dims, (1.0e-3, 0.8e-3, 1.2e-3))]
    dt, delta = oracle.grid_timestep(*lines)
    s = oracle.OracleSim(*dims, dt, delta)
    c12 = s.coefficients()
    steps = 70
    t = (np.arange(steps) - 15.0) / 5.0
    exc = [((6, 5, 6), 2, True, np.exp(-t * t).astype(np.float32)),
           ((5, 6, 7), 0, True, (0.3 * np.exp(-t * t)).astype(np.float32))]
    for pos, d, soft, smp in exc:
        s.add_excitation_sampled(pos, d, soft, smp)
    lo, hi, freqs, dirs = (2, 3, 2), (9, 8, 10), [4e9, 9e9], (1, 1, 1, 0, 1, 1)
    bid = s.add_nf2ff_box(lo, hi, freqs, dirs, 2)
    s.run_batch(steps)
    zero = np.zeros((6,) + dims, np.float32)
    _, _, boxes = fd_ref.run(c12, zero, steps, dt, [], exc, boxes=[(lo, hi, freqs, dirs, 2)])
    assert set(boxes[0]) == {0, 1, 2, 4, 5}
    for face, acc in boxes[0].items():
        for fi in range(len(freqs)):
            got = s.nf2ff_face(bid, face, fi, lo, hi)
            assert np.abs(got).max() > 0
            np.testing.assert_array_equal(got, acc[fi])


def test_probe_dft_restatements_agree_bitwise():
    """A voltage-style probe of E and a current-style probe of H only (half a
    step earlier), their running DFTs over two batches against the
    restatement on the recorded traces."""
    dims = (10, 9, 11)
    lines = [oracle.uniform_lines(n, d) for n, d in zip(dims, (1.0e-3, 0.8e-3, 1.2e-3))]
    dt, delta = oracle.grid_timestep(*lines)
    s = oracle.OracleSim(*dims, dt, delta)
    t = (np.arange(60) - 12.0) / 4.0
    samples = np.exp(-t * t).astype(np.float32)
    pe = s.add_probe([(2, (5, 4, k), -1.2e-3) for k in range(3, 8)], 1)
    ph = s.add_probe([(3, (4, 3, 5), 0.8e-3), (4, (4, 3, 5), -1.0e-3)], 1)
    freqs = [2e9, 7e9, 13e9]
    de, dh = s.add_probe_dft(pe, freqs), s.add_probe_dft(ph, freqs)
    traces = []
    for part in (samples[:25], samples[25:]):
        s.clear_excitations()
        s.add_excitation_sampled((5, 4, 5), 2, True, part)
        s.run_batch(len(part))
        traces.append(s.probe_traces())
    tr = np.concatenate(traces)
    for did, col, half in ((de, pe, 0.0), (dh, ph, 0.5)):
        want = fd_ref.probe_dft(tr[:, col], dt, freqs, half)
        assert np.abs(want).max() > 0
        np.testing.assert_array_equal(s.probe_dft(did), want)
