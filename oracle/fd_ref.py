"""Independent numpy restatement of the frequency-domain field dump -- TEST INFRASTRUCTURE.

A second restatement of the oracle's field-DFT recording, used only to
cross-check it: FrequencyDomainFieldDump::accumulate
(src/processing/fields_fd.rs:149-217), X(f) += x(t) exp(-j 2 pi f t) 2 dt,
taken after the excitations of every step whose step count after the step
is a multiple of `interval` (scale 2 dt interval), E at t = n dt and H at
(n - 1/2) dt, over a half-open region with per-axis sub-sampling.  The
twiddle is cos / sin of -2 pi f t from the C library (Python's math module)
times the scale; real and imaginary parts accumulate as separate f64
products and sums.  The field update is numpy_ref's Yee step.
"""
from __future__ import annotations

import math

import numpy as np

from .numpy_ref import _bwd, _fwd


def run(coeffs12, fields6, num_steps, dt, dumps, excitations=(), t0=0):
    """dumps: [(region (i0, i1, j0, j1, k0, k1), sub_sample, comps, freqs,
    interval)]; returns (fields, per dump an array [freq][comp] of complex
    accumulators over the sub-sampled region, k fastest)."""
    c = [np.asarray(x, dtype=np.float32) for x in coeffs12]
    ca, cb, da, db = c[0:3], c[3:6], c[6:9], c[9:12]
    F = [np.array(f, dtype=np.float32) for f in fields6]
    sels, accs = [], []
    for region, ss, comps, freqs, interval in dumps:
        sels.append(tuple(slice(region[2 * a], region[2 * a + 1], ss[a]) for a in range(3)))
        shape = F[0][sels[-1]].shape
        accs.append([[(np.zeros(shape), np.zeros(shape)) for _ in comps] for _ in freqs])
    inner = (slice(1, None),) * 3
    t = t0
    for step in range(num_steps):
        ex, ey, ez, hx, hy, hz = F
        hx = da[0] * hx + db[0] * (_fwd(ez, 1) - _fwd(ey, 2))
        hy = da[1] * hy + db[1] * (_fwd(ex, 2) - _fwd(ez, 0))
        hz = da[2] * hz + db[2] * (_fwd(ey, 0) - _fwd(ex, 1))
        nex = ca[0] * ex + cb[0] * (_bwd(hz, 1) - _bwd(hy, 2))
        ney = ca[1] * ey + cb[1] * (_bwd(hx, 2) - _bwd(hz, 0))
        nez = ca[2] * ez + cb[2] * (_bwd(hy, 0) - _bwd(hx, 1))
        ex[inner], ey[inner], ez[inner] = nex[inner], ney[inner], nez[inner]
        F = [ex, ey, ez, hx, hy, hz]
        for pos, dr, soft, samples in excitations:
            if step >= len(samples):
                continue
            v = np.float32(samples[step])
            if soft:
                F[dr][tuple(pos)] += v
            else:
                F[dr][tuple(pos)] = v
        t += 1
        for (region, ss, comps, freqs, interval), sel, acc in zip(dumps, sels, accs):
            if t % interval:
                continue
            scale = 2.0 * dt * float(interval)
            for fi, f in enumerate(freqs):
                tw = []
                for tt in (float(t) * dt, (float(t) - 0.5) * dt):
                    ph = -2.0 * math.pi * f * tt
                    tw.append((math.cos(ph) * scale, math.sin(ph) * scale))
                for ci, comp in enumerate(comps):
                    wr, wi = tw[1 if comp >= 3 else 0]
                    x = F[comp][sel].astype(np.float64)
                    re, im = acc[fi][ci]
                    acc[fi][ci] = (re + x * wr, im + x * wi)
    out = [np.array([[re + 1j * im for re, im in row] for row in acc]) for acc in accs]
    return np.stack(F), out
