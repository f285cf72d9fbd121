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

It also restates the near-field to far-field recording box (no counterpart
in the reference engine; python/openEMS/nf2ff.py records the same
quantities): on each enabled face, at the face's plane p along its normal
a, the two tangential E components (b = a + 1, c = a + 2 mod 3) at p and
the two tangential H components averaged in f64 over the planes p - 1 and
p, with the same twiddles (E at n dt, H at (n - 1/2) dt).
"""
from __future__ import annotations

import math

import numpy as np

from .numpy_ref import _bwd, _fwd


def run(coeffs12, fields6, num_steps, dt, dumps, excitations=(), t0=0, boxes=()):
    """dumps: [(region (i0, i1, j0, j1, k0, k1), sub_sample, comps, freqs,
    interval)]; boxes: [(lo, hi, freqs, directions (6 flags), interval)].
    Returns (fields, per dump an array [freq][comp] of complex accumulators
    over the sub-sampled region, k fastest, per box {face: array [freq][4]
    of (nb, nc) complex accumulators Eb, Ec, Hb, Hc})."""
    c = [np.asarray(x, dtype=np.float32) for x in coeffs12]
    ca, cb, da, db = c[0:3], c[3:6], c[6:9], c[9:12]
    F = [np.array(f, dtype=np.float32) for f in fields6]
    sels, accs = [], []
    for region, ss, comps, freqs, interval in dumps:
        sels.append(tuple(slice(region[2 * a], region[2 * a + 1], ss[a]) for a in range(3)))
        shape = F[0][sels[-1]].shape
        accs.append([[(np.zeros(shape), np.zeros(shape)) for _ in comps] for _ in freqs])
    bacc = []
    for lo, hi, freqs, dirs, interval in boxes:
        faces = {}
        for face in range(6):
            if dirs[face]:
                a = face // 2
                b, c_ = (a + 1) % 3, (a + 2) % 3
                shape = (hi[b] - lo[b] + 1, hi[c_] - lo[c_] + 1)
                faces[face] = [[[np.zeros(shape), np.zeros(shape)] for _ in range(4)] for _ in freqs]
        bacc.append(faces)
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
        for (lo, hi, freqs, dirs, interval), faces in zip(boxes, bacc):
            if t % interval:
                continue
            scale = 2.0 * dt * float(interval)
            for face, acc in faces.items():
                a = face // 2
                b, c_ = (a + 1) % 3, (a + 2) % 3
                p = hi[a] if face & 1 else lo[a]
                sl = [slice(None)] * 3
                sl[b] = slice(lo[b], hi[b] + 1)
                sl[c_] = slice(lo[c_], hi[c_] + 1)
                at = list(sl)
                at[a] = p
                am = list(sl)
                am[a] = p - 1

                def plane(comp, where):
                    v = F[comp][tuple(where)].astype(np.float64)
                    return v if b < c_ else v.T  # (nb, nc) order

                vals = [plane(b, at), plane(c_, at),
                        0.5 * (plane(3 + b, am) + plane(3 + b, at)), 0.5 * (plane(3 + c_, am) + plane(3 + c_, at))]
                for fi, f in enumerate(freqs):
                    tw = []
                    for tt in (float(t) * dt, (float(t) - 0.5) * dt):
                        ph = -2.0 * math.pi * f * tt
                        tw.append((math.cos(ph) * scale, math.sin(ph) * scale))
                    for k in range(4):
                        wr, wi = tw[0 if k < 2 else 1]
                        acc[fi][k][0] = acc[fi][k][0] + vals[k] * wr
                        acc[fi][k][1] = acc[fi][k][1] + vals[k] * wi
    out = [np.array([[re + 1j * im for re, im in row] for row in acc]) for acc in accs]
    bout = [{face: np.array([[re + 1j * im for re, im in row] for row in acc]) for face, acc in faces.items()}
            for faces in bacc]
    return np.stack(F), out, bout


def probe_dft(trace, dt, freqs, half, t0=0):
    """Running DFT of a recorded probe trace (one value per step, the first
    after step t0 + 1): X(f) += x exp(-j 2 pi f t) 2 dt with t = (step count
    after the step - half) dt, half = 1/2 for a probe of H values only."""
    acc = np.zeros(len(freqs), np.complex128)
    re, im = np.zeros(len(freqs)), np.zeros(len(freqs))
    for s, x in enumerate(np.asarray(trace, np.float64)):
        t = (float(t0 + s + 1) - half) * dt
        for fi, f in enumerate(freqs):
            ph = -2.0 * math.pi * f * t
            re[fi] = re[fi] + x * (math.cos(ph) * (2.0 * dt))
            im[fi] = im[fi] + x * (math.sin(ph) * (2.0 * dt))
    acc.real, acc.imag = re, im
    return acc
