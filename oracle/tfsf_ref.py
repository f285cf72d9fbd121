"""Independent numpy restatement of the TF/SF plane source -- TEST INFRASTRUCTURE.

A second restatement, written separately from the C++ oracle's TF/SF, used
only to cross-check it.

Kind 0 follows the reference's TfsfBoundary (src/extensions/tfsf.rs:115-355):
E_axis / H_axis from the polarization (Transverse1: the next axis after the
propagation axis carries E, the one after it H; Transverse2 swaps them); a
1D line of n + 1 E and H values in f32.  Before every H update the line
steps (H[i] += db (E[i+1] - E[i]), H[0] = (A / eta) sin(2 pi f t), E[i] +=
cb (H[i] - H[i-1]), E[last] = k E[last-1] with k the Mur coefficient) and
the whole plane `pos` of H_axis gets H - db E_line[pos]; before every E
update the whole plane `pos` of E_axis gets E + cb H_line[pos], and t
advances.  db = -dt / (mu0 d), cb = dt / (eps0 d), both f32.

Kind 1 is the corrected source this project uses (no counterpart in the
reference): the line has a hard E source E[0] = A sin(2 pi f t), steps H
forward and E with the wave equation's sign (E[i] -= cb (H[i] - H[i-1])),
closes with first-order Mur (E[last] = E_old[last-1] + k (E[last-1] -
E_old[last])); the scattered-side H plane pos - 1 gets +- dt / (mu0 d)
E_line[pos] (+ for Transverse1) and the total-side E plane pos, without its
index-0 lines, gets + cb H_line[pos - 1].
"""
from __future__ import annotations

import math

import numpy as np

from .numpy_ref import _bwd, _fwd

EPS0 = 8.854_187_817e-12
MU0 = 1.256_637_062e-6
C0 = 299_792_458.0


def run(coeffs12, fields6, num_steps, dt, delta, direction, polarization, freq, amp, layer,
        vphase=0.0, kind=0, excitations=()):
    """Advance fields6 (float32) by num_steps with the TF/SF source."""
    c = [np.asarray(x, dtype=np.float32) for x in coeffs12]
    ca, cb3, da, db3 = c[0:3], c[3:6], c[6:9], c[9:12]
    E = [np.array(f, dtype=np.float32) for f in fields6[:3]]
    H = [np.array(f, dtype=np.float32) for f in fields6[3:]]
    ext = E[0].shape
    prop = direction // 2
    e_ax, h_ax = ((prop + 1) % 3, (prop + 2) % 3) if polarization == 0 else ((prop + 2) % 3, (prop + 1) % 3)
    d = delta[prop]
    v = vphase if vphase > 0.0 else C0
    n1 = ext[prop] + 1
    e1, h1 = np.zeros(n1, np.float32), np.zeros(n1, np.float32)
    db = np.float32(-(dt / (MU0 * d)))
    cb = np.float32(dt / (EPS0 * d))
    k = np.float32((v * dt - d) / (v * dt + d))
    eta = math.sqrt(MU0 / EPS0)
    t = 0

    def plane(a, p, first=0):
        idx = [slice(first, None)] * 3
        idx[prop] = p
        return a, tuple(idx)

    inner = (slice(1, None),) * 3
    h_inc_1 = np.float32(0)
    for step in range(num_steps):
        # before the H update
        if kind == 0:
            h1[:-1] = h1[:-1] + db * (e1[1:] - e1[:-1])
            h1[0] = np.float32((amp / eta) * math.sin(2.0 * math.pi * freq * (t * dt)))
            for i in range(1, n1):  # sequential: each E uses the new H
                e1[i] = e1[i] + cb * (h1[i] - h1[i - 1])
            e1[-1] = k * e1[-2]
            e_inc = e1[layer] if layer < n1 else np.float32(0)
            a, sl = plane(H[h_ax], layer)
            a[sl] = a[sl] - db * e_inc
        else:
            e1[0] = np.float32(amp * math.sin(2.0 * math.pi * freq * (t * dt)))
            e_inc = e1[layer]
            h1[:-1] = h1[:-1] + db * (e1[1:] - e1[:-1])
            h_inc_1 = h1[layer - 1]
            en1, en = e1[-2], e1[-1]
            e1[1:] = e1[1:] - cb * (h1[1:] - h1[:-1])
            e1[-1] = en1 + k * (e1[-2] - en)
            t += 1
            cc = np.float32(dt / (MU0 * d))
            a, sl = plane(H[h_ax], layer - 1)
            a[sl] = a[sl] + cc * e_inc if e_ax == (prop + 1) % 3 else a[sl] - cc * e_inc
        ex, ey, ez = E
        H = [da[0] * H[0] + db3[0] * (_fwd(ez, 1) - _fwd(ey, 2)),
             da[1] * H[1] + db3[1] * (_fwd(ex, 2) - _fwd(ez, 0)),
             da[2] * H[2] + db3[2] * (_fwd(ey, 0) - _fwd(ex, 1))]
        # before the E update
        if kind == 0:
            h_inc = h1[layer] if layer < n1 else np.float32(0)
            a, sl = plane(E[e_ax], layer)
            a[sl] = a[sl] + cb * h_inc
            t += 1
        else:
            a, sl = plane(E[e_ax], layer, first=1)
            a[sl] = a[sl] + cb * h_inc_1
        hx, hy, hz = H
        nex = ca[0] * ex + cb3[0] * (_bwd(hz, 1) - _bwd(hy, 2))
        ney = ca[1] * ey + cb3[1] * (_bwd(hx, 2) - _bwd(hz, 0))
        nez = ca[2] * ez + cb3[2] * (_bwd(hy, 0) - _bwd(hx, 1))
        ex[inner], ey[inner], ez[inner] = nex[inner], ney[inner], nez[inner]
        for pos, dr, soft, samples in excitations:
            if step >= len(samples):
                continue
            val = np.float32(samples[step])
            if soft:
                E[dr][tuple(pos)] += val
            else:
                E[dr][tuple(pos)] = val
    return np.stack(E + H)
