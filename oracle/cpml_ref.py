"""Independent numpy restatement of the CPML update -- TEST INFRASTRUCTURE.

A second restatement, written separately from the C++ oracle's CPML, used
only to cross-check it.  It follows the reference's profile
(src/extensions/cpml.rs:68-72 for sigma_max, :98-155 for the grading, b and
a) with the two corrections this project applies to it:

- depths on the max face: E differences at l d and H differences at
  (l + 1/2) d into the layer, matching the min face's positions (the
  reference puts E a cell deeper than H there);
- the standard Roden-Gedney recursion psi <- b psi + c d with c = -a / kappa,
  and the stretched difference d / kappa + psi.

sigma_max uses the largest layer count and the smallest cell size over the
axes.  Scalar profile maths goes through Python's math module (the C
library's log, pow and exp, as the Rust and C++ code use).  The update is the
Yee step of numpy_ref.run (unfused float32 products and sums) with each
difference stretched in its own axis' slabs.  Small grids only.
"""
from __future__ import annotations

import math

import numpy as np

from .numpy_ref import _bwd, _fwd

EPS0 = 8.854_187_817e-12
Z0 = 376.730_313_668


def sigma_max(layers6, deltas, m: float, R: float) -> float:
    d = float(max(layers6)) * min(deltas)
    return -(m + 1.0) * math.log(R) / (2.0 * Z0 * d)


def profile(L: int, delta: float, dt: float, smax: float, m: float, alpha_max: float, kappa_max: float,
            is_min: bool) -> dict:
    """Per layer l (0 = the layer next to the grid's edge on the min face,
    the one next to the interior on the max face) the float32 b, c, 1/kappa
    at the E and at the H differences."""
    out = {k: np.zeros(L, np.float32) for k in ("b_e", "c_e", "ik_e", "b_h", "c_h", "ik_h")}
    width = float(L) * delta
    for l in range(L):
        de = float(L - l) * delta if is_min else float(l) * delta
        dh = de - 0.5 * delta if is_min else de + 0.5 * delta
        for depth, sfx in ((de, "e"), (dh, "h")):
            rho = min(1.0, max(0.0, depth / width))
            sigma = smax * math.pow(rho, m)
            alpha = alpha_max * (1.0 - rho)
            kappa = 1.0 + (kappa_max - 1.0) * math.pow(rho, m)
            b = math.exp(-(sigma / kappa / EPS0 + alpha / EPS0) * dt)
            sn = sigma / (EPS0 * kappa)
            an = alpha / EPS0
            den = sn + an
            a = sn / den * (1.0 - b) if abs(den) > 1e-20 else 0.0
            out["b_" + sfx][l] = np.float32(b)
            out["c_" + sfx][l] = np.float32(-a / kappa)
            out["ik_" + sfx][l] = np.float32(1.0 / kappa)
    return out


class _Axis:
    """Per index along one axis: in a slab or not, and its b, c, 1/kappa."""

    def __init__(self, ext, Lmin, Lmax, prof_min, prof_max, sfx):
        self.mask = np.zeros(ext, bool)
        self.b, self.c, self.ik = (np.zeros(ext, np.float32) for _ in range(3))
        for L, prof, g0 in ((Lmin, prof_min, 0), (Lmax, prof_max, ext - Lmax)):
            if prof is None:
                continue
            for l in range(L):
                g = g0 + l
                self.mask[g] = True
                self.b[g], self.c[g], self.ik[g] = prof["b_" + sfx][l], prof["c_" + sfx][l], prof["ik_" + sfx][l]

    def shaped(self, axis):
        s = [1, 1, 1]
        s[axis] = -1
        return tuple(v.reshape(s) for v in (self.mask, self.b, self.c, self.ik))


def _stretch(d, psi, ax: _Axis, axis: int):
    mask, b, c, ik = ax.shaped(axis)
    t1 = b * psi
    t2 = c * d
    p = t1 + t2
    t3 = d * ik
    dn = t3 + p
    return np.where(mask, dn, d), np.where(mask, p, psi)


def run(coeffs12, fields6, num_steps: int, dt: float, deltas, layers6, m: float = 3.0, R: float = 1e-6,
        alpha_max: float = 0.0, kappa_max: float = 1.0, excitations=()):
    """Advance fields6 (Ex Ey Ez Hx Hy Hz, float32) by num_steps with CPML
    slabs of layers6 (-x +x -y +y -z +z; a face is used when 0 < L < cells);
    returns (fields, profiles per face)."""
    c = [np.asarray(x, dtype=np.float32) for x in coeffs12]
    ca, cb, da, db = c[0:3], c[3:6], c[6:9], c[9:12]
    ex, ey, ez, hx, hy, hz = (np.array(f, dtype=np.float32) for f in fields6)
    ext = ex.shape
    smax = sigma_max(layers6, deltas, m, R)
    profs = [None] * 6
    for a in range(3):
        for s in range(2):
            L = int(layers6[2 * a + s])
            if 0 < L < ext[a]:
                profs[2 * a + s] = profile(L, deltas[a], dt, smax, m, alpha_max, kappa_max, s == 0)
    lay = [(int(layers6[2 * a]) if profs[2 * a] else 0, int(layers6[2 * a + 1]) if profs[2 * a + 1] else 0)
           for a in range(3)]
    axE = [_Axis(ext[a], lay[a][0], lay[a][1], profs[2 * a], profs[2 * a + 1], "e") for a in range(3)]
    axH = [_Axis(ext[a], lay[a][0], lay[a][1], profs[2 * a], profs[2 * a + 1], "h") for a in range(3)]
    psi_h = [np.zeros(ext, np.float32) for _ in range(6)]
    psi_e = [np.zeros(ext, np.float32) for _ in range(6)]
    inner = (slice(1, None),) * 3
    for step in range(num_steps):
        # H: each difference along axis a is stretched in the slabs of axis a
        d = [_fwd(ez, 1), _fwd(ey, 2), _fwd(ex, 2), _fwd(ez, 0), _fwd(ey, 0), _fwd(ex, 1)]
        for q, axis in enumerate((1, 2, 2, 0, 0, 1)):
            d[q], psi_h[q] = _stretch(d[q], psi_h[q], axH[axis], axis)
        hx = da[0] * hx + db[0] * (d[0] - d[1])
        hy = da[1] * hy + db[1] * (d[2] - d[3])
        hz = da[2] * hz + db[2] * (d[4] - d[5])
        d = [_bwd(hz, 1), _bwd(hy, 2), _bwd(hx, 2), _bwd(hz, 0), _bwd(hy, 0), _bwd(hx, 1)]
        for q, axis in enumerate((1, 2, 2, 0, 0, 1)):
            d[q], psi_e[q] = _stretch(d[q], psi_e[q], axE[axis], axis)
        nex = ca[0] * ex + cb[0] * (d[0] - d[1])
        ney = ca[1] * ey + cb[1] * (d[2] - d[3])
        nez = ca[2] * ez + cb[2] * (d[4] - d[5])
        ex[inner] = nex[inner]
        ey[inner] = ney[inner]
        ez[inner] = nez[inner]
        comps = (ex, ey, ez)
        for pos, dr, soft, samples in excitations:
            if step >= len(samples):
                continue
            v = np.float32(samples[step])
            if soft:
                comps[dr][tuple(pos)] += v
            else:
                comps[dr][tuple(pos)] = v
    return np.stack([ex, ey, ez, hx, hy, hz]), profs
