"""Independent numpy restatement of the reference Yee update -- TEST INFRASTRUCTURE.

A second oracle, written separately from ``oems_oracle.cpp``, used only to
cross-check it.  It follows src/fdtd/basic_engine.rs:191-306 (H over all
cells with zero forward differences at the max faces; E over i, j, k >= 1) and
:313-395 (soft ``+=`` / hard ``=`` after the E update).  numpy rounds every
elementwise product and sum separately, which is the same arithmetic as the
Rust code.  Small grids only: each step allocates temporaries.
"""
from __future__ import annotations

import numpy as np


def _fwd(a: np.ndarray, axis: int) -> np.ndarray:
    """a[idx+1] - a[idx] along axis, 0 at the last index."""
    d = np.zeros_like(a)
    sl_hi = [slice(None)] * 3
    sl_lo = [slice(None)] * 3
    sl_hi[axis] = slice(1, None)
    sl_lo[axis] = slice(0, -1)
    d[tuple(sl_lo)] = a[tuple(sl_hi)] - a[tuple(sl_lo)]
    return d


def _bwd(a: np.ndarray, axis: int) -> np.ndarray:
    """a[idx] - a[idx-1] along axis (garbage-free 0 at index 0, never used)."""
    d = np.zeros_like(a)
    sl_hi = [slice(None)] * 3
    sl_lo = [slice(None)] * 3
    sl_hi[axis] = slice(1, None)
    sl_lo[axis] = slice(0, -1)
    d[tuple(sl_hi)] = a[tuple(sl_hi)] - a[tuple(sl_lo)]
    return d


def run(coeffs12: np.ndarray, fields6: np.ndarray, num_steps: int, excitations=()) -> np.ndarray:
    """Advance ``fields6`` (Ex Ey Ez Hx Hy Hz) by ``num_steps``.

    ``excitations``: iterable of (pos (i,j,k), dir, soft, samples) with
    samples indexed by batch step.  Returns the new fields (float32).
    """
    c = [np.asarray(x, dtype=np.float32) for x in coeffs12]
    ca, cb, da, db = c[0:3], c[3:6], c[6:9], c[9:12]
    ex, ey, ez, hx, hy, hz = (np.array(f, dtype=np.float32) for f in fields6)
    for step in range(num_steps):
        dez_dy, dey_dz = _fwd(ez, 1), _fwd(ey, 2)
        dex_dz, dez_dx = _fwd(ex, 2), _fwd(ez, 0)
        dey_dx, dex_dy = _fwd(ey, 0), _fwd(ex, 1)
        hx = da[0] * hx + db[0] * (dez_dy - dey_dz)
        hy = da[1] * hy + db[1] * (dex_dz - dez_dx)
        hz = da[2] * hz + db[2] * (dey_dx - dex_dy)
        inner = (slice(1, None),) * 3
        cx = _bwd(hz, 1) - _bwd(hy, 2)
        cy = _bwd(hx, 2) - _bwd(hz, 0)
        cz = _bwd(hy, 0) - _bwd(hx, 1)
        nex = ca[0] * ex + cb[0] * cx
        ney = ca[1] * ey + cb[1] * cy
        nez = ca[2] * ez + cb[2] * cz
        ex[inner] = nex[inner]
        ey[inner] = ney[inner]
        ez[inner] = nez[inner]
        comps = (ex, ey, ez)
        for pos, d, soft, samples in excitations:
            if step >= len(samples):
                continue
            v = np.float32(samples[step])
            if soft:
                comps[d][tuple(pos)] += v
            else:
                comps[d][tuple(pos)] = v
    return np.stack([ex, ey, ez, hx, hy, hz])
