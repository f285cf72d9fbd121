"""Independent numpy restatement of the Mur boundary -- TEST INFRASTRUCTURE.

A second restatement, written separately from the C++ oracle's Mur faces,
used only to cross-check it.  First order follows MurAbc
(src/extensions/mur_abc.rs:60-151 set-up, :213-324 pre / post / apply):
before the E update a face keeps v = E_shift - k E_boundary for its two
tangential components, after it v += k E_shift(new), and then every face
writes v onto its boundary line, faces in order; k = (c dt - d) / (c dt + d).

Second order (no counterpart in the reference) is Mur's second-order
condition on the face interior:

    v = k E_b(n-1) - E_s(n-1) + c2 (E_b + E_s) + c3p (L_p E_b + L_p E_s)
        + c3q (L_q E_b + L_q E_s),  then v += k E_s(n+1)

with c2 = 2 d / (c dt + d), c3 = (c dt)^2 d / (2 h^2 (c dt + d)) per
tangential axis of spacing h, and L the three-point second difference
along that axis.  The face's first two and last two rows and columns keep
the first-order form.  At a min face the boundary is plane 1 (plane 0 is
never updated by the E loop), and plane 0 of a tangential axis whose min
face is also second-order Mur is left out of the face.  Every product and
sum is rounded on its own (float32), in the order written above.
"""
from __future__ import annotations

import numpy as np

from .numpy_ref import _bwd, _fwd

C0 = 299_792_458.0


class _Face:
    def __init__(self, f, ext, deltas, dt, order, enabled, vphase):
        self.ny = f // 2
        self.nyp, self.nypp = (self.ny + 1) % 3, (self.ny + 2) % 3
        n = ext[self.ny]
        is_max = f % 2 == 1
        off = 1 if (order == 2 and not is_max) else 0
        self.line = n - 1 if is_max else off
        self.shift = n - 2 if is_max else off + 1
        self.size = (ext[self.nyp], ext[self.nypp])
        lo0 = 1 if (order == 2 and enabled[2 * self.nyp]) else 0
        lo1 = 1 if (order == 2 and enabled[2 * self.nypp]) else 0
        p = np.arange(self.size[0])[:, None]
        q = np.arange(self.size[1])[None, :]
        self.live = (p >= lo0) & (q >= lo1)
        self.interior = (order == 2) & (p > lo0 + 1) & (p + 2 < self.size[0]) & (q > lo1 + 1) & (q + 2 < self.size[1])
        c = vphase if vphase > 0.0 else C0
        cdt, d = c * dt, deltas[self.ny]
        self.k = np.float32((cdt - d) / (cdt + d))
        self.c2 = np.float32(2.0 * d / (cdt + d))
        hp, hq = deltas[self.nyp], deltas[self.nypp]
        self.c3p = np.float32(cdt * cdt * d / (2.0 * hp * hp * (cdt + d)))
        self.c3q = np.float32(cdt * cdt * d / (2.0 * hq * hq * (cdt + d)))
        z = np.zeros(self.size, np.float32)
        self.v = [z.copy(), z.copy()]
        self.ob = [z.copy(), z.copy()]
        self.os = [z.copy(), z.copy()]

    def plane(self, a, line):
        """The (p, q) plane of array a at `line` along the normal axis (p
        along nyp, q along nypp)."""
        s = np.take(a, line, axis=self.ny)
        return s if self.nyp < self.nypp else s.T

    def set_plane(self, a, line, values, mask):
        idx = [slice(None)] * 3
        idx[self.ny] = line
        view = a[tuple(idx)]
        if self.nyp > self.nypp:
            view = view.T
        view[mask] = values[mask]


def _lap(w, axis):
    out = np.zeros_like(w)
    if axis == 0:
        out[1:-1, :] = (w[2:, :] + w[:-2, :]) - np.float32(2) * w[1:-1, :]
    else:
        out[:, 1:-1] = (w[:, 2:] + w[:, :-2]) - np.float32(2) * w[:, 1:-1]
    return out


def run(coeffs12, fields6, num_steps: int, dt: float, deltas, enabled=(1,) * 6, order: int = 1,
        vphase: float = 0.0, excitations=()):
    """Advance fields6 (Ex Ey Ez Hx Hy Hz, float32) by num_steps with Mur
    faces (-x +x -y +y -z +z enabled) of the given order."""
    c = [np.asarray(x, dtype=np.float32) for x in coeffs12]
    ca, cb, da, db = c[0:3], c[3:6], c[6:9], c[9:12]
    E = [np.array(f, dtype=np.float32) for f in fields6[:3]]
    hx, hy, hz = (np.array(f, dtype=np.float32) for f in fields6[3:])
    ext = E[0].shape
    faces = [_Face(f, ext, deltas, dt, order, enabled, vphase) for f in range(6) if enabled[f]]
    inner = (slice(1, None),) * 3
    for step in range(num_steps):
        ex, ey, ez = E
        hx = da[0] * hx + db[0] * (_fwd(ez, 1) - _fwd(ey, 2))
        hy = da[1] * hy + db[1] * (_fwd(ex, 2) - _fwd(ez, 0))
        hz = da[2] * hz + db[2] * (_fwd(ey, 0) - _fwd(ex, 1))
        for F in faces:  # before the E update
            for t, comp in enumerate((F.nyp, F.nypp)):
                wb, ws = F.plane(E[comp], F.line), F.plane(E[comp], F.shift)
                first = ws - F.k * wb
                if order == 2:
                    acc = F.k * F.ob[t] - F.os[t]
                    acc = acc + F.c2 * (wb + ws)
                    acc = acc + F.c3p * (_lap(wb, 0) + _lap(ws, 0))
                    acc = acc + F.c3q * (_lap(wb, 1) + _lap(ws, 1))
                    new = np.where(F.interior, acc, first)
                    F.ob[t] = np.where(F.live, wb, F.ob[t])
                    F.os[t] = np.where(F.live, ws, F.os[t])
                else:
                    new = first
                F.v[t] = np.where(F.live, new, F.v[t])
        nex = ca[0] * ex + cb[0] * (_bwd(hz, 1) - _bwd(hy, 2))
        ney = ca[1] * ey + cb[1] * (_bwd(hx, 2) - _bwd(hz, 0))
        nez = ca[2] * ez + cb[2] * (_bwd(hy, 0) - _bwd(hx, 1))
        ex[inner], ey[inner], ez[inner] = nex[inner], ney[inner], nez[inner]
        for F in faces:  # after it: every face's post, then every face's apply
            for t, comp in enumerate((F.nyp, F.nypp)):
                F.v[t] = np.where(F.live, F.v[t] + F.k * F.plane(E[comp], F.shift), F.v[t])
        for F in faces:
            for t, comp in enumerate((F.nyp, F.nypp)):
                F.set_plane(E[comp], F.line, F.v[t], F.live)
        for pos, dr, soft, samples in excitations:
            if step >= len(samples):
                continue
            v = np.float32(samples[step])
            if soft:
                E[dr][tuple(pos)] += v
            else:
                E[dr][tuple(pos)] = v
    return np.stack(E + [hx, hy, hz])
