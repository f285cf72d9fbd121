"""Independent numpy restatement of dispersive media on a grid -- TEST INFRASTRUCTURE.

numpy_ref.dispersive_step restates the per-cell updates (Drude
src/extensions/dispersive.rs:510-535, Lorentz :171-196, Debye :604-630, and
this project's second-order polarisation recursions, kinds 3 and 4) on one
value at a time.  This module runs them on a grid, vectorised over each
material's cells, to pin the order around the field update: kinds 3 and 4
read E as it is before the E update (after the H update); every material
then updates its cells after the E update, materials in list order, then the
lumped RLC elements in list order, before the excitations.  Used only to
cross-check the C++ oracle.
"""
from __future__ import annotations

import numpy as np

from .numpy_ref import _bwd, _fwd, dispersive_coeffs, rlc_coeffs


def run(coeffs12, fields6, num_steps, dt, materials, excitations=(), rlc=(), deltas=(1.0, 1.0, 1.0)):
    """materials: [(kind, params, cells (n, 3), eps_inf)]; rlc: [(pos,
    direction, type, r, l, c)] elements (LumpedRlc::post_update_e,
    src/extensions/lumped_rlc.rs:263-286, after the media, in list order;
    coefficients with the cell size along the element); returns fields."""
    c = [np.asarray(x, dtype=np.float32) for x in coeffs12]
    ca, cb, da, db = c[0:3], c[3:6], c[6:9], c[9:12]
    F = [np.array(f, dtype=np.float32) for f in fields6]
    mats = []
    for kind, params, cells, eps_inf in materials:
        idx = tuple(np.asarray(cells, dtype=np.int64).T)
        n = len(cells)
        mats.append(dict(kind=kind, co=dispersive_coeffs(kind, params, dt, eps_inf), idx=idx,
                         j=np.zeros((3, n), np.float32), pp=np.zeros((3, n), np.float32),
                         ep=np.zeros((3, n), np.float32)))
    els = [dict(pos=tuple(pos), d=d, co=rlc_coeffs(t, r, l, cc, deltas[d], dt), i=np.float32(0))
           for pos, d, t, r, l, cc in rlc]
    inner = (slice(1, None),) * 3
    dtf = np.float32(dt)
    for step in range(num_steps):
        ex, ey, ez, hx, hy, hz = F
        hx = da[0] * hx + db[0] * (_fwd(ez, 1) - _fwd(ey, 2))
        hy = da[1] * hy + db[1] * (_fwd(ex, 2) - _fwd(ez, 0))
        hz = da[2] * hz + db[2] * (_fwd(ey, 0) - _fwd(ex, 1))
        E = [ex, ey, ez]
        for m in mats:
            if m["kind"] >= 3:
                for k in range(3):
                    m["ep"][k] = E[k][m["idx"]]
        nex = ca[0] * ex + cb[0] * (_bwd(hz, 1) - _bwd(hy, 2))
        ney = ca[1] * ey + cb[1] * (_bwd(hx, 2) - _bwd(hz, 0))
        nez = ca[2] * ez + cb[2] * (_bwd(hy, 0) - _bwd(hx, 1))
        ex[inner], ey[inner], ez[inner] = nex[inner], ney[inner], nez[inner]
        for m in mats:
            a, b, cc, c2 = m["co"]
            for k in range(3):
                e = E[k][m["idx"]]
                old = m["j"][k].copy()
                if m["kind"] == 0:
                    jn = a * old + b * e
                    m["j"][k] = jn
                    E[k][m["idx"]] = e - cc * jn
                elif m["kind"] == 1:
                    jn = a * old + cc * e
                    m["j"][k] = jn
                    E[k][m["idx"]] = e - b * jn
                elif m["kind"] == 2:
                    pn = a * old + b * e
                    m["j"][k] = pn
                    E[k][m["idx"]] = e - cc * ((pn - old) / dtf)
                else:
                    pn = (a * old + b * m["pp"][k]) + cc * m["ep"][k]
                    m["pp"][k] = old
                    m["j"][k] = pn
                    E[k][m["idx"]] = e - c2 * (pn - old)
        for el in els:
            v_vv, v_il = el["co"]
            e = E[el["d"]][el["pos"]]
            en = v_vv * e + v_il * el["i"]
            el["i"] = el["i"] + e * dtf
            E[el["d"]][el["pos"]] = en
        F = [ex, ey, ez, hx, hy, hz]
        for pos, dr, soft, samples in excitations:
            if step >= len(samples):
                continue
            v = np.float32(samples[step])
            if soft:
                F[dr][tuple(pos)] += v
            else:
                F[dr][tuple(pos)] = v
    return np.stack(F)
