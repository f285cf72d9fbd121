"""Independent numpy restatement of the uniaxial PML -- TEST INFRASTRUCTURE.

A second restatement, written separately from the C++ oracle's UPML, used
only to cross-check it.

Kind 0 follows the reference's Upml (src/extensions/pml.rs:222-655): six
regions without overlap (x slabs over the whole y-z extent, y slabs between
the x slabs, z slabs between both), each L + 1 cells deep; per cell and
component n the conductivities of all three components graded along the
region's own axis only (calculate_kappa, :370-420: depth from the region's
inner node, E at the node, H half a cell further out for n = the region's
axis and half a cell in otherwise), and

    vv = (2 eps0 - k[n''] dt) / den, vvfo = (2 eps0 - k[n] dt) / den,
    vvfn = (2 eps0 + k[n] dt) / den, den = 2 eps0 + k[n''] dt

(vv = vvfn = 1, vvfo = 0 where every k is 0), applied around the field
update as flux hooks: before it F <- flux, flux <- vv F - vvfo flux; after
it flux <- F, F <- flux_before + vvfn F.

Kind 1 is the corrected uniaxial PML this project uses (no counterpart in
the reference): in the same regions and hooks every cell is graded along
each axis whose active face holds it, at the Yee position of the component
(E_n half a cell up its own axis, H_n half a cell up the two others), with
the conductivity sigma_max (depth / L)^m of each face (sigma_max from that
face's own width), and the main update of a region cell advances D with the
next axis' conductivity: Ca = (2 eps0 - s[n'] dt) / (2 eps0 + s[n'] dt) and
Cb scaled by 2 eps0 / (2 eps0 + s[n'] dt) (likewise Da / Db with the H
positions), where the cell's coefficient pair is not zero.
"""
from __future__ import annotations

import math

import numpy as np

from .numpy_ref import _bwd, _fwd

EPS0 = 8.854_187_817e-12
Z0 = 376.730_313_668


def regions(ext, L):
    """(start, size, axis, is_min) of the six regions, in the reference's order."""
    nx, ny, nz = ext
    out = []
    if 0 < L[0] < nx:
        out.append(((0, 0, 0), (L[0] + 1, ny, nz), 0, True))
    if 0 < L[1] < nx:
        out.append(((nx - L[1] - 1, 0, 0), (L[1] + 1, ny, nz), 0, False))
    xs = L[0] + 1 if L[0] > 0 else 0
    xe = nx - L[1] - 1 if L[1] > 0 else nx
    if 0 < L[2] < ny and xs < xe:
        out.append(((xs, 0, 0), (xe - xs, L[2] + 1, nz), 1, True))
    if 0 < L[3] < ny and xs < xe:
        out.append(((xs, ny - L[3] - 1, 0), (xe - xs, L[3] + 1, nz), 1, False))
    ys = L[2] + 1 if L[2] > 0 else 0
    ye = ny - L[3] - 1 if L[3] > 0 else ny
    if 0 < L[4] < nz and xs < xe and ys < ye:
        out.append(((xs, ys, 0), (xe - xs, ye - ys, L[4] + 1), 2, True))
    if 0 < L[5] < nz and xs < xe and ys < ye:
        out.append(((xs, ys, nz - L[5] - 1), (xe - xs, ye - ys, L[5] + 1), 2, False))
    return out


def _kappa0(n, axis, p, is_min, layers, width, smax, m, ext, delta):
    """calculate_kappa: (k_v, k_i) of component n at index p along `axis`."""
    d = delta[axis]
    if is_min:
        depth = float(layers - p) * d if p <= layers else 0.0
    else:
        bs = ext[axis] - layers - 1
        depth = float(p - bs) * d if p >= bs else 0.0
    if depth <= 0.0:
        return 0.0, 0.0
    kv = smax * math.pow(depth / width, m)
    di = depth + (-0.5 if n == axis else 0.5) * d
    ki = smax * math.pow(min(1.0, max(0.0, di / width)), m)
    return kv, ki


def _sigma1(L, ext, delta, axis, i, half, m, R0):
    """Largest graded conductivity along `axis` at index i (+ 1/2 if half)
    over that axis' active faces."""
    sg = 0.0
    for side in range(2):
        l = L[2 * axis + side]
        if l <= 0 or l >= ext[axis]:
            continue
        smax = -(m + 1.0) * math.log(R0) / (2.0 * Z0 * float(l) * delta[axis])
        x = float(i) + (0.5 if half else 0.0)
        depth = float(l) - x if side == 0 else x - float(ext[axis] - l - 1)
        depth = min(float(l), max(0.0, depth))
        sg = max(sg, smax * math.pow(depth / float(l), m))
    return sg


def _trio(kn, knpp, dt):
    den = 2.0 * EPS0 + knpp * dt
    return (np.float32((2.0 * EPS0 - knpp * dt) / den), np.float32((2.0 * EPS0 - kn * dt) / den),
            np.float32((2.0 * EPS0 + kn * dt) / den))


def setup(coeffs12, ext, delta, dt, L, m=3.0, R0=1e-6, kind=0):
    """Regions with their per-cell (vv, vvfo, vvfn) for E and H, and the
    coefficients (kind 1 changes Ca / Cb / Da / Db in the regions)."""
    c = [np.array(x, dtype=np.float32) for x in coeffs12]
    regs = []
    for start, size, axis, is_min in regions(ext, L):
        layers = L[2 * axis + (0 if is_min else 1)]
        width = float(layers) * delta[axis]
        smax = -(m + 1.0) * math.log(R0) / (2.0 * Z0 * width)
        cv = np.zeros((3, 3) + tuple(size), np.float32)  # [vv|vvfo|vvfn][n]
        ci = np.zeros((3, 3) + tuple(size), np.float32)
        for li in range(size[0]):
            for lj in range(size[1]):
                for lk in range(size[2]):
                    pos = (start[0] + li, start[1] + lj, start[2] + lk)
                    if kind == 1:
                        for n in range(3):
                            sv = [_sigma1(L, ext, delta, a, pos[a], n == a, m, R0) for a in range(3)]
                            si = [_sigma1(L, ext, delta, a, pos[a], n != a, m, R0) for a in range(3)]
                            npr, npp = (n + 1) % 3, (n + 2) % 3
                            cv[:, n, li, lj, lk] = _trio(sv[n], sv[npp], dt)
                            ci[:, n, li, lj, lk] = _trio(si[n], si[npp], dt)
                            for (a_, b_, s) in ((0, 3, sv[npr]), (6, 9, si[npr])):
                                if c[a_ + n][pos] != 0 or c[b_ + n][pos] != 0:
                                    den = 2.0 * EPS0 + s * dt
                                    c[a_ + n][pos] = np.float32((2.0 * EPS0 - s * dt) / den)
                                    c[b_ + n][pos] = np.float32(float(c[b_ + n][pos]) * (2.0 * EPS0 / den))
                        continue
                    k = [_kappa0(n, axis, pos[axis], is_min, layers, width, smax, m, ext, delta) for n in range(3)]
                    kv, ki = [x[0] for x in k], [x[1] for x in k]
                    for n in range(3):
                        npp = (n + 2) % 3
                        cv[:, n, li, lj, lk] = _trio(kv[n], kv[npp], dt) if sum(kv) > 0.0 else (1.0, 0.0, 1.0)
                        ci[:, n, li, lj, lk] = _trio(ki[n], ki[npp], dt) if sum(ki) > 0.0 else (1.0, 0.0, 1.0)
        regs.append((tuple(slice(s, s + z) for s, z in zip(start, size)), cv, ci))
    return regs, c


def _hook_pre(fields, regs, which):
    for sl, cv, ci, fl in regs:
        co, flux = (cv, fl[0]) if which == "e" else (ci, fl[1])
        for n in range(3):
            f_old = fields[n][sl].copy()
            help_ = co[0, n] * f_old - co[1, n] * flux[n]
            fields[n][sl] = flux[n]
            flux[n] = help_


def _hook_post(fields, regs, which):
    for sl, cv, ci, fl in regs:
        co, flux = (cv, fl[0]) if which == "e" else (ci, fl[1])
        for n in range(3):
            help_ = flux[n].copy()
            new = fields[n][sl].copy()
            flux[n] = new
            fields[n][sl] = help_ + co[2, n] * new


def run(coeffs12, fields6, num_steps, dt, delta, L, m=3.0, R0=1e-6, kind=0, excitations=()):
    """Advance fields6 (float32) by num_steps with the UPML of layers L
    (-x +x -y +y -z +z); returns (fields, coefficients used)."""
    ext = np.asarray(fields6[0]).shape
    regs0, c = setup(coeffs12, ext, delta, dt, L, m, R0, kind)
    regs = [(sl, cv, ci, ([np.zeros(cv.shape[2:], np.float32) for _ in range(3)],
                          [np.zeros(cv.shape[2:], np.float32) for _ in range(3)])) for sl, cv, ci in regs0]
    ca, cb, da, db = c[0:3], c[3:6], c[6:9], c[9:12]
    E = [np.array(f, dtype=np.float32) for f in fields6[:3]]
    H = [np.array(f, dtype=np.float32) for f in fields6[3:]]
    inner = (slice(1, None),) * 3
    for step in range(num_steps):
        _hook_pre(H, regs, "h")
        ex, ey, ez = E
        H = [da[0] * H[0] + db[0] * (_fwd(ez, 1) - _fwd(ey, 2)),
             da[1] * H[1] + db[1] * (_fwd(ex, 2) - _fwd(ez, 0)),
             da[2] * H[2] + db[2] * (_fwd(ey, 0) - _fwd(ex, 1))]
        _hook_post(H, regs, "h")
        _hook_pre(E, regs, "e")
        hx, hy, hz = H
        ex, ey, ez = E
        nex = ca[0] * ex + cb[0] * (_bwd(hz, 1) - _bwd(hy, 2))
        ney = ca[1] * ey + cb[1] * (_bwd(hx, 2) - _bwd(hz, 0))
        nez = ca[2] * ez + cb[2] * (_bwd(hy, 0) - _bwd(hx, 1))
        ex[inner], ey[inner], ez[inner] = nex[inner], ney[inner], nez[inner]
        _hook_post(E, regs, "e")
        for pos, dr, soft, samples in excitations:
            if step >= len(samples):
                continue
            v = np.float32(samples[step])
            if soft:
                E[dr][tuple(pos)] += v
            else:
                E[dr][tuple(pos)] = v
    return np.stack(E + H), c
