"""numpy restatement of the near-field to far-field transform -- TEST INFRASTRUCTURE.

The reference's `Nf2ff::calculate` (src/nf2ff/mod.rs:117-170) sets up the
observation frame and the far-field factor E = -j k eta / (4 pi) N but never
computes the radiation vectors (`integrate_surfaces`, :172-188, returns 0).
This module restates the surface-equivalence transform that factor belongs to
(Balanis, Antenna Theory, ch. 12; phasors exp(+j w t), matching the DFT sign
of src/processing/fields_fd.rs:163-167):

    J = n x H,  M = -n x E                      on the closed recording box
    N = sum J w exp(+j k r.r'),  L = sum M w exp(+j k r.r')
    E_theta = -j k exp(-j k R) / (4 pi R) (L_phi + eta N_theta)
    E_phi   = +j k exp(-j k R) / (4 pi R) (L_theta - eta N_phi)

and the result fields of python/openEMS/nf2ff.py:178-220 (P_rad = |E|^2 /
(2 eta) per angle, Prad = its integral over the requested angles, Dmax =
4 pi R^2 max P_rad / Prad).  Also: the face point list built from the
recorded box accumulators and the exact near fields of a Hertzian dipole
(Balanis eq. 4-8a..4-10c) as a known answer.

Only tests use this module.  A point list is an (n, 16) float64 array:
x y z w, J (re, im) x 3, M (re, im) x 3.
"""
from __future__ import annotations

import numpy as np

C0 = 299792458.0
Z0 = 376.730313668
PI = np.pi


def _dual(lines, lo, hi, j):
    """Half the span between the neighbouring nodes, clipped to [lo, hi]."""
    a = lines[max(j - 1, lo)]
    b = lines[min(j + 1, hi)]
    return 0.5 * (b - a)


def face_points(lo, hi, face, lines, acc):
    """Point list of one recorded face.

    acc: complex array (4, nb, nc) = Eb, Ec, Hb, Hc on the face's node grid
    (b = a+1, c = a+2 mod 3; Hb / Hc already averaged onto the face plane).
    Ec and Hb share the points (b node, c mid-cell); Eb and Hc share (b
    mid-cell, c node).  n = s e_a with s = -1 on min faces, +1 on max faces:
    J_c = s Hb, M_b = s Ec at the first set; J_b = -s Hc, M_c = -s Eb at the
    second.
    """
    a = face // 2
    b, c = (a + 1) % 3, (a + 2) % 3
    s = 1.0 if face & 1 else -1.0
    p = hi[a] if face & 1 else lo[a]
    lb, lc = lines[b], lines[c]
    pts = []
    for jb in range(lo[b], hi[b] + 1):          # Ec / Hb: b node, c cell
        for kc in range(lo[c], hi[c]):
            r = np.zeros(16)
            r[a] = lines[a][p]
            r[b] = lb[jb]
            r[c] = 0.5 * (lc[kc] + lc[kc + 1])
            r[3] = _dual(lb, lo[b], hi[b], jb) * (lc[kc + 1] - lc[kc])
            m = (jb - lo[b], kc - lo[c])
            jv, mv = s * acc[2][m], s * acc[1][m]
            r[4 + 2 * c], r[5 + 2 * c] = jv.real, jv.imag
            r[10 + 2 * b], r[11 + 2 * b] = mv.real, mv.imag
            pts.append(r)
    for jb in range(lo[b], hi[b]):              # Eb / Hc: b cell, c node
        for kc in range(lo[c], hi[c] + 1):
            r = np.zeros(16)
            r[a] = lines[a][p]
            r[b] = 0.5 * (lb[jb] + lb[jb + 1])
            r[c] = lc[kc]
            r[3] = (lb[jb + 1] - lb[jb]) * _dual(lc, lo[c], hi[c], kc)
            m = (jb - lo[b], kc - lo[c])
            jv, mv = -s * acc[3][m], -s * acc[0][m]
            r[4 + 2 * b], r[5 + 2 * b] = jv.real, jv.imag
            r[10 + 2 * c], r[11 + 2 * c] = mv.real, mv.imag
            pts.append(r)
    return np.array(pts).reshape(-1, 16)


def trapezoid_weights(x):
    x = np.asarray(x, dtype=np.float64)
    if len(x) < 2:
        return np.zeros(len(x))
    w = np.zeros(len(x))
    w[0] = 0.5 * (x[1] - x[0])
    w[-1] = 0.5 * (x[-1] - x[-2])
    w[1:-1] = 0.5 * (x[2:] - x[:-2])
    return w


def far_field(points, freq, theta, phi, radius=1.0, center=(0.0, 0.0, 0.0)):
    """Returns dict E_theta, E_phi (ntheta, nphi) complex, P_rad, Prad, Dmax."""
    theta = np.asarray(theta, dtype=np.float64)
    phi = np.asarray(phi, dtype=np.float64)
    k = 2.0 * PI * freq / C0
    pos = points[:, :3] - np.asarray(center)[None, :]
    w = points[:, 3]
    J = points[:, 4:10:2] + 1j * points[:, 5:10:2]
    M = points[:, 10:16:2] + 1j * points[:, 11:16:2]
    T, P = np.meshgrid(theta, phi, indexing="ij")
    st, ct, sp, cp = np.sin(T), np.cos(T), np.sin(P), np.cos(P)
    rhat = np.stack([st * cp, st * sp, ct], -1)
    thhat = np.stack([ct * cp, ct * sp, -st], -1)
    phhat = np.stack([-sp, cp, np.zeros_like(sp)], -1)
    ph = k * np.einsum("tpa,na->tpn", rhat, pos)
    e = w[None, None, :] * np.exp(1j * ph)
    N = np.einsum("tpn,na->tpa", e, J)
    L = np.einsum("tpn,na->tpa", e, M)
    Nt, Np = (N * thhat).sum(-1), (N * phhat).sum(-1)
    Lt, Lp = (L * thhat).sum(-1), (L * phhat).sum(-1)
    fac = 1j * k * np.exp(-1j * k * radius) / (4.0 * PI * radius)
    Et = -fac * (Lp + Z0 * Nt)
    Ep = fac * (Lt - Z0 * Np)
    Prad_a = (np.abs(Et) ** 2 + np.abs(Ep) ** 2) / (2.0 * Z0)
    wt, wp = trapezoid_weights(theta), trapezoid_weights(phi)
    Prad = float((Prad_a * radius ** 2 * np.sin(T) * wt[:, None] * wp[None, :]).sum())
    Dmax = 4.0 * PI * radius ** 2 * Prad_a.max() / Prad if Prad > 0 else 0.0
    return {"E_theta": Et, "E_phi": Ep, "P_rad": Prad_a, "Prad": Prad, "Dmax": Dmax}


def dipole_fields(pos, freq, il=1.0):
    """Exact E, H phasors of a z-directed Hertzian dipole I l at the origin
    (Balanis eq. 4-8a..4-10c) at points pos (n, 3); returns E, H (n, 3)."""
    k = 2.0 * PI * freq / C0
    x, y, z = pos[:, 0], pos[:, 1], pos[:, 2]
    r = np.sqrt(x * x + y * y + z * z)
    rho = np.sqrt(x * x + y * y)
    ct, st = z / r, rho / r
    cp = np.where(rho > 0, x / np.where(rho > 0, rho, 1), 1.0)
    sp = np.where(rho > 0, y / np.where(rho > 0, rho, 1), 0.0)
    g = np.exp(-1j * k * r)
    kr = k * r
    Er = Z0 * il * ct / (2 * PI * r ** 2) * (1 + 1 / (1j * kr)) * g
    Et = 1j * Z0 * k * il * st / (4 * PI * r) * (1 + 1 / (1j * kr) - 1 / kr ** 2) * g
    Hp = 1j * k * il * st / (4 * PI * r) * (1 + 1 / (1j * kr)) * g
    rhat = np.stack([st * cp, st * sp, ct], -1)
    thhat = np.stack([ct * cp, ct * sp, -st], -1)
    phhat = np.stack([-sp, cp, np.zeros_like(sp)], -1)
    E = Er[:, None] * rhat + Et[:, None] * thhat
    H = Hp[:, None] * phhat
    return E, H


def dipole_box_points(half, n, freq, il=1.0):
    """Point list on a cube [-half, half]^3 with n x n cells per face,
    J = n x H, M = -n x E of the exact dipole fields at cell centres."""
    edges = np.linspace(-half, half, n + 1)
    mid = 0.5 * (edges[1:] + edges[:-1])
    d = edges[1] - edges[0]
    out = []
    for a in range(3):
        b, c = (a + 1) % 3, (a + 2) % 3
        for s in (-1.0, 1.0):
            B, Cc = np.meshgrid(mid, mid, indexing="ij")
            pos = np.zeros((n * n, 3))
            pos[:, a] = s * half
            pos[:, b] = B.ravel()
            pos[:, c] = Cc.ravel()
            E, H = dipole_fields(pos, freq, il)
            nv = np.zeros(3)
            nv[a] = s
            J = np.cross(nv[None, :], H)
            M = -np.cross(nv[None, :], E)
            r = np.zeros((n * n, 16))
            r[:, :3] = pos
            r[:, 3] = d * d
            r[:, 4:10:2], r[:, 5:10:2] = J.real, J.imag
            r[:, 10:16:2], r[:, 11:16:2] = M.real, M.imag
            out.append(r)
    return np.concatenate(out)


def dipole_far_field(freq, theta, radius=1.0, il=1.0):
    """Analytic far-zone E_theta of the dipole (Balanis eq. 4-26a)."""
    k = 2.0 * PI * freq / C0
    return 1j * Z0 * k * il * np.sin(theta) * np.exp(-1j * k * radius) / (4 * PI * radius)
