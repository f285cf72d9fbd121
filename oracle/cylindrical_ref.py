"""CPU restatement of the reference's cylindrical FDTD -- TEST INFRASTRUCTURE.

Follows src/fdtd/cylindrical.rs: the geometry of CylindricalGrid (:82-176),
the coefficients of CylindricalOperator::calculate_coefficients (:240-298),
update_voltage with its R = 0 fix-up (:422-521) and update_current
(:524-591).  Two forms: `step_loops` walks the cells in the reference's
order with numpy float32 scalars (every product and difference rounded to
f32 on its own, as the Rust code does); `step` is the same arithmetic
vectorised, for larger grids.  Only tests import this module.

Parity is unpinned beyond the reference's own tests for this module
(src/fdtd/cylindrical.rs:640-760): they check grid flags, alpha wrapping,
array sizes, step/time counters and reset, and hold no numeric fixtures;
the reference is Rust and cannot be built here to make some.  The tests also
hold impulse responses worked out by hand from the reference's update lines
(one H or E value of 1, every neighbour, alpha wrap, clamped edges, R = 0),
which this restatement reproduces exactly.
"""
from __future__ import annotations

import math

import numpy as np

EPS0 = 8.854_187_817e-12  # src/constants.rs:11
MU0 = 1.256_637_062e-6    # src/constants.rs:14


def coefficients(rho, alpha, z, dt):
    """(vi[3], iv[3]) as float32 (n_rho, n_alpha, n_z) arrays, cell by cell
    (:250-298 with get_node_area :117-143, get_edge_length :146-160)."""
    nr, na, nz = len(rho) - 1, len(alpha) - 1, len(z) - 1
    vi = [np.zeros((nr, na, nz), np.float32) for _ in range(3)]
    iv = [np.zeros((nr, na, nz), np.float32) for _ in range(3)]
    for i in range(nr):
        for j in range(na):
            for k in range(nz):
                dr, da, dz = rho[i + 1] - rho[i], alpha[j + 1] - alpha[j], z[k + 1] - z[k]
                r1, r2 = rho[i], rho[i + 1]
                areas = (r1 * da * dz, dr * dz, 0.5 * (r2 * r2 - r1 * r1) * da)
                lengths = (dr, r1 * da, dz)
                for c in range(3):
                    vi[c][i, j, k] = np.float32(dt / (EPS0 * areas[c])) if areas[c] > 0.0 else 0.0
                    iv[c][i, j, k] = np.float32(dt / (MU0 * lengths[c])) if lengths[c] > 0.0 else 0.0
    return vi, iv


def flags(rho, alpha):
    """(closed_alpha, r0_included) as CylindricalGrid::new (:36-58)."""
    return abs((alpha[-1] - alpha[0]) - 2.0 * math.pi) < 1e-6, abs(rho[0]) < 1e-10


def step_loops(e, h, vi, iv, closed, r0):
    """One step() in place, in the reference's loop order (small grids)."""
    f = np.float32
    nr, na, nz = e[0].shape
    er, ea, ez = e
    hr, ha, hz = h
    for i in range(nr):
        for j in range(na):
            for k in range(nz):
                jp = (na - 1 if closed else 0) if j == 0 else j - 1
                kp, ip = max(k - 1, 0), max(i - 1, 0)
                if i > 0 or not r0:
                    c = f(f(hz[i, j, k] - hz[i, jp, k]) - f(ha[i, j, k] - ha[i, j, kp]))
                else:
                    c = f(0.0)
                er[i, j, k] = f(f(1.0) * er[i, j, k]) + f(vi[0][i, j, k] * c)
                c = f(f(hr[i, j, k] - hr[i, j, kp]) - f(hz[i, j, k] - hz[ip, j, k]))
                ea[i, j, k] = f(f(1.0) * ea[i, j, k]) + f(vi[1][i, j, k] * c)
                if i > 0 or not r0:
                    c = f(f(ha[i, j, k] - ha[ip, j, k]) - f(hr[i, j, k] - hr[i, jp, k]))
                else:
                    c = f(0.0)
                ez[i, j, k] = f(f(1.0) * ez[i, j, k]) + f(vi[2][i, j, k] * c)
    if r0:
        for j in range(na):
            for k in range(nz):
                ea[0, j, k] = 0.0
                ez[0, j, k] = f(ez[1, j, k] * f(0.5))
    for i in range(nr):
        for j in range(na):
            for k in range(nz):
                jn = (0 if closed else na - 1) if j + 1 >= na else j + 1
                kn, i_n = min(k + 1, nz - 1), min(i + 1, nr - 1)
                c = f(f(ea[i, j, kn] - ea[i, j, k]) - f(ez[i, jn, k] - ez[i, j, k]))
                hr[i, j, k] = f(f(1.0) * hr[i, j, k]) + f(iv[0][i, j, k] * c)
                c = f(f(ez[i_n, j, k] - ez[i, j, k]) - f(er[i, j, kn] - er[i, j, k]))
                ha[i, j, k] = f(f(1.0) * ha[i, j, k]) + f(iv[1][i, j, k] * c)
                c = f(f(er[i, jn, k] - er[i, j, k]) - f(ea[i_n, j, k] - ea[i, j, k]))
                hz[i, j, k] = f(f(1.0) * hz[i, j, k]) + f(iv[2][i, j, k] * c)


def _prev(a, axis, wrap):
    """a[idx - 1] along axis; index 0 takes the last (wrap) or itself."""
    p = np.roll(a, 1, axis)
    if not wrap:
        s = [slice(None)] * 3
        s[axis] = slice(0, 1)
        p[tuple(s)] = a[tuple(s)]
    return p


def _next(a, axis, wrap):
    """a[idx + 1] along axis; the last index takes the first (wrap) or itself."""
    n = np.roll(a, -1, axis)
    if not wrap:
        s = [slice(None)] * 3
        s[axis] = slice(-1, None)
        n[tuple(s)] = a[tuple(s)]
    return n


def step(e, h, vi, iv, closed, r0, steps=1):
    """`steps` x step() in place, vectorised (same f32 arithmetic)."""
    er, ea, ez = e
    hr, ha, hz = h
    for _ in range(steps):
        c_r = (hz - _prev(hz, 1, closed)) - (ha - _prev(ha, 2, False))
        c_a = (hr - _prev(hr, 2, False)) - (hz - _prev(hz, 0, False))
        c_z = (ha - _prev(ha, 0, False)) - (hr - _prev(hr, 1, closed))
        if r0:
            c_r[0] = 0.0
            c_z[0] = 0.0
        er += vi[0] * c_r
        ea += vi[1] * c_a
        ez += vi[2] * c_z
        if r0:
            ea[0] = 0.0
            ez[0] = ez[1] * np.float32(0.5)
        c_r = (_next(ea, 2, False) - ea) - (_next(ez, 1, closed) - ez)
        c_a = (_next(ez, 0, False) - ez) - (_next(er, 2, False) - er)
        c_z = (_next(er, 1, closed) - er) - (_next(ea, 0, False) - ea)
        hr += iv[0] * c_r
        ha += iv[1] * c_a
        hz += iv[2] * c_z
