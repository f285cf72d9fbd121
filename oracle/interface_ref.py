"""Scalar restatement of the reference's engine interface -- TEST INFRASTRUCTURE.

Follows `EngineInterface` and `EngineInterfaceMut`
(src/fdtd/engine_interface.rs:27-595) on host arrays, one query at a time,
with Python floats (IEEE f64, every operation rounded on its own, as Rust
evaluates it) and numpy float32 where the reference works in f32:

- snapping a position to a cell: `snap_to_grid` (:327-333) over
  `Grid::find_cell_x/y/z` (src/geometry/mod.rs:334-360, a linear scan of the
  mesh lines; a coordinate no line pair brackets goes to the last cell);
- `Grid::x_line` and `Grid::delta_x` (src/geometry/mod.rs:281-331);
- raw, node-interpolated and cell-interpolated E / H (:113-154, :380-504);
- D = eps E, B = mu H with a caller's material arrays or the vacuum
  constants (:165-199); curl H, also returned as J (:157-163, :201-206,
  :336-377);
- the voltage and current integrals (:208-305) and the energies
  (:308-324, `VectorField3D::energy`, src/arrays/field.rs:219-221, 314-316);
- the mutable interface's writes (:542-561).

Only tests use this module.  Fields are (3, nx, ny, nz) float32 arrays;
lines are three sequences of mesh lines in grid units.
"""
from __future__ import annotations

import numpy as np

EPS0 = 8.854_187_817e-12  # src/constants.rs:11
MU0 = 1.256_637_062e-6    # src/constants.rs:14

NO_INTERPOLATION, NODE_INTERPOLATE, CELL_INTERPOLATE = 0, 1, 2


class InterfaceRef:
    def __init__(self, e, h, lines, unit=1.0, dt=0.0, eps=None, mu=None, interp=NO_INTERPOLATION):
        self.e = np.asarray(e, dtype=np.float32)
        self.h = np.asarray(h, dtype=np.float32)
        self.lines = [np.asarray(v, dtype=np.float64) for v in lines]
        self.unit = float(unit)
        self.dt = float(dt)
        self.eps = None if eps is None else np.asarray(eps, dtype=np.float32)
        self.mu = None if mu is None else np.asarray(mu, dtype=np.float32)
        self.interp = interp
        self.dims = self.e.shape[1:]

    # ---- the grid (src/geometry/mod.rs) ----
    def find_cell(self, ax, x):
        l = self.lines[ax]
        xs = float(x) / self.unit
        for i in range(len(l) - 1):
            if xs >= l[i] and xs <= l[i + 1]:
                return i
        return max(len(l) - 2, 0)

    def line(self, ax, i):
        l = self.lines[ax]
        return (float(l[i]) if i < len(l) else 0.0) * self.unit

    def delta(self, ax, i):
        l = self.lines[ax]
        if i + 1 < len(l):
            return (float(l[i + 1]) - float(l[i])) * self.unit
        if i > 0:
            return (float(l[i]) - float(l[i - 1])) * self.unit
        return self.unit

    def snap(self, pos):
        return tuple(min(self.find_cell(ax, pos[ax]), self.dims[ax] - 1) for ax in range(3))

    # ---- field reads ----
    @staticmethod
    def _raw(f, i, j, k):
        return [float(f[c, i, j, k]) for c in range(3)]

    def get_e_field_raw(self, i, j, k):
        return self._raw(self.e, i, j, k)

    def get_h_field_raw(self, i, j, k):
        return self._raw(self.h, i, j, k)

    def _node(self, f, pos):
        i, j, k = self.snap(pos)
        fr = []
        for ax, c in enumerate((i, j, k)):
            v = (float(pos[ax]) - self.line(ax, c)) / self.delta(ax, c)
            fr.append(0.0 if v < 0.0 else (1.0 if v > 1.0 else v))
        fx, fy, fz = fr
        nx, ny, nz = self.dims
        i1, j1, k1 = min(i + 1, nx - 1), min(j + 1, ny - 1), min(k + 1, nz - 1)
        out = []
        for c in range(3):
            g = f[c]
            c000, c100 = float(g[i, j, k]), float(g[i1, j, k])
            c010, c110 = float(g[i, j1, k]), float(g[i1, j1, k])
            c001, c101 = float(g[i, j, k1]), float(g[i1, j, k1])
            c011, c111 = float(g[i, j1, k1]), float(g[i1, j1, k1])
            c00 = c000 * (1.0 - fx) + c100 * fx
            c01 = c001 * (1.0 - fx) + c101 * fx
            c10 = c010 * (1.0 - fx) + c110 * fx
            c11 = c011 * (1.0 - fx) + c111 * fx
            c0 = c00 * (1.0 - fy) + c10 * fy
            c1 = c01 * (1.0 - fy) + c11 * fy
            out.append(c0 * (1.0 - fz) + c1 * fz)
        return out

    def _cell(self, f, pos):
        c = self.snap(pos)
        shifted = [float(pos[ax]) + self.delta(ax, c[ax]) * 0.5 for ax in range(3)]
        return self._node(f, shifted)

    def _field(self, f, pos):
        if self.interp == NODE_INTERPOLATE:
            return self._node(f, pos)
        if self.interp == CELL_INTERPOLATE:
            return self._cell(f, pos)
        return self._raw(f, *self.snap(pos))

    def get_e_field(self, pos):
        return self._field(self.e, pos)

    def get_h_field(self, pos):
        return self._field(self.h, pos)

    def get_d_field(self, pos):
        e = self.get_e_field(pos)
        if self.eps is None:
            return [v * EPS0 for v in e]
        i, j, k = self.snap(pos)
        return [e[c] * float(self.eps[c, i, j, k]) for c in range(3)]

    def get_b_field(self, pos):
        h = self.get_h_field(pos)
        if self.mu is None:
            return [v * MU0 for v in h]
        i, j, k = self.snap(pos)
        return [h[c] * float(self.mu[c, i, j, k]) for c in range(3)]

    def _diff(self, comp, ax, i, j, k):
        c = [i, j, k]
        if c[ax] + 1 >= self.dims[ax]:
            return 0.0
        lo = self.h[comp][i, j, k]
        c[ax] += 1
        hi = self.h[comp][c[0], c[1], c[2]]
        return float(np.float32(hi) - np.float32(lo)) / self.delta(ax, (i, j, k)[ax])

    def curl_h(self, i, j, k):
        return [self._diff(2, 1, i, j, k) - self._diff(1, 2, i, j, k),
                self._diff(0, 2, i, j, k) - self._diff(2, 0, i, j, k),
                self._diff(1, 0, i, j, k) - self._diff(0, 1, i, j, k)]

    def get_rot_h_field(self, pos):
        return self.curl_h(*self.snap(pos))

    get_j_field = get_rot_h_field

    # ---- integrals and energies ----
    def calc_voltage_integral(self, start, stop):
        nx, ny, nz = self.dims
        i0, j0, k0 = self.snap(start)
        i1, j1, k1 = self.snap(stop)
        v = 0.0
        for i in range(min(i0, i1), max(i0, i1)):
            ic = min(i, nx - 1)
            v -= float(self.e[0, ic, j0, k0]) * self.delta(0, ic)
        for j in range(min(j0, j1), max(j0, j1)):
            jc = min(j, ny - 1)
            v -= float(self.e[1, i1, jc, k0]) * self.delta(1, jc)
        for k in range(min(k0, k1), max(k0, k1)):
            kc = min(k, nz - 1)
            v -= float(self.e[2, i1, j1, kc]) * self.delta(2, kc)
        return v

    def calc_current_integral(self, start, stop, normal_dir):
        nx, ny, nz = self.dims
        s = self.snap(start)
        t = self.snap(stop)
        r = [range(min(s[a], t[a]), max(s[a], t[a])) for a in range(3)]
        cur = 0.0
        h = self.h
        if normal_dir == 0:
            for j in r[1]:
                for k in r[2]:
                    jc, kc = min(j, ny - 1), min(k, nz - 1)
                    cur += float(h[1, s[0], jc, kc]) * self.delta(2, kc) - float(h[2, s[0], jc, kc]) * self.delta(1, jc)
        elif normal_dir == 1:
            for i in r[0]:
                for k in r[2]:
                    ic, kc = min(i, nx - 1), min(k, nz - 1)
                    cur += float(h[2, ic, s[1], kc]) * self.delta(0, ic) - float(h[0, ic, s[1], kc]) * self.delta(2, kc)
        else:
            for i in r[0]:
                for j in r[1]:
                    ic, jc = min(i, nx - 1), min(j, ny - 1)
                    cur += float(h[0, ic, jc, s[2]]) * self.delta(1, jc) - float(h[1, ic, jc, s[2]]) * self.delta(0, ic)
        return cur

    @staticmethod
    def _energy(f):
        v = f.astype(np.float64).ravel()
        return float(np.dot(v, v))

    def calc_e_energy(self):
        return 0.5 * EPS0 * self._energy(self.e)

    def calc_h_energy(self):
        return 0.5 * MU0 * self._energy(self.h)

    def calc_fast_energy(self):
        return 0.5 * (EPS0 * self._energy(self.e) + MU0 * self._energy(self.h))

    # ---- EngineInterfaceMut ----
    def set_e_field(self, i, j, k, value):
        self.e[:, i, j, k] = np.asarray(value, dtype=np.float32)

    def set_h_field(self, i, j, k, value):
        self.h[:, i, j, k] = np.asarray(value, dtype=np.float32)

    def add_e_field(self, i, j, k, value):
        for c in range(3):
            self.e[c, i, j, k] = np.float32(self.e[c, i, j, k]) + np.float32(value[c])


def snap_vec(lines, unit, dims, pos):
    """snap_to_grid for an (n, 3) array of positions, vectorised: on
    non-decreasing lines the scan's cell is the first line pair whose upper
    line is >= the coordinate (searchsorted), if its lower line is <= it;
    otherwise (below the first line, past the last, NaN) the last cell."""
    out = np.empty((len(pos), 3), np.int64)
    for ax in range(3):
        l = np.asarray(lines[ax], np.float64)
        x = np.asarray(pos[:, ax], np.float64) / unit
        if len(l) < 2:
            out[:, ax] = 0
            continue
        i = np.searchsorted(l[1:], x, side="left")  # first i with x <= l[i + 1]
        ok = (i < len(l) - 1) & (x >= l[np.minimum(i, len(l) - 2)])
        cell = np.where(ok, i, len(l) - 2)
        out[:, ax] = np.minimum(cell, dims[ax] - 1)
    return out


def node_vec(field3, lines, unit, dims, pos):
    """interpolate_*_field_to_node for an (n, 3) array of positions."""
    c = snap_vec(lines, unit, dims, pos)
    fr = []
    for ax in range(3):
        l = np.asarray(lines[ax], np.float64)
        i = c[:, ax]
        line = np.where(i < len(l), l[np.minimum(i, len(l) - 1)], 0.0) * unit
        hi = np.minimum(i + 1, len(l) - 1)
        d = np.where(i + 1 < len(l), (l[hi] - l[i]) * unit, np.where(i > 0, (l[i] - l[np.maximum(i - 1, 0)]) * unit, unit))
        f = (pos[:, ax] - line) / d
        fr.append(np.where(f < 0.0, 0.0, np.where(f > 1.0, 1.0, f)))
    fx, fy, fz = fr
    i, j, k = c[:, 0], c[:, 1], c[:, 2]
    i1, j1, k1 = (np.minimum(v + 1, dims[a] - 1) for a, v in enumerate((i, j, k)))
    out = np.empty((len(pos), 3))
    for comp in range(3):
        g = field3[comp].astype(np.float64)
        c00 = g[i, j, k] * (1.0 - fx) + g[i1, j, k] * fx
        c01 = g[i, j, k1] * (1.0 - fx) + g[i1, j, k1] * fx
        c10 = g[i, j1, k] * (1.0 - fx) + g[i1, j1, k] * fx
        c11 = g[i, j1, k1] * (1.0 - fx) + g[i1, j1, k1] * fx
        c0 = c00 * (1.0 - fy) + c10 * fy
        c1 = c01 * (1.0 - fy) + c11 * fy
        out[:, comp] = c0 * (1.0 - fz) + c1 * fz
    return out
