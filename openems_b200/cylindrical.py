"""Cylindrical-coordinate FDTD (rho, alpha, z) on the CUDA engine.

Mirrors src/fdtd/cylindrical.rs: `CylindricalGrid` (:13-197) and
`CylindricalOperator` (:199-391) run on the host exactly as the reference's
(f64 geometry, coefficients rounded to f32 once), and `CylindricalEngine`
(:393-638) keeps E and H in device memory and steps them with the kernels of
csrc/cylindrical.cu (oems_cyl_*), bit-identical to the reference's f32
loops.  Arrays are (n_rho, n_alpha, n_z), z fastest.
"""
from __future__ import annotations

import argparse
import ctypes
import json
import math
from typing import Optional, Sequence, Tuple

import numpy as np

from . import _native as N
from .constants import C0, EPS0, MU0

CLOSED_ALPHA_THRESHOLD = 1e-6  # src/fdtd/cylindrical.rs:11


class CylindricalGrid:
    """CylindricalGrid (src/fdtd/cylindrical.rs:13-197)."""

    def __init__(self, rho: Sequence[float], alpha: Sequence[float], z: Sequence[float]):
        self.rho = [float(v) for v in rho]
        self.alpha = [float(v) for v in alpha]
        self.z = [float(v) for v in z]
        self.n_rho = max(len(self.rho) - 1, 0)
        self.n_alpha = max(len(self.alpha) - 1, 0)
        self.n_z = max(len(self.z) - 1, 0)
        span = (self.alpha[-1] if self.alpha else 0.0) - (self.alpha[0] if self.alpha else 0.0)
        self.closed_alpha = abs(span - 2.0 * math.pi) < CLOSED_ALPHA_THRESHOLD
        self.r0_included = bool(self.rho) and abs(self.rho[0]) < 1e-10

    @classmethod
    def uniform(cls, r_min: float, r_max: float, n_rho: int, n_alpha: int, z_min: float, z_max: float,
                n_z: int) -> "CylindricalGrid":
        """:61-79: alpha always spans 0..2 pi."""
        dr = (r_max - r_min) / n_rho
        da = 2.0 * math.pi / n_alpha
        dz = (z_max - z_min) / n_z
        return cls([r_min + i * dr for i in range(n_rho + 1)], [i * da for i in range(n_alpha + 1)],
                   [z_min + i * dz for i in range(n_z + 1)])

    def get_cell_size(self, i: int, j: int, k: int) -> Tuple[float, float, float]:
        """:82-105: forward differences, backward at the last line, alpha
        wrapping around on a closed mesh."""
        r, a, z = self.rho, self.alpha, self.z
        d_rho = r[i + 1] - r[i] if i + 1 < len(r) else r[i] - r[i - 1]
        if j + 1 < len(a):
            d_alpha = a[j + 1] - a[j]
        elif self.closed_alpha:
            d_alpha = 2.0 * math.pi - a[j] + a[0]
        else:
            d_alpha = a[j] - a[j - 1]
        d_z = z[k + 1] - z[k] if k + 1 < len(z) else z[k] - z[k - 1]
        return d_rho, d_alpha, d_z

    def get_radius(self, i: int) -> float:
        return self.rho[i] if i < len(self.rho) else (self.rho[-1] if self.rho else 0.0)

    def get_node_area(self, ny: int, pos) -> float:
        """:117-143."""
        i, j, k = pos
        cs = self.get_cell_size(i, j, k)
        if ny == 0:
            return self.get_radius(i) * cs[1] * cs[2]
        if ny == 1:
            return cs[0] * cs[2]
        if ny == 2:
            r1 = self.get_radius(i)
            r2 = self.rho[i + 1] if i + 1 < len(self.rho) else r1
            return 0.5 * (r2 * r2 - r1 * r1) * cs[1]
        return 0.0

    def get_edge_length(self, ny: int, pos) -> float:
        """:146-160."""
        i, j, k = pos
        cs = self.get_cell_size(i, j, k)
        if ny == 0:
            return cs[0]
        if ny == 1:
            return self.get_radius(i) * cs[1]
        if ny == 2:
            return cs[2]
        return 0.0

    def get_cell_volume(self, pos) -> float:
        """:163-176."""
        i, j, k = pos
        cs = self.get_cell_size(i, j, k)
        r1 = self.get_radius(i)
        r2 = self.rho[i + 1] if i + 1 < len(self.rho) else r1 + cs[0]
        return 0.5 * (r2 * r2 - r1 * r1) * cs[1] * cs[2]

    def map_alpha_index(self, idx: int) -> int:
        """:179-187."""
        if not self.closed_alpha:
            return max(int(idx), 0)
        n = self.n_alpha
        return ((int(idx) % n) + n) % n

    def dimensions(self) -> Tuple[int, int, int]:
        return self.n_rho, self.n_alpha, self.n_z

    def _sizes(self):
        """Per-line cell sizes as f64 vectors (every in-range index takes the
        forward difference in get_cell_size)."""
        r, a, z = (np.asarray(v, dtype=np.float64) for v in (self.rho, self.alpha, self.z))
        return r, np.diff(r), np.diff(a), np.diff(z)


class CylindricalOperator:
    """CylindricalOperator (src/fdtd/cylindrical.rs:199-391): vv = ii = 1,
    vi = f32(dt / (eps0 area)), iv = f32(dt / (mu0 length)), 0 where the
    area or length is not positive."""

    def __init__(self, grid: CylindricalGrid, dt: float):
        self._grid = grid
        self._dt = float(dt)
        nr, na, nz = grid.dimensions()
        r, dr, da, dz = grid._sizes()
        shape = (nr, na, nz)
        R = np.broadcast_to(r[:nr, None, None], shape)
        R2 = np.broadcast_to(r[1:nr + 1, None, None], shape)
        DR = np.broadcast_to(dr[:, None, None], shape)
        DA = np.broadcast_to(da[None, :, None], shape)
        DZ = np.broadcast_to(dz[None, None, :], shape)
        # the reference's f64 expressions, same operand order (:117-160)
        areas = (R * DA * DZ, DR * DZ, 0.5 * (R2 * R2 - R * R) * DA)
        lengths = (DR, R * DA, DZ)
        with np.errstate(divide="ignore", invalid="ignore"):
            self._vi = tuple(np.where(A > 0.0, self._dt / (EPS0 * A), 0.0).astype(np.float32) for A in areas)
            self._iv = tuple(np.where(L > 0.0, self._dt / (MU0 * L), 0.0).astype(np.float32) for L in lengths)
        ones = np.ones(shape, dtype=np.float32)
        self._vv = (ones, ones, ones)
        self._ii = (ones, ones, ones)
        # :307-332 -- computed by the reference but not read by its update
        self.vv_r0 = self.vi_r0 = None
        if grid.r0_included:
            a0 = 0.5 * dr[0] * da[:, None] * dz[None, :]
            with np.errstate(divide="ignore"):
                self.vi_r0 = np.where(a0 > 0.0, self._dt / (EPS0 * a0), 0.0).astype(np.float32).ravel()
            self.vv_r0 = np.ones(na * nz, dtype=np.float32)

    def grid(self) -> CylindricalGrid:
        return self._grid

    def dt(self) -> float:
        return self._dt

    def vv(self):
        return self._vv

    def vi(self):
        return self._vi

    def ii(self):
        return self._ii

    def iv(self):
        return self._iv

    def calculate_timestep(self) -> float:
        """:345-370: the smallest per-cell Courant step, times 0.95; the
        alpha step at radius max(r, d_rho / 2)."""
        g = self._grid
        nr, na, nz = g.dimensions()
        if nr * na * nz == 0:
            return math.inf
        r, dr, da, dz = g._sizes()
        rr = np.maximum(r[:nr], dr * 0.5)[:, None, None]
        dx = dr[:, None, None]
        dy = rr * da[None, :, None]
        dzz = dz[None, None, :]
        dt_cell = 1.0 / (C0 * np.sqrt(1.0 / (dx * dx) + 1.0 / (dy * dy) + 1.0 / (dzz * dzz)))
        return float(dt_cell.min()) * 0.95


class CylindricalEngine:
    """CylindricalEngine (src/fdtd/cylindrical.rs:393-638) on the GPU."""

    def __init__(self, operator: CylindricalOperator, device: Optional[int] = None):
        self.operator = operator
        g = operator.grid()
        self._shape = g.dimensions()
        self._n = int(np.prod(self._shape))
        vi = [np.ascontiguousarray(a, dtype=np.float32) for a in operator.vi()]
        iv = [np.ascontiguousarray(a, dtype=np.float32) for a in operator.iv()]
        d = N.CylDescC()
        d.n_rho, d.n_alpha, d.n_z = self._shape
        d.closed_alpha = int(g.closed_alpha)
        d.r0_included = int(g.r0_included)
        d.dt = operator.dt()
        for c in range(3):
            d.vi[c] = N.fptr(vi[c])
            d.iv[c] = N.fptr(iv[c])
        d.device = -1 if device is None else int(device)
        h = ctypes.c_void_p()
        N.check(N.lib().oems_cyl_create(ctypes.byref(d), ctypes.byref(h)))
        self._h = h

    def close(self):
        if getattr(self, "_h", None):
            N.lib().oems_cyl_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def step(self, steps: int = 1):
        """`steps` x step(): update_voltage (with the R = 0 fix-up), then
        update_current."""
        N.check(N.lib().oems_cyl_step(self._h, int(steps)))

    def last_step_ms(self) -> float:
        """Device time of the last step() call (CUDA events on the engine's
        stream, all its steps)."""
        ms = ctypes.c_float()
        N.check(N.lib().oems_cyl_last_step_ms(self._h, ctypes.byref(ms)))
        return float(ms.value)

    def timestep(self) -> int:
        t, s = ctypes.c_uint64(), ctypes.c_double()
        N.check(N.lib().oems_cyl_time(self._h, ctypes.byref(t), ctypes.byref(s)))
        return int(t.value)

    def time(self) -> float:
        t, s = ctypes.c_uint64(), ctypes.c_double()
        N.check(N.lib().oems_cyl_time(self._h, ctypes.byref(t), ctypes.byref(s)))
        return float(s.value)

    def read_fields(self):
        """(E, H): three (n_rho, n_alpha, n_z) float32 arrays each."""
        e = [np.empty(self._shape, dtype=np.float32) for _ in range(3)]
        h = [np.empty(self._shape, dtype=np.float32) for _ in range(3)]
        N.check(N.lib().oems_cyl_read_fields(self._h, (N.PF * 3)(*map(N.fptr, e)), (N.PF * 3)(*map(N.fptr, h))))
        return tuple(e), tuple(h)

    def e_field(self):
        return self.read_fields()[0]

    def h_field(self):
        return self.read_fields()[1]

    def write_fields(self, e=None, h=None):
        """Replace E and/or H (the reference's e_field_mut / h_field_mut)."""
        ce, ch = self.read_fields() if e is None or h is None else (None, None)
        e = ce if e is None else e
        h = ch if h is None else h
        e = [np.ascontiguousarray(np.broadcast_to(a, self._shape), dtype=np.float32) for a in e]
        h = [np.ascontiguousarray(np.broadcast_to(a, self._shape), dtype=np.float32) for a in h]
        N.check(N.lib().oems_cyl_write_fields(self._h, (N.PF * 3)(*map(N.fptr, e)), (N.PF * 3)(*map(N.fptr, h))))

    def reset(self):
        N.check(N.lib().oems_cyl_reset(self._h))


# Algorithmic bytes per cell and step: each pass reads E, H and one coefficient
# triple and writes one field triple (neighbour reads hit in cache).
BYTES_PER_CELL_STEP = 2 * 12 * 4


def main(argv=None):
    """Throughput of the engine on a uniform closed mesh (fields seeded with
    noise, a hundredth of the reference's timestep so they stay finite):
    `python -m openems_b200.cylindrical --n-rho 256 --n-alpha 256 --n-z 256`."""
    ap = argparse.ArgumentParser(description=main.__doc__)
    ap.add_argument("--n-rho", type=int, default=256)
    ap.add_argument("--n-alpha", type=int, default=256)
    ap.add_argument("--n-z", type=int, default=256)
    ap.add_argument("--r0", action="store_true", help="mesh through R = 0")
    ap.add_argument("--steps", type=int, default=500)
    ap.add_argument("--warmup", type=int, default=20)
    ap.add_argument("--repeats", type=int, default=3)
    a = ap.parse_args(argv)
    g = CylindricalGrid.uniform(0.0 if a.r0 else 0.005, 0.05, a.n_rho, a.n_alpha, 0.0, 0.05, a.n_z)
    op = CylindricalOperator(g, CylindricalOperator(g, 1.0).calculate_timestep() * 0.01)
    rng = np.random.default_rng(1)
    shape = g.dimensions()
    with CylindricalEngine(op) as eng:
        eng.write_fields([rng.standard_normal(shape, dtype=np.float32) for _ in range(3)],
                         [np.zeros(shape, np.float32)] * 3)
        eng.step(a.warmup)
        ms = []
        for _ in range(a.repeats):
            eng.step(a.steps)
            ms.append(eng.last_step_ms())
        e, _h = eng.read_fields()
        finite = all(bool(np.isfinite(c).all()) for c in e)
    cells = int(np.prod(shape))
    best = min(ms)
    out = {"workload": f"cylindrical {a.n_rho}x{a.n_alpha}x{a.n_z}{' through R=0' if a.r0 else ''}, "
                       f"{a.steps} steps", "cells": cells, "ms": ms,
           "mcells_per_s": cells * a.steps / (best * 1e-3) / 1e6,
           "gb_per_s": cells * a.steps * BYTES_PER_CELL_STEP / (best * 1e-3) / 1e9,
           "bytes_per_cell_step": BYTES_PER_CELL_STEP, "fields_finite": finite}
    print(json.dumps(out))


if __name__ == "__main__":
    main()
