"""Synthetic workloads of the benchmark configurations (seeded, no data files).

plain_pec_64   : 64^3, 1 mm, vacuum, PEC faces, soft Gaussian Ez at the centre
                 (tau = 1/(pi*20 GHz), t0 = 4 tau), 2000 steps, Ez/Hy probes at
                 4 cells.
cpml_boxes_256 : 256^3, 1 mm, 8-cell CPML on all faces (m = 3, R0 = 1e-6),
                 40 dielectric boxes from numpy default_rng(2) (sides U{4..40}
                 cells, placed inside the non-PML interior, eps_r ~ U[1, 10],
                 sigma ~ U[0, 0.1] S/m, applied in order), soft Gaussian Ez
                 0-10 GHz (tau = 1/(pi*10 GHz), t0 = 4 tau) at the centre,
                 10000 steps.
"""
from __future__ import annotations

from dataclasses import dataclass, field
from typing import List, Tuple

import numpy as np

from . import fdtd


@dataclass
class Workload:
    name: str
    dims: Tuple[int, int, int]
    delta: float
    num_steps: int
    cpml_layers: int = 0
    boxes: List[Tuple] = field(default_factory=list)  # (eps_r, mu_r, sigma_e, sigma_m, region6)
    tau: float = 0.0
    source: Tuple[int, int, int] = (0, 0, 0)
    source_dir: int = 2
    probes: List[Tuple[int, Tuple[int, int, int]]] = field(default_factory=list)

    @property
    def cells(self) -> int:
        return self.dims[0] * self.dims[1] * self.dims[2]

    def excitation(self) -> fdtd.Excitation:
        return fdtd.Excitation.gaussian_pulse(self.tau, 4.0 * self.tau, self.source_dir, self.source)

    def operator(self) -> fdtd.Operator:
        op = fdtd.Operator(fdtd.Grid.uniform(*self.dims, self.delta),
                           fdtd.BoundaryConditions.all_pec())
        for b in self.boxes:
            op.set_material(*b)
        return op

    def cpml(self):
        return fdtd.CpmlBoundaries.uniform(self.cpml_layers) if self.cpml_layers else None


def dielectric_boxes(n: int, layers: int, count: int = 40, seed: int = 2):
    rng = np.random.default_rng(seed)
    lo, hi = layers, n - layers
    boxes = []
    for _ in range(count):
        size = rng.integers(4, 41, size=3)
        start = [int(rng.integers(lo, hi - int(s) + 1)) for s in size]
        eps_r = float(rng.uniform(1.0, 10.0))
        sigma = float(rng.uniform(0.0, 0.1))
        region = (start[0], start[0] + int(size[0]), start[1], start[1] + int(size[1]),
                  start[2], start[2] + int(size[2]))
        boxes.append((eps_r, 1.0, sigma, 0.0, region))
    return boxes


def plain_pec_64() -> Workload:
    cells = [(16, 16, 16), (48, 16, 32), (32, 48, 16), (40, 40, 48)]
    return Workload("plain_pec_64", (64, 64, 64), 1e-3, 2000, 0, [],
                    1.0 / (np.pi * 20e9), (32, 32, 32), 2,
                    [(2, c) for c in cells] + [(4, c) for c in cells])


def cpml_boxes(n: int = 256, steps: int = 10000) -> Workload:
    return Workload(f"cpml_boxes_{n}", (n, n, n), 1e-3, steps, 8, dielectric_boxes(n, 8),
                    1.0 / (np.pi * 10e9), (n // 2, n // 2, n // 2), 2,
                    [(2, (n // 2, n // 2, n // 2)), (2, (n // 4, n // 2, n // 2))])


@dataclass
class PatchSpec:
    """One microstrip patch antenna of the sweep workload (cells of delta):
    PEC ground layer at k_ground and substrate cells [k_ground + 1, k_patch),
    both over the whole x-y extent (through the CPML),
    PEC patch layer k_patch over [x0, x0 + W) x [y0, y0 + L), a PEC feed wire
    from the port edge (Ez at (fx, fy, k_ground + 1)) up to the patch."""

    dims: Tuple[int, int, int]
    eps_r: float
    h_cells: int
    W: int
    L: int
    x0: int
    y0: int
    fx: int
    fy: int
    k_ground: int = 10
    layers: int = 8

    @property
    def k_patch(self) -> int:
        return self.k_ground + 1 + self.h_cells

    @property
    def cells(self) -> int:
        return self.dims[0] * self.dims[1] * self.dims[2]


def patch_specs(count: int = 64, seed: int = 4, layers: int = 8) -> List[PatchSpec]:
    """Seeded patch geometries: n_{x,y,z} ~ U{48..160}; substrate eps_r ~
    U[2.2, 10.2], thickness U[0.8, 3.2] mm = 2-6 cells of 0.5 mm; W, L ~
    U[8, 40] mm = 16-80 cells clipped to the interior; feed on the L axis at
    a seeded fraction U[0.2, 0.7] of L/2 from the centre."""
    rng = np.random.default_rng(seed)
    out = []
    for _ in range(count):
        dims = tuple(int(v) for v in rng.integers(48, 161, size=3))
        eps_r = float(rng.uniform(2.2, 10.2))
        h = int(np.clip(round(rng.uniform(0.8, 3.2) / 0.5), 2, 6))
        W = int(rng.integers(16, 81))
        L = int(rng.integers(16, 81))
        frac = float(rng.uniform(0.2, 0.7))
        margin = layers + 4
        W = max(4, min(W, dims[0] - 2 * margin))
        L = max(4, min(L, dims[1] - 2 * margin))
        x0 = (dims[0] - W) // 2
        y0 = (dims[1] - L) // 2
        fx = x0 + W // 2
        fy = y0 + L // 2 - int(round(frac * (L // 2)))
        out.append(PatchSpec(dims, eps_r, h, W, L, x0, y0, fx, fy, layers + 2, layers))
    return out


def patch_sweep_instance(spec: PatchSpec, delta: float = 0.5e-3, decay_db: float = 50.0,
                         max_steps: int = 60000, fmax: float = 8e9):
    """Operator, port and source of one patch (imported lazily: sweep.py
    depends on fdtd only)."""
    from .sweep import SweepInstance
    nx, ny, nz = spec.dims
    lo = spec.layers
    op = fdtd.Operator(fdtd.Grid.uniform(nx, ny, nz, delta), fdtd.BoundaryConditions.all_pec())
    kg, kp = spec.k_ground, spec.k_patch
    # ground plane and substrate run through the CPML to the domain edge, so
    # that substrate surface waves leave instead of ringing at a slab end
    op.set_material(spec.eps_r, 1.0, 0.0, 0.0, (0, nx, 0, ny, kg + 1, kp))
    op.set_pec((0, nx, 0, ny, kg, kg + 1))
    op.set_pec((spec.x0, spec.x0 + spec.W, spec.y0, spec.y0 + spec.L, kp, kp + 1))
    if kp > kg + 2:
        op.set_pec((spec.fx, spec.fx + 1, spec.fy, spec.fy + 1, kg + 2, kp))
    tau = 1.0 / (np.pi * fmax)
    wave = fdtd.Excitation.gaussian_pulse(tau, 4.0 * tau, 2, (spec.fx, spec.fy, kg + 1))
    return SweepInstance(op, (spec.fx, spec.fy, kg + 1), 2, wave, 50.0, spec.eps_r, 0.0,
                         fdtd.CpmlBoundaries.uniform(lo), decay_db, max_steps)
