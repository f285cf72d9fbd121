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
