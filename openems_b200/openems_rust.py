"""The reference's Python module surface (`openems_rust`, src/python/mod.rs)
on the B200 engine.

Same names, arguments and errors as the PyO3 module, so scripts written for
it (the reference's python/gpu_benchmark.py) run unchanged after
`from openems_b200 import openems_rust` (or with this module registered as
`openems_rust`):

    Grid.uniform / Grid.from_lines, num_cells(), cell_size()
    OpenEMS(num_timesteps=10000): gpu_available(), set_grid, set_engine_type,
        set_verbose, set_show_progress, set_gauss_excite(f0, fc),
        add_gauss_excite(f0, fc, direction=2, position=(0, 0, 0)),
        set_boundary_cond([6 strings]), set_end_criteria(db), run()
    SimulationStats(timesteps, wall_time, speed_mcells_per_sec, peak_energy,
        final_energy)
    C0, EPS0, MU0, Z0, VERSION

Differences: there is one engine, the CUDA one, so set_engine_type accepts
"gpu" / "gpu_v2" / "cuda" and refuses the reference's CPU engine names with
the reference's error type; set_boundary_cond also accepts "pml" / "pml_N" /
"3" (CPML) and "mur" / "2" (first-order Mur), which the reference refuses
(:198-231); PMC stays refused.  Excitations are the reference's:
Excitation::gaussian(f0, fc / f0) at the given cell, the grid centre for
(0, 0, 0) (:238-266); for f0 = 0, where the reference's relative bandwidth
divides by zero, the pulse takes its f0 -> 0 limit (f_max = fc / 2).
"""
from __future__ import annotations

import math
from dataclasses import dataclass
from typing import List, Optional, Sequence, Tuple

from . import _native as N
from . import constants as _c
from . import fdtd
from .xml_config import run_operator

C0, EPS0, MU0, Z0 = _c.C0, _c.EPS0, _c.MU0, _c.Z0
VERSION = "1.0.0"  # the reference crate's version (Cargo.toml), whose API this mirrors


class Grid:
    """Grid (src/python/mod.rs:21-55)."""

    def __init__(self, inner: fdtd.Grid):
        self.inner = inner

    @staticmethod
    def uniform(nx: int, ny: int, nz: int, delta: float) -> "Grid":
        return Grid(fdtd.Grid.uniform(nx, ny, nz, delta))

    @staticmethod
    def from_lines(x: Sequence[float], y: Sequence[float], z: Sequence[float]) -> "Grid":
        return Grid(fdtd.Grid.cartesian(list(x), list(y), list(z)))

    def num_cells(self) -> int:
        nx, ny, nz = self.inner.dimensions()
        return nx * ny * nz

    def cell_size(self) -> Tuple[float, float, float]:
        return self.inner.cell_size()


@dataclass
class SimulationStats:
    """SimulationStats (src/python/mod.rs:58-82)."""

    timesteps: int
    wall_time: float
    speed_mcells_per_sec: float
    peak_energy: float
    final_energy: float

    def __repr__(self):
        return (f"SimulationStats(timesteps={self.timesteps}, wall_time={self.wall_time:.3f}s, "
                f"speed={self.speed_mcells_per_sec:.2f} MC/s)")


@dataclass
class _Source:
    freq: float
    bandwidth: float
    direction: int
    position: Tuple[int, int, int]


class OpenEMS:
    """OpenEMS (src/python/mod.rs:95-290)."""

    def __init__(self, num_timesteps: int = 10000):
        self.grid: Optional[Grid] = None
        self.num_timesteps = int(num_timesteps)
        self.end_criteria_db: Optional[float] = None
        self.engine_type = "gpu"
        self.excitations: List[_Source] = []
        self.faces = [fdtd.BoundaryCondition.pec() for _ in range(6)]
        self.verbose = 1
        self.show_progress = True

    @staticmethod
    def gpu_available() -> bool:
        try:
            import torch
            return bool(torch.cuda.is_available())
        except ImportError:
            return False

    def set_grid(self, grid: Grid):
        self.grid = grid

    def set_engine_type(self, engine: str):
        e = engine.lower()
        if e in ("gpu", "gpu_v2", "cuda"):
            self.engine_type = e
            return
        if e in ("basic", "simd", "parallel"):
            raise RuntimeError(f"the {e} CPU engine is not part of this build; use 'gpu'")
        raise RuntimeError(f"Unknown engine type: {engine}. Use 'basic', 'simd', 'parallel', or 'gpu'")

    def set_verbose(self, level: int):
        self.verbose = int(level)

    def set_show_progress(self, show: bool):
        self.show_progress = bool(show)

    def set_gauss_excite(self, f0: float, fc: float):
        self.excitations = [_Source(f0, fc, 2, (0, 0, 0))]

    def add_gauss_excite(self, f0: float, fc: float, direction: int = 2, position=(0, 0, 0)):
        self.excitations.append(_Source(f0, fc, int(direction), tuple(int(v) for v in position)))

    def set_boundary_cond(self, bc: Sequence[str]):
        if len(bc) != 6:
            raise RuntimeError("Boundary conditions must be a list of 6 elements")
        faces = []
        for b in bc:
            t = str(b).lower()
            if t in ("pec", "0"):
                faces.append(fdtd.BoundaryCondition.pec())
            elif t in ("pmc", "1"):
                raise RuntimeError("PMC boundaries not yet supported")
            elif t in ("mur", "2"):
                faces.append(fdtd.BoundaryCondition("mur"))
            elif t in ("pml", "3") or t.startswith("pml_"):
                n = 8 if not t.startswith("pml_") else int(t[4:]) if t[4:].isdigit() else -1
                if n < 1:
                    raise RuntimeError(f"Unknown boundary condition: {b}")
                faces.append(fdtd.BoundaryCondition.pml(n))
            else:
                raise RuntimeError(f"Unknown boundary condition: {b}")
        self.faces = faces

    def set_end_criteria(self, db: float):
        self.end_criteria_db = float(db)

    def _excitation(self, src: _Source, dims) -> fdtd.Excitation:
        pos = src.position if src.position != (0, 0, 0) else (dims[0] // 2, dims[1] // 2, dims[2] // 2)
        if src.freq != 0:
            return fdtd.Excitation.gaussian(src.freq, src.bandwidth / src.freq, src.direction, pos)
        tau = 1.0 / (math.pi * 0.5 * src.bandwidth)
        return fdtd.Excitation.gaussian_pulse(tau, 4.0 * tau, src.direction, pos)

    def run(self) -> SimulationStats:
        if self.grid is None:
            raise RuntimeError("Grid not set. Call set_grid() first.")
        bcs = fdtd.BoundaryConditions.from_array(self.faces)
        op = fdtd.Operator(self.grid.inner, bcs)
        dims = op.dimensions()
        excs = [self._excitation(s, dims) for s in self.excitations]
        end_db = self.end_criteria_db
        cap = self.num_timesteps if end_db is None else 1_000_000  # src/fdtd/simulation.rs:225-229
        try:
            r = run_operator(op, excs, cap, end_db, tuple(f.kind == "mur" for f in self.faces))
        except N.OpenEMSError as e:
            raise RuntimeError(str(e)) from None
        return SimulationStats(int(r["timesteps"]), float(r["wall_s"]), float(r["mcells_per_s"]),
                               float(r["peak_energy"]), float(r["energy"]))
