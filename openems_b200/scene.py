"""Dispersive scattering scene: every extension on one large grid.

A Drude sphere wrapped in a second-order Lorentz shell, next to a z-directed
wire dipole fed by a 50 ohm lumped port, in CPML, with an NF2FF recording box
inside the CPML and f64 port and surface DFTs.  At n = 384 (1 mm cells,
sphere radius 96, shell 8 cells, 20,000 steps) this is the large-grid
configuration; smaller n scale every length by n / 384.

    python -m openems_b200.scene [--n 384] [--steps 20000]

prints one JSON line: throughput, S11 and far-field directivity per
frequency.
"""
from __future__ import annotations

import argparse
import json
import time
from dataclasses import dataclass, field
from typing import Tuple

import numpy as np

from . import fdtd


@dataclass
class ScatterScene:
    n: int = 384
    delta: float = 1e-3
    layers: int = 8
    steps: int = 20000
    freqs: Tuple[float, ...] = (2e9, 3.5e9, 5e9)
    drude: Tuple[float, float] = (2 * np.pi * 5e9, 1e9)      # omega_p, gamma (rad/s)
    lorentz: Tuple[float, float, float, float] = (2 * np.pi * 4e9, 1e8, 3.0, 2.0)  # w0, gamma, d_eps, eps_inf
    nf2ff_interval: int = 10
    extra: dict = field(default_factory=dict)

    def scale(self, v: float) -> int:
        return max(1, int(round(v * self.n / 384)))

    @property
    def center(self) -> int:
        return self.n // 2

    @property
    def radius(self) -> int:
        return self.scale(96)

    @property
    def shell(self) -> int:
        return self.scale(8)

    @property
    def arm(self) -> int:
        return self.scale(20)

    @property
    def port(self) -> Tuple[int, int, int]:
        c = self.center
        return (c - self.radius - self.shell - self.scale(24), c, c)

    @property
    def box(self):
        lo = self.layers + self.scale(10)
        hi = self.n - 1 - lo
        return (lo,) * 3, (hi,) * 3

    def cells(self):
        """Drude sphere and Lorentz shell cells, (m, 3) each: cell centres
        within radius (shell: the next `shell` cells outward)."""
        c, r, t = self.center, self.radius, self.shell
        lo, hi = c - r - t - 1, c + r + t + 2
        g = np.arange(lo, hi)
        I, J, K = np.meshgrid(g, g, g, indexing="ij")
        d = np.sqrt((I + 0.5 - c) ** 2 + (J + 0.5 - c) ** 2 + (K + 0.5 - c) ** 2)
        pts = np.stack([I, J, K], -1)
        return pts[d <= r].astype(np.uint64), pts[(d > r) & (d <= r + t)].astype(np.uint64)

    def operator(self):
        """Operator with the shell's eps_inf, the dipole arms and the port
        resistor; returns (operator, port, sphere cells, shell cells)."""
        n = self.n
        op = fdtd.Operator(fdtd.Grid.uniform(n, n, n, self.delta), fdtd.BoundaryConditions.all_pec())
        sphere, shell = self.cells()
        op.set_material_cells(self.lorentz[3], 1.0, 0.0, 0.0, shell)
        px, py, pz = self.port
        op.set_pec((px, px + 1, py, py + 1, pz - self.arm, pz))
        op.set_pec((px, px + 1, py, py + 1, pz + 1, pz + 1 + self.arm))
        port = fdtd.LumpedPort(1, 50.0, self.port, 2, excite=1.0).apply(op)
        return op, port, sphere, shell

    def waveform(self) -> fdtd.Excitation:
        """Modulated Gaussian 1-6 GHz (centre 3.5 GHz)."""
        return fdtd.Excitation.gaussian_modulated(3.5e9, 2.5 / 3.5, 2, self.port)

    def attach(self, eng, port, sphere, shell):
        """CPML, dispersive materials, port probes / DFTs and the NF2FF box."""
        eng.add_cpml(fdtd.CpmlBoundaries.uniform(self.layers))
        wp, g = self.drude
        eng.add_dispersive(fdtd.DrudeMaterial(wp, g, second_order=True), sphere)
        w0, gl, de, ei = self.lorentz
        eng.add_dispersive(fdtd.LorentzMaterial(w0, gl, de, eps_inf=ei, second_order=True), shell)
        port.add_probes(eng, np.asarray(self.freqs))
        lo, hi = self.box
        return fdtd.Nf2ffBox(eng, lo, hi, list(self.freqs), interval=self.nf2ff_interval)


def run(scene: ScatterScene, batch: int = 1000, kernels: str = "auto"):
    t0 = time.perf_counter()
    op, port, sphere, shell = scene.operator()
    eng = fdtd.Engine(op, kernels=kernels)
    box = scene.attach(eng, port, sphere, shell)
    exc = port.excitation(scene.waveform())
    dt = op.timestep()
    t1 = time.perf_counter()
    dev = 0.0
    launches = 0
    start = 0
    while start < scene.steps:
        n = min(batch, scene.steps - start)
        eng.run_batch(fdtd.EngineBatch(num_steps=n, excitations=[
            fdtd.ScheduledExcitation.from_excitation(exc, start, n, dt)]))
        k, s = eng.last_batch_stats()
        dev += s
        launches += k
        start += n
    t2 = time.perf_counter()
    port.calc_port(eng)
    th = np.arange(0, 181, 5.0)
    ph = np.arange(0, 361, 10.0)
    c = scene.center * scene.delta
    ff = box.calc_nf2ff(list(scene.freqs), th, ph, center=(c, c, c))
    cells = scene.n ** 3
    return {
        "workload": f"scatter_{scene.n}: Drude sphere r={scene.radius}, Lorentz shell {scene.shell}, "
                    f"50 ohm port dipole, CPML {scene.layers}, NF2FF box, {scene.steps} steps",
        "cells": cells, "steps": scene.steps, "dispersive_cells": int(len(sphere) + len(shell)),
        "mcells_per_s_device": cells * scene.steps / dev / 1e6,
        "mcells_per_s_wall": cells * scene.steps / (t2 - t1) / 1e6,
        "setup_s": t1 - t0, "run_s": t2 - t1, "device_s": dev, "kernel_launches": launches,
        "launch_shape": eng.launch_info(),
        "freqs": list(scene.freqs),
        "s11_db": [float(20 * np.log10(abs(v))) for v in port.s11()],
        "dmax": [float(v) for v in ff.Dmax], "prad": [float(v) for v in ff.Prad],
        "p_acc": [float(v) for v in port.P_acc],
    }


def main(argv=None):
    p = argparse.ArgumentParser(description=__doc__.splitlines()[0])
    p.add_argument("--n", type=int, default=384)
    p.add_argument("--steps", type=int, default=20000)
    p.add_argument("--kernels", default="auto")
    a = p.parse_args(argv)
    print(json.dumps(run(ScatterScene(n=a.n, steps=a.steps), kernels=a.kernels)))


if __name__ == "__main__":
    main()
