"""openEMS XML configuration files: parse, build the simulation, run it.

The reference reads an openEMS XML file in `parse_config`
(src/io/xml.rs:12-46): the FDTD element's NumberOfTimesteps, endCriteria,
f0 and fc (:95-143) and the BoundaryCond face codes (:146-183, mapped by
`boundary_from_code` :212-221: 0 PEC, 1 PMC, 2 Mur, 3 PML with 8 layers,
4 periodic); its geometry parser is a placeholder (:185-210) and the grid is
never read, so its command line (src/main.rs:118-142) always runs a default
20^3 grid without sources.  `parse_config` here returns the same fields with
the same defaults and, beyond them, what the openEMS format carries for a
run: the RectilinearGrid lines (times DeltaUnit), the FDTD element's
Excitation (Type 0 Gaussian with centre f0 and cutoff fc: tau = 1 / (pi fc),
a pulse without carrier for f0 = 0, else modulated at f0; 1 sinusoidal f0;
2 Dirac; 3 step),
face codes also written as "PEC" / "PMC" / "MUR" / "PML_n", and the
ContinuousStructure's Material, Metal and Excitation properties with their
Box primitives (applied in ascending Priority).

Mapping of boxes to the grid (cells i lie between lines i and i + 1): a
Material covers the cells whose centres lie inside the box; a Metal and an
Excitation snap each corner to the nearest line and cover the cells from the
lower line index up to the upper one (at least one cell per axis, so a zero-
thickness sheet is one cell thick); a Metal sets PEC there, an Excitation
puts a soft source of its Excite vector's components on every covered cell.

`run` builds the Operator (with CPML on PML faces and Mur on Mur faces) and
runs the engine in batches to NumberOfTimesteps or, with endCriteria, until
the energy has fallen by -10 log10(endCriteria) dB below its peak (openEMS
writes endCriteria as an energy ratio, e.g. 1e-5 = -50 dB; the reference
passes the raw number as a dB value, src/main.rs:130).
"""
from __future__ import annotations

import math
import xml.etree.ElementTree as ET
from dataclasses import dataclass, field
from typing import List, Optional, Sequence, Tuple

import numpy as np

from . import _native as N
from . import fdtd

FACE_NAMES = ("xmin", "xmax", "ymin", "ymax", "zmin", "zmax")


@dataclass
class GridConfig:
    x_lines: List[float]
    y_lines: List[float]
    z_lines: List[float]
    unit: float = 1.0


@dataclass
class BoxProperty:
    """A Material (eps_r, mu_r, kappa = sigma_e, sigma_m), Metal or
    Excitation property with its boxes ((p1, p2, priority), in drawing
    units)."""

    kind: str
    name: str
    boxes: List[Tuple[Tuple[float, float, float], Tuple[float, float, float], int]] = field(default_factory=list)
    eps_r: float = 1.0
    mu_r: float = 1.0
    sigma_e: float = 0.0
    sigma_m: float = 0.0
    excite: Tuple[float, float, float] = (0.0, 0.0, 0.0)


@dataclass
class SimulationConfig:
    """SimulationConfig (src/io/xml.rs:49-66) plus the run-relevant parts of
    the openEMS format."""

    num_timesteps: int = 0
    end_criteria: Optional[float] = None
    excitation_type: int = 0
    f0: float = 0.0
    fc: float = 0.0
    boundaries: List[int] = field(default_factory=lambda: [0] * 6)
    pml_layers: List[int] = field(default_factory=lambda: [8] * 6)
    grid: Optional[GridConfig] = None
    properties: List[BoxProperty] = field(default_factory=list)

    @property
    def end_criteria_db(self) -> Optional[float]:
        """endCriteria as a decay in dB (an energy ratio r gives -10 log10 r)."""
        if self.end_criteria is None or not self.end_criteria > 0:
            return None
        return -10.0 * math.log10(self.end_criteria) if self.end_criteria < 1 else self.end_criteria


def _num(text, default, kind=float):
    try:
        return kind(text)
    except (TypeError, ValueError):
        return default


def _face_code(text) -> Tuple[int, Optional[int]]:
    """Face code and PML layers: numbers as the reference, or openEMS names."""
    if text is None:
        return 0, None
    t = text.strip().upper()
    if t.startswith("PML"):
        n = _num(t[4:], 8, int) if t.startswith("PML_") else 8
        return 3, n
    named = {"PEC": 0, "PMC": 1, "MUR": 2, "PERIODIC": 4}
    if t in named:
        return named[t], None
    try:
        return int(t), None
    except ValueError:
        return 0, None  # the reference's parse::<i32>().unwrap_or(0)


def _lines(el) -> List[float]:
    if el is None or not (el.text or "").strip():
        return []
    return sorted(float(v) for v in el.text.replace(";", ",").split(",") if v.strip())


def _point(el) -> Tuple[float, float, float]:
    return tuple(_num(el.get(a), 0.0) for a in ("X", "Y", "Z"))


def parse_config(source) -> SimulationConfig:
    """Parses an openEMS XML file (path) or XML text."""
    text = source if isinstance(source, str) and source.lstrip().startswith("<") else open(source).read()
    try:
        root = ET.fromstring(text)
    except ET.ParseError as e:
        raise N.ConfigError(f"XML parse error: {e}") from None
    cfg = SimulationConfig()
    fd = root.find("FDTD") if root.tag != "FDTD" else root
    if fd is not None:
        # an integer, else 10000 as the reference's parse().unwrap_or(10000)
        cfg.num_timesteps = _num(fd.get("NumberOfTimesteps"), 10000, int) \
            if fd.get("NumberOfTimesteps") is not None else 0
        cfg.end_criteria = _num(fd.get("endCriteria"), None)
        cfg.f0 = _num(fd.get("f0"), 0.0)
        cfg.fc = _num(fd.get("fc"), 0.0)
        exc = fd.find("Excitation")
        if exc is not None:
            cfg.excitation_type = _num(exc.get("Type"), 0, int)
            cfg.f0 = _num(exc.get("f0"), cfg.f0)
            cfg.fc = _num(exc.get("fc"), cfg.fc)
        bc = fd.find("BoundaryCond")
        if bc is not None:
            for f, name in enumerate(FACE_NAMES):
                code, layers = _face_code(bc.get(name))
                cfg.boundaries[f] = code
                if layers is not None:
                    cfg.pml_layers[f] = layers
    cs = root.find("ContinuousStructure")
    if cs is not None:
        rg = cs.find("RectilinearGrid")
        if rg is not None:
            cfg.grid = GridConfig(_lines(rg.find("XLines")), _lines(rg.find("YLines")), _lines(rg.find("ZLines")),
                                  _num(rg.get("DeltaUnit"), 1.0))
        props = cs.find("Properties")
        for p in (props if props is not None else []):
            kind = p.tag
            if kind not in ("Material", "Metal", "Excitation"):
                continue
            bp = BoxProperty(kind, p.get("Name", ""))
            pr = p.find("Property")
            if kind == "Material" and pr is not None:
                bp.eps_r = _num(pr.get("Epsilon"), 1.0)
                bp.mu_r = _num(pr.get("Mue"), 1.0)
                bp.sigma_e = _num(pr.get("Kappa"), 0.0)
                bp.sigma_m = _num(pr.get("Sigma"), 0.0)
            if kind == "Excitation":
                ex = [_num(v, 0.0) for v in (p.get("Excite") or "0,0,0").split(",")]
                bp.excite = tuple((ex + [0.0, 0.0, 0.0])[:3])
            prims = p.find("Primitives")
            for b in (prims.findall("Box") if prims is not None else []):
                p1, p2 = b.find("P1"), b.find("P2")
                if p1 is None or p2 is None:
                    continue
                bp.boxes.append((_point(p1), _point(p2), _num(b.get("Priority"), 0, int)))
            cfg.properties.append(bp)
    return cfg


def boundary_from_code(code: int, layers: int = 8) -> fdtd.BoundaryCondition:
    """boundary_from_code (src/io/xml.rs:212-221); unknown codes are PEC."""
    kind = {0: "pec", 1: "pmc", 2: "mur", 3: "pml", 4: "periodic"}.get(code, "pec")
    return fdtd.BoundaryCondition(kind, layers if kind == "pml" else 0)


def _cell_range_centres(lines: np.ndarray, a: float, b: float) -> Tuple[int, int]:
    lo, hi = min(a, b), max(a, b)
    c = 0.5 * (lines[1:] + lines[:-1])
    idx = np.nonzero((c >= lo) & (c <= hi))[0]
    return (int(idx[0]), int(idx[-1]) + 1) if len(idx) else (0, 0)


def _cell_range_snap(lines: np.ndarray, a: float, b: float) -> Tuple[int, int]:
    i0 = int(np.argmin(np.abs(lines - min(a, b))))
    i1 = int(np.argmin(np.abs(lines - max(a, b))))
    n = len(lines) - 1
    i0 = min(i0, n - 1)
    return i0, min(max(i1, i0 + 1), n)


@dataclass
class Built:
    operator: fdtd.Operator
    boundaries: fdtd.BoundaryConditions
    sources: List[Tuple[Tuple[int, int, int], int, float]]  # (cell, component, weight)
    mur_faces: Tuple[bool, ...]


def build(cfg: SimulationConfig) -> Built:
    """Operator with the materials and metals, the soft-source cells and the
    boundary set-up of a parsed configuration."""
    if cfg.grid is None or min(len(cfg.grid.x_lines), len(cfg.grid.y_lines), len(cfg.grid.z_lines)) < 2:
        # the reference's command line falls back to this grid (src/main.rs:118-128)
        grid = fdtd.Grid.uniform(20, 20, 20, 1e-3)
        lines = [np.arange(21) * 1e-3] * 3
    else:
        lines = [np.asarray(v, dtype=np.float64) * cfg.grid.unit
                 for v in (cfg.grid.x_lines, cfg.grid.y_lines, cfg.grid.z_lines)]
        grid = fdtd.Grid.cartesian(*lines)
    bcs = fdtd.BoundaryConditions.from_array([boundary_from_code(c, n) for c, n in
                                              zip(cfg.boundaries, cfg.pml_layers)])
    op = fdtd.Operator(grid, bcs)
    unit = cfg.grid.unit if cfg.grid is not None else 1.0
    sources = []
    items = [(b[2], k, p, b) for k, p in enumerate(cfg.properties) for b in p.boxes]
    for _, _, p, (p1, p2, _) in sorted(items, key=lambda t: (t[0], t[1])):
        if p.kind == "Material":
            r = [_cell_range_centres(lines[a], p1[a] * unit, p2[a] * unit) for a in range(3)]
            if all(hi > lo for lo, hi in r):
                op.set_material(p.eps_r, p.mu_r, p.sigma_e, p.sigma_m, tuple(v for lo_hi in r for v in lo_hi))
        else:
            r = [_cell_range_snap(lines[a], p1[a] * unit, p2[a] * unit) for a in range(3)]
            if p.kind == "Metal":
                op.set_pec(tuple(v for lo_hi in r for v in lo_hi))
            else:
                for comp in range(3):
                    if p.excite[comp] == 0.0:
                        continue
                    for i in range(*r[0]):
                        for j in range(*r[1]):
                            for k in range(*r[2]):
                                sources.append(((i, j, k), comp, float(p.excite[comp])))
    mur = tuple(c == 2 for c in cfg.boundaries)
    return Built(op, bcs, sources, mur)


def waveform(cfg: SimulationConfig, position, component, weight) -> fdtd.Excitation:
    """The FDTD element's excitation at one source cell."""
    t = cfg.excitation_type
    if t == 0:
        # f0 centre and fc cutoff: tau = 1 / (pi fc), a pulse without carrier
        # for f0 = 0, else modulated at f0 (the reference's
        # Excitation::gaussian reads its second argument as a fractional
        # bandwidth of a non-zero centre, src/fdtd/excitation.rs:67-86)
        if not cfg.fc > 0:
            raise N.ConfigError("a Gaussian excitation needs fc > 0")
        tau = 1.0 / (math.pi * cfg.fc)
        e = fdtd.Excitation.gaussian_pulse(tau, 4.0 * tau, component, position) if cfg.f0 == 0 else \
            fdtd.Excitation.gaussian_modulated(cfg.f0, cfg.fc / cfg.f0, component, position)
    elif t == 1:
        e = fdtd.Excitation.sinusoidal(cfg.f0, component, position)
    elif t == 2:
        e = fdtd.Excitation.dirac(1.0, component, position)
    elif t == 3:
        e = fdtd.Excitation(fdtd.ExcitationType.Step, (), component, tuple(position))
    else:
        raise N.ConfigError(f"excitation type {t} is not supported")
    return e.with_amplitude(e.amplitude * weight)


def run_operator(operator: fdtd.Operator, excitations: Sequence[fdtd.Excitation], cap: int,
                 end_db: Optional[float] = None, mur_faces: Sequence[bool] = (False,) * 6, device: int = -1,
                 batch: int = 1000, storage: str = "f32") -> dict:
    """Runs an operator (CPML from its PML faces, Mur on `mur_faces`) with
    soft / hard point sources for `cap` steps or until the energy has
    decayed by end_db below its peak (the peak carried across batches, as
    Simulation::run does); returns the run's figures and the engine."""
    import time
    eng = fdtd.Engine(operator, device=device, storage=storage)
    if any(mur_faces):
        eng.add_mur(fdtd.MurAbcConfig(enabled=tuple(bool(v) for v in mur_faces)))
    dt = operator.timestep()
    start, peak, reason, final_db = 0, 0.0, 0, 0.0
    t0 = time.perf_counter()
    while start < cap:
        n = min(batch, cap - start)
        res = eng.run_batch(fdtd.EngineBatch(
            num_steps=n, excitations=[fdtd.ScheduledExcitation.from_excitation(x, start, n, dt) for x in excitations],
            termination=fdtd.TerminationConfig(max_timesteps=n, energy_decay_db=end_db, check_interval=100),
            energy_monitoring=fdtd.EnergyMonitorConfig(sample_interval=100, track_peak=True),
            initial_peak_energy=peak))
        start += res.timesteps_executed
        peak = max(peak, res.peak_energy)
        reason, final_db = int(res.termination_reason), res.final_decay_db
        if res.termination_reason != fdtd.TerminationReason.StepsCompleted or res.timesteps_executed == 0:
            break
    wall = time.perf_counter() - t0
    dims = operator.dimensions()
    cells = dims[0] * dims[1] * dims[2]
    e, h = eng.energy()
    return {"dims": list(dims), "timesteps": start, "termination_reason": reason, "final_decay_db": final_db,
            "sources": len(excitations), "wall_s": wall, "mcells_per_s": cells * start / max(wall, 1e-12) / 1e6,
            "peak_energy": peak, "energy": e + h, "engine": eng}


def run(cfg: SimulationConfig, device: int = -1, batch: int = 1000, storage: str = "f32") -> dict:
    """Runs a parsed configuration on the GPU; returns the run's figures."""
    b = build(cfg)
    excs = [waveform(cfg, pos, comp, w) for pos, comp, w in b.sources]
    end_db = cfg.end_criteria_db
    cap = cfg.num_timesteps if cfg.num_timesteps > 0 else (10000 if end_db is None else 10 ** 7)
    return run_operator(b.operator, excs, cap, end_db, b.mur_faces, device, batch, storage)


def debug_dumps(op: "fdtd.Operator", stem: str, material: bool, operator: bool) -> List[str]:
    """The --debug-material / --debug-operator files of an operator (cell
    data on its mesh lines); returns the paths written."""
    from . import field_io
    g = op.grid
    lines = [np.asarray(v, dtype=np.float64) * g.unit for v in (g.x_lines, g.y_lines, g.z_lines)]
    c = op.coefficients()
    out = []
    if material:
        ids, _ = fdtd.compress_coefficients(c)
        path = stem + ".material.vtk"
        field_io.write_field_vtk(path, ids.astype(np.float32), lines, "material")
        out.append(path)
    if operator:
        for k, name in enumerate(("ca", "cb", "da", "db")):
            path = stem + "." + name + ".vtk"
            field_io.write_vector_field_vtk(path, c[3 * k:3 * k + 3], lines, name.capitalize())
            out.append(path)
    return out


def main(argv: Optional[Sequence[str]] = None):
    """python -m openems_b200.xml_config FILE.xml [--no-simulation]
    [--dump-statistics] [--storage f16] with the reference's flags
    (src/main.rs:15-53, 100-185); prints one JSON line.  --engine names
    the reference's CPU engines and is kept for its command lines: every run
    uses the CUDA engine.  --num-threads and --disable-dumps are accepted
    and, as in the reference, change nothing.  --debug-material writes
    FILE.material.vtk (each cell's material: its index among the distinct
    coefficient sets, oems_compress_coefficients) and --debug-operator
    FILE.ca.vtk / .cb.vtk / .da.vtk / .db.vtk (the coefficients as vector
    fields), legacy VTK as the reference's writer; the reference parses the
    two flags but writes nothing.  --dump-statistics writes FILE.stats.json
    with the reference's keys."""
    import argparse
    import json
    import os
    import sys
    p = argparse.ArgumentParser(description="run an openEMS XML configuration on the B200 engine")
    p.add_argument("input")
    p.add_argument("--no-simulation", action="store_true", help="parse and set up only")
    p.add_argument("--dump-statistics", action="store_true", help="write FILE.stats.json")
    p.add_argument("--engine", default="cuda", help="basic | simd | parallel | cuda (all run on the GPU)")
    p.add_argument("--num-threads", type=int, default=0)
    p.add_argument("--disable-dumps", action="store_true")
    p.add_argument("--debug-material", action="store_true")
    p.add_argument("--debug-operator", action="store_true")
    p.add_argument("-v", "--verbose", type=int, default=1)
    p.add_argument("--storage", choices=("f32", "f16", "bf16"), default="f32")
    p.add_argument("--batch", type=int, default=1000)
    a = p.parse_args(argv)
    if a.engine not in ("basic", "simd", "parallel", "cuda") and a.verbose > 0:
        print(f"unknown engine type '{a.engine}', using the CUDA engine", file=sys.stderr)
    if not os.path.exists(a.input):
        raise SystemExit(f"input file not found: {a.input}")
    cfg = parse_config(a.input)
    if a.debug_material or a.debug_operator:
        debug_dumps(build(cfg).operator, os.path.splitext(a.input)[0], a.debug_material, a.debug_operator)
    if a.no_simulation:
        b = build(cfg)
        print(json.dumps({"dims": list(b.operator.dimensions()), "sources": len(b.sources),
                          "timestep": b.operator.timestep(), "boundaries": cfg.boundaries}))
        return
    r = run(cfg, batch=a.batch, storage=a.storage)
    eng = r.pop("engine")
    if a.dump_statistics:
        # the reference's keys (main.rs:163-172): simulated time is steps x dt
        stats = {"timesteps": r["timesteps"], "sim_time": r["timesteps"] * eng.dt, "wall_time": r["wall_s"],
                 "peak_energy": r["peak_energy"], "final_energy": r["energy"],
                 "speed_mcells_per_sec": r["mcells_per_s"]}
        with open(os.path.splitext(a.input)[0] + ".stats.json", "w") as f:
            json.dump(stats, f, indent=2)
    print(json.dumps(r))


if __name__ == "__main__":
    main()
