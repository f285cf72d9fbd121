"""Probe collections with the reference's processing API.

`Processing`, `VoltageProbe`, `CurrentProbe` and `FieldProbe`
(src/processing/probes.rs:8-303) keep a probe's name, its cells and its
(time, value) samples.  Two ways to fill them on the CUDA engine:

- `process(engine, time)` samples every probe on the present fields, as the
  reference's `Processing::process` does between steps (one launch per
  probe, `oems_engine_eval_terms`);
- `record(engine)` registers the probes with the engine so that every step
  of the following batches records them on the GPU, in the post-step launch,
  and `collect(engine)` appends the steps of the most recent batch (time =
  the step count after each step times dt).

Both give the reference's sums: VoltageProbe / CurrentProbe add their cell
values in order in f32 (a direction other than 0..2 records 0), FieldProbe
records the six components as f64.  `frequency_response` is the reference's:
the FFT of the samples (numpy's, unnormalised like rustfft's), read at bin
round(f * n * dt), 0 past the last bin.
"""
from __future__ import annotations

import math
from typing import List, Sequence, Tuple

import numpy as np

from .fdtd import ProbeTerms, current_probe, voltage_probe

Cell = Tuple[int, int, int]


def _bin(f: float, n: int, dt: float) -> int:
    """(f * n * dt).round() as usize: half away from zero, negatives and NaN to 0."""
    x = f * n * dt
    if not x > 0.0:
        return 0
    if math.isinf(x):
        return 1 << 64
    r = math.floor(x)
    return int(r) + (1 if x - r >= 0.5 else 0)


def _frequency_response(values: Sequence[float], frequencies, dt: float) -> np.ndarray:
    n = len(values)
    spectrum = np.fft.fft(np.asarray(values, dtype=np.float64)) if n else np.zeros(0, np.complex128)
    out = np.zeros(len(frequencies), dtype=np.complex128)
    for q, f in enumerate(frequencies):
        b = _bin(float(f), n, dt)
        if b < n:
            out[q] = spectrum[b]
    return out


class _TermProbe:
    """A probe given by a term list (`terms()` of the subclass)."""

    def __init__(self, name: str, start: Cell, end: Cell):
        self.name = name
        self.start = tuple(int(v) for v in start)
        self.end = tuple(int(v) for v in end)
        self.times: List[float] = []
        self.values: List[float] = []
        self._ids = {}

    def sample(self, engine, time: float) -> None:
        self.times.append(float(time))
        self.values.append(engine.evaluate_probe(self.terms()))

    def frequency_response(self, frequencies, dt: float) -> np.ndarray:
        return _frequency_response(self.values, frequencies, dt)


class VoltageProbe(_TermProbe):
    """VoltageProbe::new(name, start, end, direction) (:79-96): E[direction]
    summed from start to end inclusive along that axis."""

    def __init__(self, name: str, start: Cell, end: Cell, direction: int):
        super().__init__(name, start, end)
        self.direction = int(direction)

    def terms(self) -> ProbeTerms:
        return voltage_probe(self.start, self.end, self.direction)


class CurrentProbe(_TermProbe):
    """CurrentProbe::new(name, start, end, normal_direction) (:171-191): the
    tangential H of the face cells, first component added, second subtracted."""

    def __init__(self, name: str, start: Cell, end: Cell, normal_direction: int):
        super().__init__(name, start, end)
        self.normal_direction = int(normal_direction)

    def terms(self) -> ProbeTerms:
        return current_probe(self.start, self.end, self.normal_direction)


class FieldProbe:
    """FieldProbe::new(name, position) (:276-303): E and H at one cell."""

    def __init__(self, name: str, position: Cell):
        self.name = name
        self.position = tuple(int(v) for v in position)
        self.times: List[float] = []
        self.e_values: List[Tuple[float, float, float]] = []
        self.h_values: List[Tuple[float, float, float]] = []
        self._ids = {}

    def _component(self, c: int) -> ProbeTerms:
        return ProbeTerms([(c, self.position, 1.0)], 1)

    def sample(self, engine, time: float) -> None:
        v = [engine.evaluate_probe(self._component(c)) for c in range(6)]
        self.times.append(float(time))
        self.e_values.append(tuple(v[:3]))
        self.h_values.append(tuple(v[3:]))


class Processing:
    """Processing (:8-61): the probes of a run."""

    def __init__(self):
        self.voltage_probes: List[VoltageProbe] = []
        self.current_probes: List[CurrentProbe] = []
        self.field_probes: List[FieldProbe] = []

    def add_voltage_probe(self, probe: VoltageProbe) -> None:
        self.voltage_probes.append(probe)

    def add_current_probe(self, probe: CurrentProbe) -> None:
        self.current_probes.append(probe)

    def add_field_probe(self, probe: FieldProbe) -> None:
        self.field_probes.append(probe)

    def process(self, engine, time: float) -> None:
        """Processing::process (:43-55): every probe sampled now."""
        for p in self.voltage_probes:
            p.sample(engine, time)
        for p in self.current_probes:
            p.sample(engine, time)
        for p in self.field_probes:
            p.sample(engine, time)

    def record(self, engine) -> "Processing":
        """Record every probe at each step of the engine's following batches."""
        key = id(engine)
        # the engine is kept with its probe ids, so its id stays its own
        for p in self.voltage_probes + self.current_probes:
            p._ids[key] = (engine, engine.add_probe(p.terms()))
        for p in self.field_probes:
            p._ids[key] = (engine, [engine.add_point_probe(c, p.position) for c in range(6)])
        return self

    @staticmethod
    def _recorded(p, engine):
        e = p._ids.get(id(engine))
        return e[1] if e is not None and e[0] is engine else None

    def collect(self, engine) -> int:
        """Append the recorded steps of the engine's most recent batch; returns
        the number of steps."""
        tr = engine.probe_traces()
        steps = tr.shape[0]
        end = engine.current_timestep()
        times = [(end - steps + 1 + s) * engine.dt for s in range(steps)]
        for p in self.voltage_probes + self.current_probes:
            pid = self._recorded(p, engine)
            if pid is not None:
                p.times.extend(times)
                p.values.extend(tr[:, pid].tolist())
        for p in self.field_probes:
            pids = self._recorded(p, engine)
            if pids is not None:
                cols = tr[:, pids]
                p.times.extend(times)
                p.e_values.extend(tuple(r[:3]) for r in cols.tolist())
                p.h_values.extend(tuple(r[3:]) for r in cols.tolist())
        return steps
