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

Also the field dumps of src/processing/fields_fd.rs:
`FrequencyDomainFieldDump` over the engine's GPU accumulators and
`TimeDomainFieldDump`'s snapshot cadence and file names.
"""
from __future__ import annotations

import enum
import math
from typing import List, Optional, Sequence, Tuple

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


# ---------------------------------------------------------------------------
# field dumps (src/processing/fields_fd.rs)
# ---------------------------------------------------------------------------

class FdDumpType(enum.IntEnum):
    """FdDumpType (fields_fd.rs:49-56): which fields a dump keeps.  JField
    keeps E and RotH keeps E and H, as in the reference."""

    EField = 0
    HField = 1
    Both = 2
    JField = 3
    RotH = 4


_FD_COMPONENTS = {FdDumpType.EField: 0x07, FdDumpType.HField: 0x38, FdDumpType.Both: 0x3F,
                  FdDumpType.JField: 0x07, FdDumpType.RotH: 0x3F}
_STATE_FIELD_DFT = 8  # OEMS_STATE_FIELD_DFT


class FrequencyDomainFieldDump:
    """FrequencyDomainFieldDump (fields_fd.rs:31-317) over an engine's whole
    grid.  The accumulators live on the GPU and take every `interval`-th step
    of the batches run after the dump is created: X(f) += x(t) exp(-j 2 pi f
    t) 2 dt interval, E at t = n dt and H at (n - 1/2) dt (the reference
    takes one time for both, from each accumulate call).  Sub-sampling is
    fixed at creation, as set_sub_sample before the first accumulate.  The
    accessors return the reference's shapes: per frequency three complex
    arrays of nx * ny * nz values in i, j, k order, zero between sub-samples."""

    def __init__(self, engine, frequencies: Sequence[float], dump_type: FdDumpType = FdDumpType.Both,
                 sub_sample=(1, 1, 1), interval: int = 1):
        self._engine = engine
        self._freqs = [float(f) for f in frequencies]
        self.dump_type = FdDumpType(dump_type)
        self.sub_sample = tuple(max(int(s), 1) for s in sub_sample)
        self.interval = max(int(interval), 1)
        self.dims = tuple(int(n) for n in engine.dims)
        mask = _FD_COMPONENTS[self.dump_type]
        self.dump_e, self.dump_h = bool(mask & 0x07), bool(mask & 0x38)
        nx, ny, nz = self.dims
        self._id = engine.add_field_dft((0, nx, 0, ny, 0, nz), self._freqs, components=mask,
                                        sub_sample=self.sub_sample, interval=self.interval)
        self._start = engine.current_timestep()

    def frequencies(self) -> List[float]:
        return list(self._freqs)

    def num_frequencies(self) -> int:
        return len(self._freqs)

    def num_samples(self) -> int:
        """Steps accumulated since creation or reset."""
        now = self._engine.current_timestep()
        return now // self.interval - self._start // self.interval

    def _full(self, freq_idx: int, base: int):
        nx, ny, nz = self.dims
        sx, sy, sz = self.sub_sample
        out = []
        for c in range(3):
            full = np.zeros((nx, ny, nz), dtype=np.complex128)
            full[::sx, ::sy, ::sz] = self._engine.field_dft(self._id, freq_idx, base + c)
            out.append(full.reshape(-1))
        return out

    def get_e_field(self, freq_idx: int):
        """[Ex, Ey, Ez] accumulators of frequency freq_idx, or None (:220-227)."""
        if not self.dump_e or not 0 <= freq_idx < len(self._freqs):
            return None
        return self._full(freq_idx, 0)

    def get_h_field(self, freq_idx: int):
        if not self.dump_h or not 0 <= freq_idx < len(self._freqs):
            return None
        return self._full(freq_idx, 3)

    def _linear(self, i, j, k) -> int:
        return (i * self.dims[1] + j) * self.dims[2] + k

    @staticmethod
    def _magnitude(f, idx):
        return math.sqrt(sum(abs(f[c][idx]) ** 2 for c in range(3)))

    def get_e_magnitude(self, freq_idx: int, i: int, j: int, k: int) -> float:
        """|E| of the phasor at one cell (:238-245); 0 without E."""
        e = self.get_e_field(freq_idx)
        return 0.0 if e is None else self._magnitude(e, self._linear(i, j, k))

    def get_h_magnitude(self, freq_idx: int, i: int, j: int, k: int) -> float:
        h = self.get_h_field(freq_idx)
        return 0.0 if h is None else self._magnitude(h, self._linear(i, j, k))

    def extract_e_magnitude(self, freq_idx: int) -> Optional[np.ndarray]:
        """|E| per cell as float32 (nx, ny, nz), or None (:258-279)."""
        e = self.get_e_field(freq_idx)
        if e is None:
            return None
        m = np.sqrt(sum(np.abs(e[c]) ** 2 for c in range(3)))
        return m.astype(np.float32).reshape(self.dims)

    def extract_e_phase(self, freq_idx: int, component: int) -> Optional[np.ndarray]:
        """arg of one E component per cell as float32, component clamped to
        2 (:281-301), or None."""
        e = self.get_e_field(freq_idx)
        if e is None:
            return None
        return np.angle(e[min(int(component), 2)]).astype(np.float32).reshape(self.dims)

    def reset(self) -> None:
        """Zero the accumulators (the dump's own state section) and restart
        the sample count (:303-320)."""
        k = -1
        for idx, (kind, nbytes, variant) in enumerate(self._engine.state_sections()):
            if kind == _STATE_FIELD_DFT:
                k += 1
                if k == self._id:
                    self._engine.write_state(idx, bytes(nbytes), variant)
                    break
        self._start = self._engine.current_timestep()


class TimeDomainFieldDump:
    """TimeDomainFieldDump (fields_fd.rs:325-385): the cadence and names of
    time-domain snapshots; `write` puts the engine's present fields in the
    next file (openems_b200.field_io.dump_fields)."""

    def __init__(self, interval: int, path_prefix: str):
        self.interval = int(interval)
        self.sub_sample = (1, 1, 1)
        self.path_prefix = path_prefix
        self.padding = 8
        self._file_index = 0

    def set_sub_sample(self, rate) -> None:
        self.sub_sample = tuple(int(r) for r in rate)

    def should_dump(self, timestep: int) -> bool:
        return self.interval > 0 and int(timestep) % self.interval == 0

    def get_filename(self) -> str:
        return f"{self.path_prefix}_{self._file_index:0{self.padding}d}"

    def increment(self) -> None:
        self._file_index += 1

    def file_index(self) -> int:
        return self._file_index

    def reset(self) -> None:
        self._file_index = 0

    def write(self, engine, grid, fmt: str = "vtk") -> str:
        """The present fields under get_filename(): "vtk" writes
        <name>_E.vtk and <name>_H.vtk, "oems" the binary container <name>.h5
        with the snapshot's time.  The index then moves on.  Returns the
        name (vtk) or the path (oems)."""
        from .field_io import dump_fields
        name = self.get_filename()
        if fmt == "vtk":
            dump_fields(engine, grid, name, fmt="vtk")
        else:
            name += ".h5"
            dump_fields(engine, grid, name, fmt="oems", timestep=engine.current_timestep() * engine.dt)
        self.increment()
        return name
