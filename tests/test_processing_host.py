"""The host side of the probe collections (src/processing/probes.rs tests):
names, cells, the collection and frequency_response on given samples.
Sampling on the engine is in tests/test_gpu_processing.py."""
import numpy as np
import pytest

from openems_b200.processing import CurrentProbe, FieldProbe, Processing, VoltageProbe, _bin


def test_processing_default_and_collection():
    """test_processing_default / test_processing_collection."""
    p = Processing()
    assert not p.voltage_probes and not p.current_probes and not p.field_probes
    p.add_voltage_probe(VoltageProbe("v", (5, 5, 0), (5, 5, 10), 2))
    p.add_current_probe(CurrentProbe("i", (5, 0, 0), (5, 10, 10), 0))
    p.add_field_probe(FieldProbe("f", (5, 5, 5)))
    assert (len(p.voltage_probes), len(p.current_probes), len(p.field_probes)) == (1, 1, 1)


def test_probe_name_storage_and_positions():
    """test_probe_name_storage / test_probe_positions."""
    v = VoltageProbe("voltage_1", (1, 2, 3), (4, 5, 6), 0)
    c = CurrentProbe("current_1", (10, 20, 30), (40, 50, 60), 2)
    f = FieldProbe("field_1", (7, 8, 9))
    assert (v.name, c.name, f.name) == ("voltage_1", "current_1", "field_1")
    assert v.start == (1, 2, 3) and v.end == (4, 5, 6) and v.direction == 0
    assert c.start == (10, 20, 30) and c.end == (40, 50, 60) and c.normal_direction == 2
    assert f.position == (7, 8, 9)


def test_frequency_response():
    """test_voltage_probe_frequency_response, test_current_probe_frequency_response,
    test_voltage_probe_frequency_response_out_of_range."""
    v = VoltageProbe("test_freq", (5, 5, 0), (5, 5, 4), 2)
    v.times = [i * 1e-9 for i in range(16)]
    v.values = [1.0] * 16
    r = v.frequency_response([0.0, 1e8, 2e8], 1e-9)
    assert len(r) == 3 and abs(r[0]) > 0.5
    # constant signal: all of it in bin 0 (= n), nothing in bins 2 and 3
    assert r[0] == 16.0 and abs(r[1]) < 1e-12 and abs(r[2]) < 1e-12
    c = CurrentProbe("test_freq", (5, 0, 0), (5, 4, 4), 0)
    c.values = [1.0] * 8
    r = c.frequency_response([0.0, 1e8], 1e-9)
    assert len(r) == 2 and abs(r[0]) > 0.5
    v = VoltageProbe("test_oor", (5, 5, 0), (5, 5, 4), 2)
    v.values = [1.0] * 4
    r = v.frequency_response([1e12], 1e-9)
    assert len(r) == 1 and r[0] == 0.0
    # the bin of a sine: f * n * dt rounded, the DFT's n/2 there
    v.values = np.sin(2 * np.pi * 3 * np.arange(32) / 32).tolist()
    r = v.frequency_response([3 / (32 * 1e-9)], 1e-9)
    assert abs(r[0] - (-16j)) < 1e-12
    assert VoltageProbe("e", (0, 0, 0), (0, 0, 0), 0).frequency_response([0.0], 1e-9)[0] == 0.0


def test_bin_rounding():
    """Rust's f64::round (half away from zero) and the saturating cast to usize."""
    assert _bin(0.5, 1, 1.0) == 1 and _bin(1.5, 1, 1.0) == 2 and _bin(2.5, 1, 1.0) == 3
    assert _bin(0.49999999999999994, 1, 1.0) == 0
    assert _bin(-3.0, 1, 1.0) == 0 and _bin(float("nan"), 1, 1.0) == 0
    assert _bin(float("inf"), 1, 1.0) >= 1 << 63


class _FakeEngine:
    """Records probe registrations and serves fixed traces (host logic only)."""

    def __init__(self):
        self.n, self.dt, self.step = 0, 2e-12, 0
        self.traces = None

    def add_probe(self, terms):
        self.n += 1
        return self.n - 1

    def add_point_probe(self, c, pos):
        self.n += 1
        return self.n - 1

    def probe_traces(self):
        return self.traces

    def current_timestep(self):
        return self.step


def test_record_and_collect_columns_and_times():
    """record registers the probes in order (a field probe takes six columns);
    collect appends each probe's column with time = step count x dt, and
    only for the engine it was recorded on."""
    p = Processing()
    p.add_voltage_probe(VoltageProbe("v", (0, 0, 0), (0, 0, 3), 2))
    p.add_field_probe(FieldProbe("f", (1, 1, 1)))
    p.add_current_probe(CurrentProbe("i", (0, 0, 1), (2, 2, 1), 2))
    eng, other = _FakeEngine(), _FakeEngine()
    p.record(eng)
    assert eng.n == 1 + 1 + 6
    eng.traces = np.arange(3 * 8, dtype=np.float64).reshape(3, 8)
    eng.step = 10
    assert p.collect(eng) == 3
    v, i, f = p.voltage_probes[0], p.current_probes[0], p.field_probes[0]
    assert v.values == [0.0, 8.0, 16.0] and i.values == [1.0, 9.0, 17.0]
    assert f.e_values[0] == (2.0, 3.0, 4.0) and f.h_values[2] == (21.0, 22.0, 23.0)
    assert v.times == [8 * 2e-12, 9 * 2e-12, 10 * 2e-12]
    other.traces = np.zeros((2, 8))
    p.collect(other)
    assert len(v.values) == 3


# ---- field dumps (src/processing/fields_fd.rs tests) over a stand-in engine --

from openems_b200.processing import FdDumpType, FrequencyDomainFieldDump, TimeDomainFieldDump  # noqa: E402


class _FdEngine:
    """add_field_dft / field_dft / state sections of an engine, with
    accumulators = deterministic complex values on the sub-sampled points."""

    def __init__(self, dims):
        self.dims, self.dt, self.step = dims, 1e-12, 0
        self.dumps, self.writes = [], []

    def add_field_dft(self, region, freqs, components, sub_sample, interval):
        shape = tuple(-(-(region[2 * a + 1] - region[2 * a]) // sub_sample[a]) for a in range(3))
        self.dumps.append((shape, components, len(freqs)))
        return len(self.dumps) - 1

    def field_dft(self, dump_id, f, c):
        shape = self.dumps[dump_id][0]
        n = int(np.prod(shape))
        return ((np.arange(n) + 1.0 + 10 * c + 100 * f) * (1 + 1j)).reshape(shape)

    def current_timestep(self):
        return self.step

    def state_sections(self):
        return [(1, 64, 0)] + [(8, 16 * (k + 1), 0) for k in range(len(self.dumps))]

    def write_state(self, idx, data, variant):
        self.writes.append((idx, len(data), variant, set(data)))


def test_fd_dump_creation_and_sample_count():
    """test_fd_dump_creation, test_fd_reset: frequencies, samples counted
    per interval since creation or reset; reset zeroes the dump's own
    accumulator section."""
    eng = _FdEngine((10, 10, 10))
    eng.step = 7
    FrequencyDomainFieldDump(eng, [5e9], FdDumpType.HField)
    d = FrequencyDomainFieldDump(eng, [1e9, 2e9, 3e9], FdDumpType.Both, interval=2)
    assert d.num_frequencies() == 3 and d.frequencies() == [1e9, 2e9, 3e9]
    assert d.num_samples() == 0
    eng.step = 12  # steps 8, 10, 12
    assert d.num_samples() == 3
    d.reset()
    assert eng.writes == [(2, 32, 0, {0})] and d.num_samples() == 0
    assert eng.dumps[1][1] == 0x3F and eng.dumps[0][1] == 0x38


def test_fd_accessors_and_magnitude():
    """get_e_field / get_h_field by dump type, the full i, j, k layout with
    sub-sampling, get_e_magnitude, extract_e_magnitude / extract_e_phase
    (test_extract_magnitude, test_sub_sampling)."""
    eng = _FdEngine((5, 4, 6))
    d = FrequencyDomainFieldDump(eng, [1e9, 2e9], FdDumpType.EField, sub_sample=(2, 1, 3))
    assert d.get_h_field(0) is None and d.get_e_field(2) is None and d.get_h_magnitude(0, 0, 0, 0) == 0.0
    e = d.get_e_field(1)
    assert len(e) == 3 and all(a.shape == (5 * 4 * 6,) for a in e)
    full = e[2].reshape(5, 4, 6)
    np.testing.assert_array_equal(full[::2, :, ::3], eng.field_dft(0, 1, 2))
    assert full[1, 0, 0] == 0 and full[0, 0, 1] == 0
    want = np.sqrt(sum(abs(e[c].reshape(5, 4, 6)[2, 3, 3]) ** 2 for c in range(3)))
    assert d.get_e_magnitude(1, 2, 3, 3) == pytest.approx(want, rel=1e-15)
    mag = d.extract_e_magnitude(1)
    assert mag.dtype == np.float32 and mag.shape == (5, 4, 6) and mag[2, 3, 3] == np.float32(want)
    ph = d.extract_e_phase(0, 7)
    assert ph.dtype == np.float32 and ph[0, 0, 0] == np.float32(np.pi / 4)
    assert FrequencyDomainFieldDump(eng, [1e9], FdDumpType.JField).get_h_field(0) is None
    assert FrequencyDomainFieldDump(eng, [1e9], FdDumpType.RotH).get_h_field(0) is not None


def test_td_dump():
    """test_td_dump: every 100 steps, names prefix_00000000, ..."""
    dump = TimeDomainFieldDump(100, "field_dump")
    assert dump.should_dump(0) and not dump.should_dump(50) and dump.should_dump(100)
    assert dump.get_filename() == "field_dump_00000000"
    dump.increment()
    assert dump.get_filename() == "field_dump_00000001" and dump.file_index() == 1
    dump.reset()
    assert dump.file_index() == 0
    assert not TimeDomainFieldDump(0, "x").should_dump(0)


def test_td_dump_writes_the_next_snapshot(tmp_path):
    """write: the engine's present fields under the next name, VTK pair or
    the binary container, then the index moves on."""
    import openems_b200 as oe

    class Fields:
        dt = 1e-12

        def read_fields(self):
            e = np.zeros((3, 2, 3, 4), np.float32)
            e[2, 1, 2, 3] = 1.5
            return e, np.zeros_like(e)

        def current_timestep(self):
            return 300

    grid = oe.Grid.uniform(2, 3, 4, 1e-3)
    dump = TimeDomainFieldDump(100, str(tmp_path / "snap"))
    name = dump.write(Fields(), grid)
    assert name.endswith("snap_00000000") and dump.file_index() == 1
    assert (tmp_path / "snap_00000000_E.vtk").exists() and (tmp_path / "snap_00000000_H.vtk").exists()
    path = dump.write(Fields(), grid, fmt="oems")
    assert path.endswith("snap_00000001.h5") and (tmp_path / "snap_00000001.h5").exists()
