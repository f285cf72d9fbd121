"""The host side of the probe collections (src/processing/probes.rs tests):
names, cells, the collection and frequency_response on given samples.
Sampling on the engine is in tests/test_gpu_processing.py."""
import numpy as np

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
