"""Checkpoint blobs (openems_b200.checkpoint) on CPU, against a stand-in
engine that keeps its sections in host memory: pack / unpack round trips
and every refusal, which happen before any section is written."""
import numpy as np
import pytest

from openems_b200 import checkpoint as C


class FakeEngine:
    """Sections (kind, bytes, variant): variant is the field storage type of
    the fields section (0 float, 1 half, 2 bfloat16), as the engine reports it."""

    def __init__(self, dims=(6, 5, 4), dt=1.25e-12, kinds=((1, 480, 0), (2, 96, 0), (10, 64, 0), (11, 64, 0)),
                 seed=0, fail_at=None):
        rng = np.random.default_rng(seed)
        self.dims, self.dt = dims, dt
        self.kinds = [tuple(k) for k in kinds]
        self.data = [rng.integers(0, 256, n, dtype=np.uint8).tobytes() for _, n, _ in self.kinds]
        self.counters = (int(rng.integers(1, 10_000)), int(rng.integers(0, 10_000)))
        self.writes = 0
        self.resets = 0
        self.fail_at = fail_at

    def state_sections(self):
        return list(self.kinds)

    def read_state(self, i, n):
        assert n == self.kinds[i][1]
        return self.data[i]

    def write_state(self, i, data, variant=0):
        assert len(data) == self.kinds[i][1] and variant == self.kinds[i][2]
        if i == self.fail_at:
            raise RuntimeError("device copy failed")
        self.data[i] = bytes(data)
        self.writes += 1

    def reset(self):
        self.data = [bytes(len(d)) for d in self.data]
        self.counters = (0, 0)
        self.resets += 1

    def state_counters(self):
        return self.counters

    def set_state_counters(self, ts, tf):
        self.counters = (ts, tf)


def test_round_trip():
    a, b = FakeEngine(seed=1), FakeEngine(seed=2)
    blob = C.pack(a)
    assert len(blob) == C.HEADER.size + sum(C.SECTION.size + n for _, n, _ in a.kinds)
    snap = C.unpack(b, blob)
    assert b.data == a.data and b.counters == a.counters
    assert snap.dims == a.dims and snap.dt == a.dt and [k for k, _, _ in snap.sections] == [1, 2, 10, 11]
    assert C.pack(b) == blob


def test_file_round_trip(tmp_path):
    a, b = FakeEngine(seed=3), FakeEngine(seed=4)
    n = C.save(a, tmp_path / "ck.oems")
    assert n == (tmp_path / "ck.oems").stat().st_size and not (tmp_path / "ck.oems.tmp").exists()
    C.load(b, tmp_path / "ck.oems")
    assert b.data == a.data and b.counters == a.counters


def test_empty_sections_and_no_extensions():
    a, b = FakeEngine(kinds=((1, 0, 0),), seed=5), FakeEngine(kinds=((1, 0, 0),), seed=6)
    C.unpack(b, C.pack(a))
    assert b.counters == a.counters


@pytest.mark.parametrize("mutate,match", [
    (lambda b: b"XXXXSNAP" + b[8:], "not an engine checkpoint"),
    (lambda b: b[:8] + (3).to_bytes(4, "little") + b[12:], "version 3"),
    (lambda b: b[:20], "shorter than its header"),
    (lambda b: b[:-1], "truncated"),
    (lambda b: b[:C.HEADER.size + 4], "truncated in section 0"),
    (lambda b: b + b"\0", "1 bytes after the last section"),
])
def test_malformed_blobs_are_refused(mutate, match):
    a, b = FakeEngine(seed=7), FakeEngine(seed=8)
    before = list(b.data)
    with pytest.raises(C.CheckpointError, match=match):
        C.unpack(b, mutate(C.pack(a)))
    assert b.data == before and b.writes == 0


@pytest.mark.parametrize("other,match", [
    (dict(dims=(6, 5, 5)), "grid"),
    (dict(dt=1.2500000000000002e-12), "dt"),
    (dict(kinds=((1, 480, 0), (2, 96, 0))), "sections"),                      # engine without TF/SF
    (dict(kinds=((1, 480, 0), (3, 96, 0), (10, 64, 0), (11, 64, 0))), "sections"),  # Mur instead of CPML
    (dict(kinds=((1, 240, 1), (2, 96, 0), (10, 64, 0), (11, 64, 0))), "sections"),  # 2-byte field storage
])
def test_mismatched_engines_are_refused(other, match):
    a, b = FakeEngine(seed=9), FakeEngine(seed=10, **other)
    before = list(b.data)
    with pytest.raises(C.CheckpointError, match=match):
        C.unpack(b, C.pack(a))
    assert b.data == before and b.writes == 0


def test_checkpoint_error_is_a_config_error():
    from openems_b200 import _native as N
    assert issubclass(C.CheckpointError, N.ConfigError)


def test_half_and_bfloat16_fields_are_told_apart():
    """Half and bfloat16 field sections have the same size; the variant
    (storage type) keeps a snapshot of one from loading into the other."""
    f16 = ((1, 240, 1), (2, 96, 0))
    bf16 = ((1, 240, 2), (2, 96, 0))
    a, b = FakeEngine(kinds=f16, seed=11), FakeEngine(kinds=bf16, seed=12)
    before = list(b.data)
    with pytest.raises(C.CheckpointError, match="variant"):
        C.unpack(b, C.pack(a))
    assert b.data == before and b.writes == 0
    c = FakeEngine(kinds=f16, seed=13)
    C.unpack(c, C.pack(a))
    assert c.data == a.data


def test_version1_blob_loads_into_a_float_engine():
    a, b = FakeEngine(seed=14), FakeEngine(seed=15)
    blob = bytearray(C.pack(a))
    blob[8:12] = (1).to_bytes(4, "little")
    C.unpack(b, bytes(blob))
    assert b.data == a.data


def test_failed_write_resets_the_engine():
    a, b = FakeEngine(seed=16), FakeEngine(seed=17, fail_at=2)
    with pytest.raises(C.CheckpointError, match="reset"):
        C.unpack(b, C.pack(a))
    assert b.resets == 1 and b.writes == 2
    assert all(d == bytes(len(d)) for d in b.data) and b.counters == (0, 0)
