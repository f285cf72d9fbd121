"""Engine checkpoints: the whole evolving state of an engine as one blob,
loaded into an engine built the same way to continue the run bit for bit.

The engine lists its state as sections (oems_engine_state_sections): the
fields in their storage type and every extension's state -- CPML psi, Mur,
probe DFTs, dispersive and lumped-RLC state, UPML flux, field-DFT and NF2FF
accumulators, the TF/SF 1D grid -- plus the step counters.  The reference
has only read_fields / write_fields for this (src/fdtd/engine_impl.rs:59-70),
which leave the extension state behind.  Blob layout, little-endian:

    b"OEMSSNAP", u32 version (2), u32 section count,
    u64 timestep, u64 TF/SF step, f64 dt, u64 nx, ny, nz,
    per section: u32 kind, u32 variant, u64 bytes, the bytes.

The variant tells apart sections of one kind and size that hold different
encodings: the fields section's is the storage type (0 float, 1 IEEE half,
2 bfloat16; half and bfloat16 fields have the same byte count).  Version 1
blobs wrote 0 there and still load into float engines.

Loading checks the grid, dt and every section's kind, variant and size
against the target engine before it writes anything.
"""
from __future__ import annotations

import os
import struct
from dataclasses import dataclass
from typing import List, Tuple

from . import _native as N

MAGIC = b"OEMSSNAP"
VERSION = 2
READABLE = (1, 2)
HEADER = struct.Struct("<8sIIQQdQQQ")
SECTION = struct.Struct("<IIQ")
KINDS = {1: "fields", 2: "cpml", 3: "mur", 4: "probe_dft", 5: "dispersive", 6: "lumped_rlc", 7: "upml",
         8: "field_dft", 9: "nf2ff", 10: "tfsf_e", 11: "tfsf_h"}


class CheckpointError(N.ConfigError):
    """A checkpoint that is malformed or does not fit the engine."""


@dataclass
class Snapshot:
    timestep: int
    tfsf_step: int
    dt: float
    dims: Tuple[int, int, int]
    sections: List[Tuple[int, bytes, int]]  # kind, bytes, variant


def pack(engine) -> bytes:
    """The engine's state as a checkpoint blob."""
    secs = engine.state_sections()
    ts, tf = engine.state_counters()
    parts = [HEADER.pack(MAGIC, VERSION, len(secs), ts, tf, float(engine.dt), *(int(d) for d in engine.dims))]
    for i, (kind, n, variant) in enumerate(secs):
        parts.append(SECTION.pack(kind, variant, n))
        parts.append(engine.read_state(i, n))
    return b"".join(parts)


def parse(blob) -> Snapshot:
    """Splits a blob into its header and sections (no engine involved)."""
    buf = memoryview(blob).cast("B")
    if len(buf) < HEADER.size:
        raise CheckpointError("checkpoint shorter than its header")
    magic, version, count, ts, tf, dt, nx, ny, nz = HEADER.unpack_from(buf, 0)
    if magic != MAGIC:
        raise CheckpointError("not an engine checkpoint")
    if version not in READABLE:
        raise CheckpointError(f"checkpoint version {version}, this build reads {READABLE}")
    pos, sections = HEADER.size, []
    for k in range(count):
        if pos + SECTION.size > len(buf):
            raise CheckpointError(f"checkpoint truncated in section {k}")
        kind, variant, n = SECTION.unpack_from(buf, pos)
        pos += SECTION.size
        if pos + n > len(buf):
            raise CheckpointError(f"checkpoint truncated in section {k} ({KINDS.get(kind, kind)})")
        sections.append((kind, bytes(buf[pos:pos + n]), variant))
        pos += n
    if pos != len(buf):
        raise CheckpointError(f"{len(buf) - pos} bytes after the last section")
    return Snapshot(ts, tf, dt, (nx, ny, nz), sections)


def unpack(engine, blob) -> Snapshot:
    """Loads a blob into an engine with the same grid, dt, extensions and
    field storage.  Every check runs before the first section is written.
    If a write still fails part-way (a CUDA error), the engine is reset --
    fields, extension state and counters cleared -- before the error is
    raised, so it never continues from a mix of old and loaded state."""
    snap = parse(blob)
    if tuple(int(d) for d in engine.dims) != snap.dims:
        raise CheckpointError(f"checkpoint grid {snap.dims}, engine grid {tuple(engine.dims)}")
    if float(engine.dt) != snap.dt:
        raise CheckpointError(f"checkpoint dt {snap.dt!r}, engine dt {engine.dt!r}")
    want = [tuple(s) for s in engine.state_sections()]
    got = [(kind, len(data), variant) for kind, data, variant in snap.sections]
    if got != want:
        names = lambda s: [(KINDS.get(k, k), n, v) for k, n, v in s]  # noqa: E731
        raise CheckpointError(f"checkpoint sections (kind, bytes, variant) {names(got)} do not match the "
                              f"engine's {names(want)}")
    try:
        for i, (_, data, variant) in enumerate(snap.sections):
            engine.write_state(i, data, variant)
        engine.set_state_counters(snap.timestep, snap.tfsf_step)
    except Exception as exc:
        engine.reset()
        raise CheckpointError(f"loading the checkpoint failed part-way; the engine was reset: {exc}") from exc
    return snap


def save(engine, path) -> int:
    """Writes the engine's checkpoint to `path` (through a temporary file
    renamed into place); returns its size in bytes."""
    blob = pack(engine)
    path = os.fspath(path)
    tmp = path + ".tmp"
    with open(tmp, "wb") as f:
        f.write(blob)
    os.replace(tmp, path)
    return len(blob)


def load(engine, path) -> Snapshot:
    with open(path, "rb") as f:
        return unpack(engine, f.read())
