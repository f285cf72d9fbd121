"""Field data files: the openEMS binary container and legacy VTK.

`Hdf5Writer` / `Hdf5Reader` restate the reference's writer and reader
(src/io/hdf5.rs:263-426, :53-213) for a build without the `hdf5` feature,
which is what the reference's default build writes: a little-endian binary
container

    b"OEMS", version bytes 1 0 0 0, i32 mesh type,
    3 x (u64 count, count x f64 mesh lines),
    u64 count + f64 timesteps, u64 count + f64 frequencies,
    u64 n, n x (u64 name length, name, u64 count, count x f32)     scalar fields
    u64 n, n x (u64 name length, name, 3 x (u64 count, count x f32)) vector fields
    u64 n, n x (u64 name length, name, u64 count, count x (f64 re, f64 im))

The reference writes empty timestep and frequency lists and drops
attributes; so does this writer unless `set_timesteps` / `set_frequencies`
are called (then the lists hold them, which the reference's reader reads
too).  The reader here also returns the fields, which the reference's
reader skips.

`write_field_vtk` / `write_vector_field_vtk` restate src/io/vtk.rs:10-126:
legacy ASCII rectilinear grids with cell data, numbers printed like Rust's
`{}` (shortest round-trip digits, never an exponent), so the files are
byte-identical to the reference's for the same data.

`dump_fields` / `dump_field_dft` take the data from an engine's device
buffers (one read per component) into either format.
"""
from __future__ import annotations

import os
import struct
from dataclasses import dataclass, field
from typing import Dict, List, Optional, Sequence, Tuple

import numpy as np

CARTESIAN, CYLINDRICAL = 0, 1


def mesh_type_from(v: int) -> int:
    """MeshType::from (src/io/hdf5.rs:24-31): 1 cylindrical, else cartesian."""
    return CYLINDRICAL if v == 1 else CARTESIAN


class Hdf5Writer:
    """Hdf5Writer (src/io/hdf5.rs:263-426), binary-container form."""

    def __init__(self, path):
        self.path = os.fspath(path)
        self.current_group = "/"
        self.mesh_lines: Optional[List[np.ndarray]] = None
        self.mesh_type = CARTESIAN
        self.scalar_fields: List[Tuple[str, np.ndarray]] = []
        self.vector_fields: List[Tuple[str, Tuple[np.ndarray, ...]]] = []
        self.complex_fields: List[Tuple[str, np.ndarray]] = []
        self.attributes: Dict[str, np.ndarray] = {}
        self.timesteps = np.zeros(0)
        self.frequencies = np.zeros(0)

    def set_current_group(self, group: str):
        self.current_group = group

    def write_rect_mesh(self, lines: Sequence[Sequence[float]], mesh_type: int = CARTESIAN):
        self.mesh_lines = [np.asarray(v, dtype=np.float64) for v in lines]
        self.mesh_type = int(mesh_type)

    def write_scalar_field(self, name: str, data):
        self.scalar_fields.append((name, np.asarray(data, dtype=np.float32).ravel()))

    def write_scalar_field_f64(self, name: str, data):
        self.write_scalar_field(name, np.asarray(data, dtype=np.float64).astype(np.float32))

    def write_vector_field(self, name: str, components):
        self.vector_fields.append((name, tuple(np.asarray(c, dtype=np.float32).ravel() for c in components)))

    def write_complex_field(self, name: str, data):
        self.complex_fields.append((name, np.asarray(data, dtype=np.complex128).ravel()))

    def write_attribute(self, name: str, values):
        # kept in memory only: the binary container has no attribute section
        self.attributes[name] = np.asarray(values, dtype=np.float64)

    def set_timesteps(self, t):
        self.timesteps = np.asarray(t, dtype=np.float64)

    def set_frequencies(self, f):
        self.frequencies = np.asarray(f, dtype=np.float64)

    def close(self):
        u64 = struct.Struct("<Q")
        with open(self.path, "wb") as f:
            f.write(b"OEMS")
            f.write(bytes([1, 0, 0, 0]))
            f.write(struct.pack("<i", self.mesh_type))
            for lines in (self.mesh_lines or [np.zeros(0)] * 3):
                f.write(u64.pack(len(lines)))
                f.write(lines.astype("<f8").tobytes())
            for arr in (self.timesteps, self.frequencies):
                f.write(u64.pack(len(arr)))
                f.write(arr.astype("<f8").tobytes())
            f.write(u64.pack(len(self.scalar_fields)))
            for name, data in self.scalar_fields:
                nb = name.encode()
                f.write(u64.pack(len(nb)) + nb + u64.pack(len(data)))
                f.write(data.astype("<f4").tobytes())
            f.write(u64.pack(len(self.vector_fields)))
            for name, comps in self.vector_fields:
                nb = name.encode()
                f.write(u64.pack(len(nb)) + nb)
                for c in comps:
                    f.write(u64.pack(len(c)))
                    f.write(c.astype("<f4").tobytes())
            f.write(u64.pack(len(self.complex_fields)))
            for name, data in self.complex_fields:
                nb = name.encode()
                f.write(u64.pack(len(nb)) + nb + u64.pack(len(data)))
                f.write(np.stack([data.real, data.imag], 1).astype("<f8").tobytes())


@dataclass
class Hdf5Reader:
    """Hdf5Reader (src/io/hdf5.rs:36-258) for the binary container; also
    returns the fields."""

    path: str
    mesh_lines: List[np.ndarray]
    mesh_type: int
    timesteps: np.ndarray
    frequencies: np.ndarray
    scalar_fields: Dict[str, np.ndarray] = field(default_factory=dict)
    vector_fields: Dict[str, Tuple[np.ndarray, ...]] = field(default_factory=dict)
    complex_fields: Dict[str, np.ndarray] = field(default_factory=dict)

    @classmethod
    def open(cls, path) -> "Hdf5Reader":
        with open(path, "rb") as f:
            buf = f.read()
        if buf[:4] != b"OEMS":
            raise ValueError("Invalid file format")
        pos = 8
        mesh_type = mesh_type_from(struct.unpack_from("<i", buf, pos)[0])
        pos += 4

        def count():
            nonlocal pos
            n = struct.unpack_from("<Q", buf, pos)[0]
            pos += 8
            return n

        def f64s(n):
            nonlocal pos
            a = np.frombuffer(buf, "<f8", n, pos).copy()
            pos += 8 * n
            return a

        def f32s(n):
            nonlocal pos
            a = np.frombuffer(buf, "<f4", n, pos).copy()
            pos += 4 * n
            return a

        def name():
            nonlocal pos
            n = count()
            s = buf[pos:pos + n].decode()
            pos += n
            return s

        lines = [f64s(count()) for _ in range(3)]
        ts = f64s(count())
        fr = f64s(count())
        r = cls(os.fspath(path), lines, mesh_type, ts, fr)
        if pos == len(buf):  # header only
            return r
        for _ in range(count()):
            k = name()
            r.scalar_fields[k] = f32s(count())
        for _ in range(count()):
            k = name()
            r.vector_fields[k] = tuple(f32s(count()) for _ in range(3))
        for _ in range(count()):
            k = name()
            a = f64s(2 * count())
            r.complex_fields[k] = a[0::2] + 1j * a[1::2]
        return r

    def is_valid(self) -> bool:
        return all(len(v) > 0 for v in self.mesh_lines)

    def dimensions(self) -> Tuple[int, int, int]:
        return tuple(max(len(v) - 1, 1) for v in self.mesh_lines)


# ---------------------------------------------------------------------------
# legacy VTK (ASCII)
# ---------------------------------------------------------------------------


def rust_float(x, dtype=np.float64) -> str:
    """A float as Rust's `{}` prints it: the shortest digits that round-trip
    in its own precision, positional notation."""
    return np.format_float_positional(dtype(x), unique=True, trim="-")


def _vtk_header(f, title: str, lines: Sequence[np.ndarray]):
    nx, ny, nz = (len(v) - 1 for v in lines)
    f.write("# vtk DataFile Version 3.0\n")
    f.write(f"{title}\n")
    f.write("ASCII\n")
    f.write("DATASET RECTILINEAR_GRID\n")
    f.write(f"DIMENSIONS {nx + 1} {ny + 1} {nz + 1}\n")
    for axis, v in zip("XYZ", lines):
        f.write(f"{axis}_COORDINATES {len(v)} float\n")
        f.write("".join(rust_float(x) + " " for x in v) + "\n")
    f.write(f"CELL_DATA {nx * ny * nz}\n")


def write_field_vtk(path, data: np.ndarray, lines: Sequence[Sequence[float]], field_name: str):
    """write_field_vtk (src/io/vtk.rs:10-56): data (nx, ny, nz), f32 values,
    i outermost, k innermost."""
    lines = [np.asarray(v, dtype=np.float64) for v in lines]
    d = np.asarray(data, dtype=np.float32)
    with open(path, "w") as f:
        _vtk_header(f, "openEMS field data", lines)
        f.write(f"SCALARS {field_name} float 1\n")
        f.write("LOOKUP_TABLE default\n")
        f.write("".join(rust_float(v, np.float32) + "\n" for v in d.ravel()))


def write_vector_field_vtk(path, components, lines: Sequence[Sequence[float]], field_name: str):
    """write_vector_field_vtk (src/io/vtk.rs:58-126): three (nx, ny, nz)
    f32 components, one 'x y z' line per cell."""
    lines = [np.asarray(v, dtype=np.float64) for v in lines]
    x, y, z = (np.asarray(c, dtype=np.float32).ravel() for c in components)
    with open(path, "w") as f:
        _vtk_header(f, "openEMS vector field data", lines)
        f.write(f"VECTORS {field_name} float\n")
        f.write("".join(f"{rust_float(a, np.float32)} {rust_float(b, np.float32)} {rust_float(c, np.float32)}\n"
                        for a, b, c in zip(x, y, z)))


# ---------------------------------------------------------------------------
# from an engine
# ---------------------------------------------------------------------------


def dump_fields(engine, grid, path, fmt: str = "oems", timestep: Optional[float] = None):
    """E and H of an engine (read back from its device buffers) as vector
    fields "E-Field" / "H-Field": fmt "oems" writes the binary container
    (with the time of the snapshot when given), "vtk" two VTK files
    `path` + "_E.vtk" / "_H.vtk"."""
    e, h = engine.read_fields()
    lines = [np.asarray(v, dtype=np.float64) * grid.unit for v in (grid.x_lines, grid.y_lines, grid.z_lines)]
    if fmt == "vtk":
        write_vector_field_vtk(os.fspath(path) + "_E.vtk", e, lines, "E-Field")
        write_vector_field_vtk(os.fspath(path) + "_H.vtk", h, lines, "H-Field")
        return
    w = Hdf5Writer(path)
    w.write_rect_mesh(lines, CARTESIAN)
    if timestep is not None:
        w.set_timesteps([timestep])
    w.write_vector_field("E-Field", e)
    w.write_vector_field("H-Field", h)
    w.close()


def dump_field_dft(engine, dump_id: int, freqs: Sequence[float], components: Sequence[int], path, lines=None):
    """A frequency-domain field dump of an engine (oems_engine_read_field_dft
    per frequency and component) as complex fields "<component>_f<index>"
    in the binary container, with the frequencies."""
    names = ("Ex", "Ey", "Ez", "Hx", "Hy", "Hz")
    w = Hdf5Writer(path)
    if lines is not None:
        w.write_rect_mesh(lines, CARTESIAN)
    w.set_frequencies(freqs)
    for fi in range(len(freqs)):
        for c in components:
            w.write_complex_field(f"{names[c]}_f{fi}", engine.field_dft(dump_id, fi, c))
    w.close()
