"""The binary field container and legacy VTK writers (src/io/hdf5.rs,
src/io/vtk.rs) on CPU: byte layout, the reference's round-trip test, and
Rust's float printing."""
import struct

import numpy as np
import pytest

from openems_b200 import field_io as F


def test_binary_layout_known_answer(tmp_path):
    """The exact bytes of the reference's write_binary for a mesh, one
    scalar, one vector and one complex field (attributes are not written)."""
    p = tmp_path / "a.oems"
    w = F.Hdf5Writer(p)
    w.write_rect_mesh([[0.0, 1e-3], [0.0], [0.0, 2e-3, 5e-3]], F.CARTESIAN)
    w.write_scalar_field("s", [1.5, -2.0])
    w.write_vector_field("v", ([1.0], [2.0], [3.0]))
    w.write_complex_field("c", [1 + 2j])
    w.write_attribute("ignored", [7.0])
    w.close()
    Q, d, f = (lambda n: struct.pack("<Q", n)), (lambda *v: struct.pack(f"<{len(v)}d", *v)), \
        (lambda *v: struct.pack(f"<{len(v)}f", *v))
    want = (b"OEMS" + bytes([1, 0, 0, 0]) + struct.pack("<i", 0)
            + Q(2) + d(0.0, 1e-3) + Q(1) + d(0.0) + Q(3) + d(0.0, 2e-3, 5e-3)
            + Q(0) + Q(0)
            + Q(1) + Q(1) + b"s" + Q(2) + f(1.5, -2.0)
            + Q(1) + Q(1) + b"v" + Q(1) + f(1.0) + Q(1) + f(2.0) + Q(1) + f(3.0)
            + Q(1) + Q(1) + b"c" + Q(1) + d(1.0, 2.0))
    assert p.read_bytes() == want


def test_binary_roundtrip(tmp_path):
    """test_binary_roundtrip (src/io/hdf5.rs:475-497), plus the fields back."""
    p = tmp_path / "test.oems"
    w = F.Hdf5Writer(p)
    assert w.current_group == "/"
    w.write_rect_mesh([[0.0, 0.001, 0.002]] * 3, F.CARTESIAN)
    w.write_scalar_field("test_field", [1.0, 2.0, 3.0, 4.0])
    w.write_complex_field("z", np.array([1 - 1j, 0.5j]))
    w.set_frequencies([1e9, 2e9])
    w.close()
    r = F.Hdf5Reader.open(p)
    assert r.is_valid() and r.mesh_type == F.CARTESIAN and len(r.mesh_lines[0]) == 3
    assert r.dimensions() == (2, 2, 2)
    assert list(r.frequencies) == [1e9, 2e9] and len(r.timesteps) == 0
    assert list(r.scalar_fields["test_field"]) == [1.0, 2.0, 3.0, 4.0]
    assert np.array_equal(r.complex_fields["z"], [1 - 1j, 0.5j])
    assert [F.mesh_type_from(v) for v in (0, 1, 99)] == [F.CARTESIAN, F.CYLINDRICAL, F.CARTESIAN]
    (tmp_path / "bad").write_bytes(b"HDF5....")
    with pytest.raises(ValueError):
        F.Hdf5Reader.open(tmp_path / "bad")


def test_rust_float_printing():
    """Rust's {}: shortest round-trip digits, never an exponent."""
    assert [F.rust_float(v) for v in (0.0, 1.0, -2.5, 1e-7, 0.001, 1e21)] == \
        ["0", "1", "-2.5", "0.0000001", "0.001", "1000000000000000000000"]
    assert F.rust_float(0.1, np.float32) == "0.1"
    assert F.rust_float(np.float32(1) / 3, np.float32) == "0.33333334"


def test_vtk_scalar_and_vector_text(tmp_path):
    lines = [[0.0, 0.001, 0.002], [0.0, 0.5], [0.0, 1e-7]]
    data = np.array([[[0.25]], [[-1.0]]], dtype=np.float32)
    p = tmp_path / "s.vtk"
    F.write_field_vtk(p, data, lines, "Ez")
    assert p.read_text() == ("# vtk DataFile Version 3.0\nopenEMS field data\nASCII\nDATASET RECTILINEAR_GRID\n"
                             "DIMENSIONS 3 2 2\nX_COORDINATES 3 float\n0 0.001 0.002 \nY_COORDINATES 2 float\n"
                             "0 0.5 \nZ_COORDINATES 2 float\n0 0.0000001 \nCELL_DATA 2\nSCALARS Ez float 1\n"
                             "LOOKUP_TABLE default\n0.25\n-1\n")
    q = tmp_path / "v.vtk"
    F.write_vector_field_vtk(q, (data, 2 * data, np.zeros_like(data)), lines, "E-Field")
    text = q.read_text()
    assert text.startswith("# vtk DataFile Version 3.0\nopenEMS vector field data\n")
    assert text.endswith("CELL_DATA 2\nVECTORS E-Field float\n0.25 0.5 0\n-1 -2 0\n")
