"""openEMS XML configuration ingestion (host side): the reference's
parse_config semantics (src/io/xml.rs:95-221) and the openEMS grid /
property boxes mapped onto cells."""
import json

import numpy as np
import pytest

import openems_b200 as oe
from openems_b200 import xml_config as X

PATCH = """<?xml version="1.0"?>
<openEMS>
  <FDTD NumberOfTimesteps="300" endCriteria="1e-5" f0="0" fc="20e9">
    <Excitation Type="0" f0="0" fc="20e9"/>
    <BoundaryCond xmin="PML_6" xmax="PML_6" ymin="3" ymax="2" zmin="PEC" zmax="0"/>
  </FDTD>
  <ContinuousStructure CoordSystem="0">
    <Properties>
      <Material Name="substrate">
        <Property Epsilon="4.0" Kappa="0.01" Mue="1" Sigma="0"/>
        <Primitives><Box Priority="0"><P1 X="2" Y="2" Z="0"/><P2 X="14" Y="10" Z="3"/></Box></Primitives>
      </Material>
      <Metal Name="patch">
        <Primitives><Box Priority="10"><P1 X="5" Y="4" Z="3"/><P2 X="11" Y="8" Z="3"/></Box></Primitives>
      </Metal>
      <Excitation Name="feed" Type="0" Excite="0,0,1">
        <Primitives><Box Priority="5"><P1 X="8" Y="6" Z="0"/><P2 X="8" Y="6" Z="2"/></Box></Primitives>
      </Excitation>
    </Properties>
    <RectilinearGrid DeltaUnit="0.001" CoordSystem="0">
      <XLines>0,1,2,3,4,5,6,7,8,9,10,11,12,13,14,15,16</XLines>
      <YLines>0,1,2,3,4,5,6,7,8,9,10,11,12</YLines>
      <ZLines>0,1,2,3,4,5,6,7,8</ZLines>
    </RectilinearGrid>
  </ContinuousStructure>
</openEMS>
"""


def test_reference_fields_and_defaults():
    """FDTD attributes and BoundaryCond codes as src/io/xml.rs:95-183 reads
    them: unparsable timesteps give 10000, unparsable codes 0 (PEC)."""
    c = X.parse_config('<openEMS><FDTD NumberOfTimesteps="1234" endCriteria="1e-4" f0="1e9" fc="2e9">'
                       '<BoundaryCond xmin="0" xmax="1" ymin="2" ymax="3" zmin="4" zmax="x"/></FDTD></openEMS>')
    assert (c.num_timesteps, c.end_criteria, c.f0, c.fc) == (1234, 1e-4, 1e9, 2e9)
    assert c.boundaries == [0, 1, 2, 3, 4, 0]
    assert [X.boundary_from_code(v).kind for v in range(6)] == ["pec", "pmc", "mur", "pml", "periodic", "pec"]
    assert X.boundary_from_code(3).layers == 8
    d = X.parse_config('<openEMS><FDTD NumberOfTimesteps="1e4"/></openEMS>')
    assert d.num_timesteps == 10000 and d.end_criteria is None and d.boundaries == [0] * 6
    e = X.parse_config("<openEMS/>")
    assert e.num_timesteps == 0 and e.grid is None and e.properties == []
    with pytest.raises(oe.ConfigError):
        X.parse_config("<openEMS><FDTD></openEMS>")


def test_openems_names_grid_and_end_criteria():
    c = X.parse_config(PATCH)
    assert c.boundaries == [3, 3, 3, 2, 0, 0] and c.pml_layers[:2] == [6, 6] and c.pml_layers[2] == 8
    assert c.end_criteria_db == pytest.approx(50.0)
    assert len(c.grid.x_lines) == 17 and c.grid.unit == 1e-3
    assert [p.kind for p in c.properties] == ["Material", "Metal", "Excitation"]
    assert c.properties[0].eps_r == 4.0 and c.properties[0].sigma_e == 0.01
    assert c.properties[2].excite == (0.0, 0.0, 1.0)


def test_boxes_mapped_onto_cells():
    c = X.parse_config(PATCH)
    b = X.build(c)
    op = b.operator
    assert op.dimensions() == (16, 12, 8)
    co = op.coefficients()
    ca, cb = co[0:3], co[3:6]
    free = cb[0, 0, 0, 7]
    # substrate: cells with centres in [2, 14] x [2, 10] x [0, 3] mm (lossy eps 4)
    assert cb[0, 3, 3, 1] != free and 0 < ca[0, 3, 3, 1] < 1
    assert cb[0, 1, 3, 1] == free and cb[0, 3, 3, 3] == free
    # patch: a zero-thickness sheet at z = 3 mm is one cell (k = 3) thick, x 5..11, y 4..8
    assert np.all(ca[:, 5:11, 4:8, 3] == 0) and np.all(cb[:, 5:11, 4:8, 3] == 0)
    assert cb[0, 5, 4, 4] != 0 and cb[0, 4, 4, 3] != 0
    # feed: Ez soft sources on the cells of the line x = 8, y = 6, z 0..2
    assert sorted(b.sources) == [((8, 6, 0), 2, 1.0), ((8, 6, 1), 2, 1.0)]
    assert b.mur_faces == (False, False, False, True, False, False)
    assert b.boundaries.cpml_layers() == (6, 6, 8, 0, 0, 0)


def test_command_line_without_simulation(tmp_path, capsys):
    f = tmp_path / "patch.xml"
    f.write_text(PATCH)
    X.main([str(f), "--no-simulation"])
    out = json.loads(capsys.readouterr().out)
    assert out["dims"] == [16, 12, 8] and out["sources"] == 2 and out["boundaries"] == [3, 3, 3, 2, 0, 0]


def test_command_line_accepts_the_reference_flags(tmp_path, capsys):
    """The reference's flags (src/main.rs:15-53) parse; the engine names of
    its CPU engines run on the GPU engine, and the debug / thread flags
    change nothing (as in the reference)."""
    f = tmp_path / "patch.xml"
    f.write_text(PATCH)
    X.main([str(f), "--no-simulation", "--engine", "parallel", "--num-threads", "4", "--disable-dumps",
            "--debug-material", "--debug-operator", "-v", "0", "--dump-statistics"])
    out = json.loads(capsys.readouterr().out)
    assert out["dims"] == [16, 12, 8]
    assert not (tmp_path / "patch.stats.json").exists()  # no run, no statistics
    with pytest.raises(SystemExit):
        X.main([str(tmp_path / "missing.xml"), "--no-simulation"])


def test_debug_dumps(tmp_path):
    """--debug-material: one cell value per material (vacuum, substrate,
    PEC sheet); --debug-operator: the coefficients as VTK vector fields."""
    from openems_b200.field_io import write_field_vtk
    f = tmp_path / "patch.xml"
    f.write_text(PATCH)
    X.main([str(f), "--no-simulation", "--debug-material", "--debug-operator"])
    mat = (tmp_path / "patch.material.vtk").read_text().splitlines()
    n = mat.index("LOOKUP_TABLE default")
    vals = np.array([float(v) for v in mat[n + 1:]])
    assert len(vals) == 16 * 12 * 8 and set(np.unique(vals)) >= {0.0, 1.0, 2.0}
    op = X.build(X.parse_config(str(f))).operator
    ids, table = oe.compress_coefficients(op.coefficients())
    assert np.array_equal(vals.reshape(16, 12, 8), ids.astype(np.float64))
    # the same writer gives the same bytes
    g = op.grid
    lines = [np.asarray(v) * g.unit for v in (g.x_lines, g.y_lines, g.z_lines)]
    write_field_vtk(tmp_path / "again.vtk", ids.astype(np.float32), lines, "material")
    assert (tmp_path / "again.vtk").read_text() == (tmp_path / "patch.material.vtk").read_text()
    for name in ("ca", "cb", "da", "db"):
        txt = (tmp_path / f"patch.{name}.vtk").read_text()
        assert f"VECTORS {name.capitalize()} float" in txt and txt.count("\n") > 16 * 12 * 8


def test_waveform_of_the_fdtd_excitation():
    """Type 0 with centre f0 and cutoff fc: a pulse without carrier (tau =
    1 / (pi fc), t0 = 4 tau) for f0 = 0, else modulated at f0 with the same
    tau; fc = 0 is refused rather than giving an infinite tau."""
    import math
    c = X.parse_config(PATCH)
    w = X.waveform(c, (8, 6, 0), 2, 2.0)
    tau = 1 / (math.pi * 20e9)
    assert w.excitation_type == oe.ExcitationType.Gaussian and w.params == pytest.approx((4 * tau, tau))
    assert w.amplitude == 2.0 and w.direction == 2 and w.soft_source
    c.f0 = 5e9
    m = X.waveform(c, (8, 6, 0), 2, 1.0)
    assert m.excitation_type == oe.ExcitationType.GaussianModulated
    assert m.params[0] == 5e9 and m.params[2] == pytest.approx(tau)
    c.fc = 0.0
    with pytest.raises(oe.ConfigError):
        X.waveform(c, (8, 6, 0), 2, 1.0)
