"""An openEMS XML configuration run on the engine equals the oracle run of the
same operator, CPML and sources (bit for bit)."""
import numpy as np
import pytest

import oracle
from openems_b200 import xml_config as X
from test_xml_config import PATCH

pytestmark = pytest.mark.gpu


def test_xml_run_matches_oracle():
    xml = PATCH.replace('<BoundaryCond xmin="PML_6" xmax="PML_6" ymin="3" ymax="2" zmin="PEC" zmax="0"/>',
                        '<BoundaryCond xmin="PML_6" xmax="PML_6" ymin="PML_4" ymax="PML_4" zmin="PEC" '
                        'zmax="PML_3"/>')
    cfg = X.parse_config(xml)
    r = X.run(cfg)
    assert r["timesteps"] == 300 and r["sources"] == 2
    e, h = r["engine"].read_fields()
    b = X.build(cfg)
    op = b.operator
    s = oracle.OracleSim(*op.dimensions(), op.timestep(), op.cell_size())
    s.set_coefficients(op.coefficients())
    s.enable_cpml(b.boundaries.cpml_layers())
    for pos, comp, w in b.sources:
        x = X.waveform(cfg, pos, comp, w)
        s.add_excitation_analytic(x.position, x.direction, x.soft_source, int(x.excitation_type), list(x.params),
                                  x.amplitude, 0, 300)
    s.run_batch(300)
    ref = s.fields()
    got = np.concatenate([e, h])
    assert np.abs(ref).max() > 0
    assert np.array_equal(got, ref), np.abs(got - ref).max()
