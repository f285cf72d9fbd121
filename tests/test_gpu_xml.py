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


def test_reference_python_surface_cavity_matches_oracle():
    """The reference's benchmark driver's cavity (python/gpu_benchmark.py:
    uniform grid, PEC walls, add_gauss_excite(2e9, 1e9) at the centre)
    through the mirrored module: steps, and final energy against the
    oracle's run of the same source."""
    from openems_b200 import openems_rust as ems
    n, steps = 24, 120
    sim = ems.OpenEMS(num_timesteps=steps)
    sim.set_grid(ems.Grid.uniform(n, n, n, 0.1 / n))
    sim.set_engine_type("gpu")
    sim.set_boundary_cond(["pec"] * 6)
    sim.add_gauss_excite(2e9, 1e9, direction=2, position=(n // 2,) * 3)
    sim.set_verbose(0)
    sim.set_show_progress(False)
    st = sim.run()
    assert st.timesteps == steps and st.speed_mcells_per_sec > 0
    lines = [oracle.uniform_lines(n, 0.1 / n) for _ in range(3)]
    dt, d3 = oracle.grid_timestep(*lines)
    s = oracle.OracleSim(n, n, n, dt, d3)
    x = sim._excitation(sim.excitations[0], (n, n, n))
    s.add_excitation_analytic(x.position, x.direction, x.soft_source, int(x.excitation_type), list(x.params),
                              x.amplitude, 0, steps)
    s.run_batch(steps)
    e, h = s.energy()
    assert st.final_energy == pytest.approx(e + h, rel=1e-10)
    # peak over the energy samples (every 100 steps): the source is still
    # feeding the cavity at step 120, so the final energy can exceed it
    assert st.peak_energy > 0


def test_command_line_dumps_statistics(tmp_path, capsys):
    """--dump-statistics writes FILE.stats.json with the reference's keys
    (src/main.rs:163-172) after the run."""
    import json
    from openems_b200 import xml_config as X
    from test_xml_config import PATCH
    f = tmp_path / "patch.xml"
    f.write_text(PATCH)
    X.main([str(f), "--dump-statistics", "--batch", "200"])
    out = json.loads(capsys.readouterr().out.strip().splitlines()[-1])
    st = json.loads((tmp_path / "patch.stats.json").read_text())
    assert set(st) == {"timesteps", "sim_time", "wall_time", "peak_energy", "final_energy", "speed_mcells_per_sec"}
    assert st["timesteps"] == out["timesteps"] > 0 and st["speed_mcells_per_sec"] > 0
    assert st["sim_time"] > 0 and st["peak_energy"] >= st["final_energy"] >= 0
