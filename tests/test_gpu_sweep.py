"""Batched port sweep (oems_sweep): concurrency does not change results, each
instance equals a direct engine run with a LumpedPort, and one instance
matches the oracle."""
import numpy as np
import pytest

import oracle
import openems_b200 as oe
from openems_b200 import workloads as W
from openems_b200.sweep import Sweep

pytestmark = pytest.mark.gpu

FREQS = np.linspace(0.5e9, 12e9, 47)


def mini_specs():
    out = []
    for dims, eps, h, w, l, frac in [((34, 38, 30), 4.4, 2, 14, 12, 0.3),
                                     ((40, 33, 28), 2.2, 3, 16, 10, 0.5),
                                     ((30, 30, 32), 9.8, 4, 10, 12, 0.6),
                                     ((45, 36, 26), 6.0, 2, 20, 16, 0.2)]:
        x0, y0 = (dims[0] - w) // 2, (dims[1] - l) // 2
        fx, fy = x0 + w // 2, y0 + l // 2 - int(round(frac * (l // 2)))
        out.append(W.PatchSpec(dims, eps, h, w, l, x0, y0, fx, fy, k_ground=8, layers=6))
    return out


def instances():
    return [W.patch_sweep_instance(s, delta=0.5e-3, decay_db=50.0, max_steps=20000, fmax=12e9)
            for s in mini_specs()]


def run_sweep(concurrency):
    sw = Sweep(FREQS, concurrency=concurrency)
    ids = [sw.add(i) for i in instances()]
    sw.run(batch_steps=700)
    return sw, [sw.result(i) for i in ids]


def test_concurrency_does_not_change_results():
    _, a = run_sweep(1)
    _, b = run_sweep(3)
    for ra, rb in zip(a, b):
        assert ra["timesteps"] == rb["timesteps"]
        assert np.array_equal(ra["uf"], rb["uf"]) and np.array_equal(ra["if"], rb["if"])


def test_sweep_matches_direct_engine_and_is_passive():
    sw, res = run_sweep(2)
    wall, cell_steps = sw.stats()
    assert wall > 0 and cell_steps == sum(r["cells"] * r["timesteps"] for r in res)
    for inst, r in zip(instances(), res):
        assert r["termination_reason"] == 1  # decayed by 50 dB
        # passive; the DFT of a run cut at -50 dB carries ~1e-3 truncation error
        assert np.all(np.abs(r["s11"]) <= 1.0 + 5e-3)
        # the same instance through the Python API, one engine
        op = inst.operator
        port = oe.LumpedPort(1, inst.port_resistance, inst.port_position, inst.port_direction,
                             excite=1.0, eps_r=inst.port_eps_r).apply(op)
        eng = oe.Engine(op, autotune=False, kernels="register")
        eng.add_cpml(inst.cpml)
        port.add_probes(eng, FREQS)
        exc = port.excitation(inst.waveform)
        dt, start = op.timestep(), 0
        while start < r["timesteps"]:
            n = min(700, r["timesteps"] - start)
            eng.run_batch(oe.EngineBatch(
                num_steps=n, excitations=[oe.ScheduledExcitation.from_excitation(exc, start, n, dt)]))
            start += n
        port.calc_port(eng)
        assert np.array_equal(port.uf_tot, r["uf"]) and np.array_equal(port.if_tot, r["if"])
        assert np.allclose(port.s11(), r["s11"], rtol=1e-12, atol=1e-14)


def test_sweep_instance_matches_oracle():
    sw, res = run_sweep(1)
    inst, r, spec = instances()[1], res[1], mini_specs()[1]
    lines = [oracle.uniform_lines(n, 0.5e-3) for n in spec.dims]
    dt, delta = oracle.grid_timestep(*lines)
    s = oracle.OracleSim(*spec.dims, dt, delta, threads=4)
    nx, ny, nz = spec.dims
    lo, kg, kp = spec.layers, spec.k_ground, spec.k_patch
    s.set_material(spec.eps_r, 1.0, 0.0, 0.0, (0, nx, 0, ny, kg + 1, kp))
    s.set_pec((0, nx, 0, ny, kg, kg + 1))
    s.set_pec((spec.x0, spec.x0 + spec.W, spec.y0, spec.y0 + spec.L, kp, kp + 1))
    s.set_pec((spec.fx, spec.fx + 1, spec.fy, spec.fy + 1, kg + 2, kp))
    scale = s.set_lumped(inst.port_position, 2, 50.0, 0.0, spec.eps_r, 0.0)
    s.enable_cpml((lo,) * 6)
    op = inst.operator
    ids = []
    for kind in (0, 1):
        t = oe.port_probe(op, inst.port_position, 2, kind)
        ids.append(s.add_probe_dft(s.add_probe([(c, q, -w) for c, q, w in t.terms], t.mode), FREQS))
    w = inst.waveform
    s.add_excitation_analytic(inst.port_position, 2, True, int(w.excitation_type), list(w.params),
                              w.amplitude * scale, 0, r["timesteps"])
    s.run_batch(r["timesteps"])
    for d, key in zip(ids, ("uf", "if")):
        ref = s.probe_dft(d)
        assert np.abs(r[key] - ref).max() <= 1e-12 * np.abs(ref).max()


def test_paused_instances_continue_bit_for_bit():
    """run_until stops every instance at the cap and keeps its engine; the
    continued runs equal uninterrupted ones, the paused results equal runs
    capped at the same step count, and finish() ends an instance there."""
    _, full = run_sweep(2)
    sw = Sweep(FREQS, concurrency=2)
    sw.set_trace_steps(1500)
    ids = [sw.add(i) for i in instances()]
    sw.run_until(1000, batch_steps=700)
    part = [sw.result(i) for i in ids]
    for r in part:
        assert r["paused"] and r["timesteps"] == 1000
    # the same instances run to 1000 steps only
    capped = Sweep(FREQS, concurrency=2)
    cids = [capped.add(W.patch_sweep_instance(s, delta=0.5e-3, decay_db=0.0, max_steps=1000, fmax=12e9))
            for s in mini_specs()]
    capped.run(batch_steps=700)
    for p, c in zip(part, (capped.result(i) for i in cids)):
        assert not c["paused"]
        assert np.array_equal(p["uf"], c["uf"]) and np.array_equal(p["if"], c["if"])
    sw.finish(ids[0])
    sw.run_until(1600, batch_steps=700)
    assert sw.result(ids[0])["timesteps"] == 1000 and not sw.result(ids[0])["paused"]
    assert all(sw.result(i)["timesteps"] == 1600 for i in ids[1:])
    sw.run(batch_steps=700)
    for i, f in zip(ids[1:], full[1:]):
        r = sw.result(i)
        assert not r["paused"] and r["timesteps"] == f["timesteps"]
        assert np.array_equal(r["uf"], f["uf"]) and np.array_equal(r["if"], f["if"])
        assert sw.trace(i).shape == (1500, 2)


def test_advance_from_threads_matches_sweep_run():
    """Instances advanced one by one from several threads (through stages,
    then to their end) give the bits of the batched run."""
    import threading
    _, full = run_sweep(2)
    sw = Sweep(FREQS, concurrency=2)
    ids = [sw.add(i) for i in instances()]

    def drive(mine):
        for i in mine:
            for cap in (700, 1400):
                sw.advance(i, cap, batch_steps=700)
                assert sw.result(i)["timesteps"] == cap and sw.result(i)["paused"]
            sw.advance(i, 10 ** 9, batch_steps=700)

    ts = [threading.Thread(target=drive, args=(ids[k::2],)) for k in range(2)]
    for t in ts:
        t.start()
    for t in ts:
        t.join()
    for i, f in zip(ids, full):
        r = sw.result(i)
        assert not r["paused"] and r["timesteps"] == f["timesteps"]
        assert np.array_equal(r["uf"], f["uf"]) and np.array_equal(r["if"], f["if"])


@pytest.mark.parametrize("check,tau", [("mean", 0.15), ("max", 0.05)])
def test_staged_early_stop_against_full_runs(check, tau):
    """The staged early stop on the small patches: a predicted instance stops
    at a stage with its S11 within 0.5 dB of the full run's (mean over the
    band, clipped at -30 dB); a decayed or fallback instance carries the full
    run's bits."""
    from openems_b200 import early_stop as E
    full = E.full_sweep(instances(), FREQS, concurrency=2, batch_steps=700)
    plan = E.StagePlan(stages=(1024, 2048, 4096), check=check, tau=tau)
    st = E.staged_sweep(instances(), FREQS, plan, concurrency=2, batch_steps=700)
    band = plan.band(FREQS)
    for r, f in zip(st["results"], full["results"]):
        if r["how"] == "predicted":
            assert r["steps"] in plan.stages and r["steps"] < f["timesteps"]
            assert E.s11_db_mean_error(r["s11"], f["s11"], band) < 0.5
        else:
            assert r["steps"] == f["timesteps"]
            assert np.array_equal(r["s11"], f["s11"])


def test_command_line_matches_direct_sweep(tmp_path, capsys):
    """`python -m openems_b200.sweep` on one rank: the whole share, in instance
    order, equal to a direct Sweep of the same seeded instances."""
    import json

    from openems_b200 import sweep as S
    out = tmp_path / "s11.npz"
    S.main(["--count", "3", "--freqs", "41", "--max-steps", "3000", "--batch-steps", "1000", "--out", str(out)])
    line = json.loads(capsys.readouterr().out.strip().splitlines()[-1])
    assert line["ranks"] == 1 and line["instances"] == 3 and line["cell_steps"] > 0
    got = np.load(out)
    sw = Sweep(np.linspace(0.0, 8e9, 41), concurrency=2)
    ids = [sw.add(W.patch_sweep_instance(s, decay_db=50.0, max_steps=3000)) for s in W.patch_specs(3, seed=4)]
    sw.run(1000)
    want = [sw.result(i) for i in ids]
    assert np.array_equal(got["timesteps"], [r["timesteps"] for r in want])
    assert np.array_equal(got["s11"], np.array([r["s11"] for r in want]))
