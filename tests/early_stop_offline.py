"""Offline evaluation of staged early termination on oracle traces (CPU).

Runs seeded patches of the small family (openems_b200.predictor.family_specs)
to -50 dB energy decay on the oracle, built exactly as the GPU sweep builds
them (test_gpu_sweep.py::test_sweep_instance_matches_oracle), and keeps
their port traces, energy samples and full-run S11.  It then replays a
StagePlan's decisions instance by instance as staged_sweep would.  At each
stage the engine's port DFTs of the first K steps are rebuilt from the
trace, and check_instance runs on them.  The result is the step ratio
against the plain runs and every stopped instance's S11 error.

    python tests/early_stop_offline.py --seed 50 --count 80 [--cache DIR]

prints the standard and the dense plan side by side.  The step ratio is an
upper bound on the sweep's instances/hour ratio: the GPU sweep also pays for
pauses and host checks.
"""
from __future__ import annotations

import argparse
import json
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

import oracle  # noqa: E402
import openems_b200 as oe  # noqa: E402
from openems_b200 import early_stop as ES  # noqa: E402
from openems_b200 import predictor as P  # noqa: E402
from openems_b200 import workloads as W  # noqa: E402


def run_instance(spec, threads: int = 8) -> dict:
    """Full oracle run of one small-family patch: trace (steps, 2) of port
    u, i; energy samples (timestep, e, h, total) every 100 steps; S11."""
    inst = W.patch_sweep_instance(spec, delta=0.5e-3, decay_db=50.0, max_steps=P.HORIZON, fmax=12e9)
    lines = [oracle.uniform_lines(n, 0.5e-3) for n in spec.dims]
    dt, delta = oracle.grid_timestep(*lines)
    s = oracle.OracleSim(*spec.dims, dt, delta, threads=threads)
    nx, ny, nz = spec.dims
    kg, kp = spec.k_ground, spec.k_patch
    s.set_material(spec.eps_r, 1.0, 0.0, 0.0, (0, nx, 0, ny, kg + 1, kp))
    s.set_pec((0, nx, 0, ny, kg, kg + 1))
    s.set_pec((spec.x0, spec.x0 + spec.W, spec.y0, spec.y0 + spec.L, kp, kp + 1))
    if kp > kg + 2:
        s.set_pec((spec.fx, spec.fx + 1, spec.fy, spec.fy + 1, kg + 2, kp))
    scale = s.set_lumped(inst.port_position, 2, 50.0, 0.0, spec.eps_r, 0.0)
    s.enable_cpml((spec.layers,) * 6)
    for kind in (0, 1):
        t = oe.port_probe(inst.operator, inst.port_position, 2, kind)
        s.add_probe([(c, q, -w) for c, q, w in t.terms], t.mode)
    w = inst.waveform
    s.add_excitation_analytic(inst.port_position, 2, True, int(w.excitation_type), list(w.params),
                              w.amplitude * scale, 0, P.HORIZON)
    r = s.run_batch(P.HORIZON, sample_interval=100, track_peak=True, check_interval=100, energy_decay_db=50.0)
    tr = s.probe_traces()[:, :2].copy()
    uf = P.head_dft(tr[:, 0], 1, dt, P.FREQS, 0.0)
    if_ = P.head_dft(tr[:, 1], 1, dt, P.FREQS, 0.5)
    return {"trace": tr, "energy": np.array(r["energy_samples"], dtype=np.float64).reshape(-1, 4),
            "s11": P.s11(uf, if_, 50.0), "steps": int(r["timesteps_executed"]), "dt": dt}


def level_db(rec: dict, K: int) -> float:
    """The paused instance's energy level at K: its last sample against the
    peak so far (what the sweep reports as final_decay_db)."""
    en = rec["energy"]
    m = en[:, 0] <= K
    if not m.any():
        return 0.0
    tot = en[m, 3]
    return float(10 * np.log10(tot[-1] / tot.max())) if tot.max() > 0 and tot[-1] > 0 else 0.0


def replay(records, plan: ES.StagePlan, limit_db: float = 0.5) -> dict:
    """staged_sweep's decisions on recorded runs: per instance the steps it
    runs and, if stopped early, its largest S11 error over the band."""
    band = plan.band(P.FREQS)
    steps, errors, how = [], [], []
    for rec in records:
        tr, dt, full = rec["trace"], rec["dt"], rec["steps"]
        used, err, h = full, 0.0, "full"
        for K in plan.stages:
            if full <= K:
                h = "decayed"
                break
            r = {"uf": P.head_dft(tr[:K, 0], 1, dt, P.FREQS, 0.0), "if": P.head_dft(tr[:K, 1], 1, dt, P.FREQS, 0.5),
                 "final_decay_db": level_db(rec, K)}
            pred, d, _ = ES.check_instance(tr, r, K, dt, P.FREQS, P.HORIZON, 50.0, plan)
            if d < plan.tau:
                used, err, h = K, ES.s11_db_error(pred, rec["s11"], band), "predicted"
                break
        steps.append(used)
        errors.append(err)
        how.append(h)
    full = np.array([r["steps"] for r in records], dtype=np.float64)
    errors = np.array(errors)
    return {"step_ratio": float(full.mean() / np.mean(steps)), "predicted": how.count("predicted"),
            "decayed": how.count("decayed"), "full": how.count("full"), "max_err_db": float(errors.max()),
            f"over_{limit_db}db": int((errors > limit_db).sum()), "steps": steps, "errors": errors.tolist()}


def load_or_run(seed: int, count: int, cache: str = None, threads: int = 8):
    specs = P.family_specs(count, seed)
    out = []
    for n, spec in enumerate(specs):
        path = os.path.join(cache, f"s{seed}_{n:04d}.npz") if cache else None
        if path and os.path.exists(path):
            z = np.load(path)
            out.append({"trace": z["trace"], "energy": z["energy"], "s11": z["s11"], "steps": int(z["steps"]),
                        "dt": float(z["dt"])})
            continue
        rec = run_instance(spec, threads)
        if path:
            os.makedirs(cache, exist_ok=True)
            np.savez(path, **rec)
        out.append(rec)
    return out


def main(argv=None):
    ap = argparse.ArgumentParser(description=__doc__.split("\n\n")[0])
    ap.add_argument("--seed", type=int, default=50)
    ap.add_argument("--count", type=int, default=80)
    ap.add_argument("--cache", default=None, help="keep the oracle runs here (npz per instance)")
    ap.add_argument("--threads", type=int, default=8)
    a = ap.parse_args(argv)
    from threadpoolctl import threadpool_limits
    records = load_or_run(a.seed, a.count, a.cache, a.threads)
    with threadpool_limits(a.threads):
        for name, plan in (("standard (tau 0.05)", ES.StagePlan(tau=0.05)), ("dense", ES.StagePlan.dense())):
            r = replay(records, plan)
            r.pop("steps"), r.pop("errors")
            print(json.dumps({"plan": name, "seed": a.seed, "count": len(records),
                              "full_steps_mean": float(np.mean([x["steps"] for x in records])), **r}))


if __name__ == "__main__":
    main()
