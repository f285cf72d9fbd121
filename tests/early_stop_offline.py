"""Offline evaluation of staged early termination on oracle traces (CPU).

Runs seeded patches of the small family (openems_b200.predictor.family_specs)
to -50 dB energy decay on the oracle, built exactly as the GPU sweep builds
them (test_gpu_sweep.py::test_sweep_instance_matches_oracle), and keeps
their port traces, energy samples and full-run S11.  It then replays a
StagePlan's decisions instance by instance as staged_sweep would.  At each
stage the engine's port DFTs of the first K steps are rebuilt from the
trace, and stage_check runs on them.  The result is the step ratio
against the plain runs and every stopped instance's S11 error.

    python tests/early_stop_offline.py --seed 50 --count 80 [--cache DIR]
        [--net [--agree DB --slack S]]

prints the standard and the dense plan side by side (with --net: the dense
plan accepted by the trained network, optionally with stage agreement).  The step ratio is an
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


def load_net():
    """The deployed acceptance network (openems_b200/data/stage_net.npz) as
    its float64 restatement with bf16 operands, and its threshold."""
    from oracle.tailnet_ref import StageNetRef
    d = np.load(os.path.join(ROOT, "openems_b200", "data", "stage_net.npz"))
    ref = StageNetRef([(d[f"w{k}"], d[f"b{k}"]) for k in range(4)], (d["w4"], d["b4"]), (d["w5"], d["b5"]))
    return ref, float(np.asarray(d["threshold"]).reshape(-1)[0])


def replay(records, plan: ES.StagePlan, limit_db: float = 0.5, net=None) -> dict:
    """staged_sweep's decisions on recorded runs: per instance the steps it
    runs and, if stopped early, its largest S11 error over the band.  net:
    load_net()'s pair, to accept by the network's score as staged_sweep does
    (with the plan's stage-agreement check and slack when agree_db is set)."""
    band = plan.band(P.FREQS)
    steps, errors, how = [], [], []
    for rec in records:
        tr, dt, full = rec["trace"], rec["dt"], rec["steps"]
        used, err, h = full, 0.0, "full"
        prev = None
        for K in plan.stages:
            if full <= K:
                h = "decayed"
                break
            r = {"uf": P.head_dft(tr[:K, 0], 1, dt, P.FREQS, 0.0), "if": P.head_dft(tr[:K, 1], 1, dt, P.FREQS, 0.5),
                 "final_decay_db": level_db(rec, K)}
            c = ES.stage_check(tr, r, K, dt, P.FREQS, P.HORIZON, 50.0, plan)
            pred = c["pred"]
            agree = ES.s11_db_error(pred, prev, band) if prev is not None else np.inf
            prev = pred
            if net is not None:
                x, sc = ES.stage_features(tr, c, K, P.HORIZON, plan)
                score = float(net[0].forward(x[None], sc[None], bf16=True)[0, 0])
                ok = score < net[1] + (plan.net_slack if plan.agree_db is not None else 0.0)
            else:
                ok = (c["check_mean"] if plan.check == "mean" else c["check_max"]) < plan.tau
            if plan.agree_db is not None:
                ok = ok and agree < plan.agree_db
            if ok:
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
    ap.add_argument("--net", action="store_true", help="accept by the trained network (dense plan only)")
    ap.add_argument("--agree", type=float, default=None, help="stage agreement bound in dB (StagePlan.agree_db)")
    ap.add_argument("--slack", type=float, default=0.0, help="added to the network's threshold with --agree")
    a = ap.parse_args(argv)
    from threadpoolctl import threadpool_limits
    records = load_or_run(a.seed, a.count, a.cache, a.threads)
    net = load_net() if a.net else None
    dense = ES.StagePlan.dense(agree_db=a.agree, net_slack=a.slack)
    plans = (("dense", dense),) if a.net else (("standard (tau 0.05)", ES.StagePlan(tau=0.05)), ("dense", dense))
    with threadpool_limits(a.threads):
        for name, plan in plans:
            r = replay(records, plan, net=net)
            r.pop("steps"), r.pop("errors")
            print(json.dumps({"plan": name, "seed": a.seed, "count": len(records),
                              "full_steps_mean": float(np.mean([x["steps"] for x in records])), **r}))


if __name__ == "__main__":
    main()
