"""Staged early termination of port sweeps.

Every instance of a sweep runs to the first stage (K steps) and pauses
(oems_sweep_advance keeps its engine).  Its S11 is then predicted from the
engine's port DFTs of the K simulated steps plus the matrix-pencil
continuation of the last window of the port traces (predictor.py), summed up
to the step where the plain run is estimated to stop (plain_end).  The
residual check repeats the prediction from a window that ends `lag` steps
earlier: when the two predicted S11 curves agree to within `tau` dB over the
band (both clipped at -30 dB), the prediction is accepted and the instance
ends there.  Otherwise the instance continues to the next stage, and after the
last stage runs on to the plain end condition (-50 dB energy decay), whose
S11 is exact: the full run is the fallback and the reference for the error.
Instances that decay before a stage are exact as well.

`calibrate` records the check and the prediction error of every instance at
every stage against its full run, so that `tau` can be chosen on a training
family; `main` times a staged sweep against the plain full-length sweep of the
same instances.
"""
from __future__ import annotations

import math
import os
import time
from concurrent.futures import ThreadPoolExecutor
from dataclasses import dataclass
from typing import Dict, List, Optional, Sequence

import numpy as np

from . import predictor as P
from . import workloads as W
from .sweep import Sweep

FLOOR_DB = -30.0


def s11_db(s: np.ndarray, floor: float = FLOOR_DB) -> np.ndarray:
    return np.maximum(20.0 * np.log10(np.maximum(np.abs(s), 1e-30)), floor)


def s11_db_error(a: np.ndarray, b: np.ndarray, band: np.ndarray, floor: float = FLOOR_DB) -> float:
    """Largest |dB(a) - dB(b)| over the band, both clipped at `floor` dB."""
    return float(np.abs(s11_db(a, floor) - s11_db(b, floor))[band].max())


def s11_db_mean_error(a: np.ndarray, b: np.ndarray, band: np.ndarray, floor: float = FLOOR_DB) -> float:
    """Mean |dB(a) - dB(b)| over the band, both clipped at `floor` dB."""
    return float(np.abs(s11_db(a, floor) - s11_db(b, floor))[band].mean())


def pencil_s11(trace: np.ndarray, uf: np.ndarray, if_: np.ndarray, K: int, dt: float, freqs: np.ndarray,
               horizon: int, lag: int = 0, R: float = 50.0, u_modes=None, parts: bool = False,
               **pencil) -> np.ndarray:
    """S11 predicted at K: the engine's DFTs of steps [0, K - lag) (those of
    [0, K) minus the last `lag` trace samples) plus the pencil continuation
    of the window that ends at K - lag.  trace: (>= K, 2) port u, i.
    u_modes: the port voltage's pencil modes of that window, if already
    computed.  parts=True returns (S11, head u, tail u, head i, tail i)."""
    uh, ih = uf.copy(), if_.copy()
    if lag:
        uh -= P.head_dft(trace[K - lag:K, 0], K - lag + 1, dt, freqs, 0.0)
        ih -= P.head_dft(trace[K - lag:K, 1], K - lag + 1, dt, freqs, 0.5)
    ke = K - lag
    ut = P.pencil_tail_dft(trace[:ke, 0], ke, dt, freqs, 0.0, horizon, modes=u_modes, **pencil)
    it = P.pencil_tail_dft(trace[:ke, 1], ke, dt, freqs, 0.5, horizon, **pencil)
    if parts:
        return P.s11(uh + ut, ih + it, R), uh, ut, ih, it
    return P.s11(uh + ut, ih + it, R)


def plain_end(u: np.ndarray, K: int, level_db: float, dt: float, decay_db: float, cap: int,
              modes=None, **pencil) -> int:
    """Step at which the plain run would stop: its field energy, now
    `level_db` below the peak, is continued with the pencil modes of the port
    voltage (each mode's energy |c|^2 decaying at twice its rate) down to
    -decay_db, rounded up to the run's 100-step energy checks, at most `cap`.
    modes: pencil_modes(u, K, dt, **pencil) if already computed."""
    p, c = modes if modes is not None else P.pencil_modes(u, K, dt, **pencil)
    target = 10.0 ** ((-abs(decay_db) - level_db) / 10.0)  # E(end) / E(now)
    if len(p) == 0 or target >= 1.0:
        return K
    rate, w = -2.0 * p.real, np.abs(c) ** 2

    def rest(t):
        return (w * np.exp(-rate * t)).sum() / w.sum()

    lo, hi = 0.0, (cap - K) * dt
    if rest(hi) > target:
        return cap
    for _ in range(60):
        mid = 0.5 * (lo + hi)
        lo, hi = (mid, hi) if rest(mid) > target else (lo, mid)
    return int(min(cap, np.ceil((K + hi / dt) / 100.0) * 100))


@dataclass
class StagePlan:
    """Stages (step counts), the residual check's lag and threshold, the band
    it is evaluated on and the pencil settings: at stage K the window is
    `window_frac` K samples (at most `max_window`), decimated to about
    `samples` points."""

    stages: Sequence[int] = (2048, 4096, 8192, 16384)
    lag: int = 256
    tau: float = 0.1
    fmin: float = 0.5e9
    window_frac: float = 0.75
    max_window: int = 12288
    samples: int = 384
    max_modes: int = 40
    end_estimate: bool = True
    check: str = "max"  # residual statistic over the band: "max" or "mean" |dB difference|
    # stage agreement: a stage is accepted only if its prediction is within
    # agree_db (largest |dB difference| over the band) of the previous
    # stage's; None leaves it out.  net_slack is added to the network's
    # threshold when the agreement check is on.
    agree_db: Optional[float] = None
    net_slack: float = 0.0

    @classmethod
    def dense(cls, **kw) -> "StagePlan":
        """The strict-check operating point with a denser pencil: ten stages
        from 1,024 to 24,576 steps, 512 samples per window, up to 150 modes,
        largest-error check at 0.1 dB (chosen on the seed-5 training patches
        as the largest threshold with no instance above 0.5 dB)."""
        base = dict(stages=(1024, 1536, 2048, 3072, 4096, 6144, 8192, 12288, 16384, 24576), samples=512,
                    max_modes=150, tau=0.1, check="max")
        base.update(kw)
        return cls(**base)

    def band(self, freqs: np.ndarray) -> np.ndarray:
        return np.asarray(freqs) >= self.fmin

    def pencil(self, K: int) -> dict:
        window = min(int(self.window_frac * K), self.max_window)
        return dict(window=window, decimate=max(1, window // self.samples), max_modes=self.max_modes)


def stage_check(trace, r, K, dt, freqs, horizon, decay_db, plan: StagePlan) -> dict:
    """Everything known about an instance paused at stage K: the pencil
    prediction of S11 ("pred"), the residual check's largest and mean |dB|
    difference over the band ("check_max", "check_mean"), the same largest
    difference against the prediction from a window 1024 steps earlier
    ("check_far"), how far the prediction moves when its continuation is
    scaled by 1.1 ("tail_sens", largest |dB| change over the band), the
    estimated end step of the plain run ("end"), the port voltage's pencil
    mode count ("modes"), the pencil window ("window") and the energy level
    below the peak ("level", dB)."""
    pen = plan.pencil(K)
    um = P.pencil_modes(trace[:K, 0], K, dt, **pen)  # serves both the end estimate and the prediction
    end = plain_end(trace[:, 0], K, r["final_decay_db"], dt, decay_db, horizon, modes=um, **pen) \
        if plan.end_estimate else horizon
    end = max(end, K)
    a, uh, ut, ih, it = pencil_s11(trace, r["uf"], r["if"], K, dt, freqs, end, 0, u_modes=um, parts=True, **pen)
    b = pencil_s11(trace, r["uf"], r["if"], K, dt, freqs, end, plan.lag, **pen)
    far = min(4 * plan.lag, K // 2)
    c = pencil_s11(trace, r["uf"], r["if"], K, dt, freqs, end, far, **pen)
    band = plan.band(freqs)
    sens = s11_db_error(P.s11(uh + 1.1 * ut, ih + 1.1 * it), a, band)
    return {"pred": a, "check_max": s11_db_error(a, b, band), "check_mean": s11_db_mean_error(a, b, band),
            "check_far": s11_db_error(a, c, band), "tail_sens": sens,
            "end": end, "modes": len(um[0]), "window": pen["window"], "level": float(r["final_decay_db"])}


def stage_features(trace, c: dict, K: int, horizon: int, plan: StagePlan):
    """The learned rule's inputs (stage_net.window_input, scalar_input) from
    a stage_check record."""
    from . import stage_net as SN
    x = SN.window_input(trace, K, c["window"])
    sc = SN.scalar_input(c["check_max"], c["check_mean"], c["check_far"], c["tail_sens"], c["level"], K, c["end"])
    return x, sc


def check_instance(trace, r, K, dt, freqs, horizon, decay_db, plan: StagePlan, both: bool = False):
    """(prediction at K, residual-check value in dB, continuation end step);
    with both=True the check value is the pair (max, mean) over the band."""
    c = stage_check(trace, r, K, dt, freqs, horizon, decay_db, plan)
    if both:
        return c["pred"], (c["check_max"], c["check_mean"]), c["end"]
    return c["pred"], c["check_mean"] if plan.check == "mean" else c["check_max"], c["end"]


def _pool():
    return ThreadPoolExecutor(max_workers=max(1, os.cpu_count() or 1))


def staged_sweep(instances, freqs: np.ndarray, plan: StagePlan, concurrency: int = 16,
                 batch_steps: int = 2000, net=None) -> dict:
    """Runs the staged sweep; returns per instance S11, how it was obtained
    ("decayed", "predicted" at a stage, or "full" fallback) and the steps
    run.  `concurrency` worker threads each take one instance at a time
    through its stages (oems_sweep_advance) and checks, so the host checks of
    one instance overlap the device runs of the others.  With a trained
    stage_net.StageNet `net`, a stage is accepted when the network's
    predicted error is below its threshold instead of by the residual check
    alone (the check values are among the network's inputs)."""
    import queue
    import threading

    from threadpoolctl import threadpool_limits
    dt = instances[0].operator.timestep()
    horizon = max(i.max_timesteps for i in instances)
    decay_db = instances[0].energy_decay_db
    sw = Sweep(freqs, concurrency=concurrency)
    sw.set_trace_steps(max(plan.stages))
    ids = [sw.add(i) for i in instances]
    todo = queue.Queue()
    for i in ids:
        todo.put(i)
    out: Dict[int, dict] = {}
    errors: List[BaseException] = []
    check_s = [0.0]
    lock = threading.Lock()
    net_lock = threading.Lock()

    band = plan.band(freqs)

    def one(i):
        prev = None
        for K in plan.stages:
            sw.advance(i, K, batch_steps)
            r = sw.result(i)
            if not r["paused"]:
                return {"s11": r["s11"], "how": "decayed", "steps": r["timesteps"], "stage": K}
            tc = time.perf_counter()
            trace = sw.trace(i)
            c = stage_check(trace, r, K, dt, freqs, horizon, decay_db, plan)
            d = c["check_mean"] if plan.check == "mean" else c["check_max"]
            agree = s11_db_error(c["pred"], prev, band) if prev is not None else math.inf
            prev = c["pred"]
            if net is not None:
                x, sc = stage_features(trace, c, K, horizon, plan)
                with net_lock:  # one forward at a time (the network keeps its activations)
                    score = float(net.predict(x[None], sc[None])[0])
                ok = score < net.threshold + (plan.net_slack if plan.agree_db is not None else 0.0)
            else:
                score, ok = d, d < plan.tau
            if plan.agree_db is not None:
                ok = ok and agree < plan.agree_db
            with lock:
                check_s[0] += time.perf_counter() - tc
            if ok:
                sw.finish(i)
                return {"s11": c["pred"], "how": "predicted", "steps": K, "stage": K, "check_db": d,
                        "score": score, "agree_db": agree, "end": c["end"]}
        sw.advance(i, horizon, batch_steps)
        r = sw.result(i)
        return {"s11": r["s11"], "how": "full", "steps": r["timesteps"], "stage": None}

    def worker():
        while True:
            try:
                i = todo.get_nowait()
            except queue.Empty:
                return
            try:
                res = one(i)
            except BaseException as e:  # reported after the other workers end
                with lock:
                    errors.append(e)
                return
            with lock:
                out[i] = res

    t0 = time.perf_counter()
    with threadpool_limits(1):
        threads = [threading.Thread(target=worker) for _ in range(max(1, concurrency))]
        for t in threads:
            t.start()
        for t in threads:
            t.join()
    wall = time.perf_counter() - t0
    sw.close()
    if errors:
        raise errors[0]
    return {"results": [out[i] for i in ids], "wall_s": wall, "check_s": check_s[0]}


def full_sweep(instances, freqs: np.ndarray, concurrency: int = 16, batch_steps: int = 2000,
               packed: bool = False) -> dict:
    """The plain batched sweep: every instance to its end condition (packed:
    all instances stepped together through one pack)."""
    t0 = time.perf_counter()
    sw = Sweep(freqs, concurrency=concurrency, packed=packed)
    ids = [sw.add(i) for i in instances]
    sw.run(batch_steps)
    res = [sw.result(i) for i in ids]
    wall = time.perf_counter() - t0
    sw.close()
    return {"results": res, "wall_s": wall}


def calibrate(instances, freqs: np.ndarray, plan: StagePlan, full_s11: List[np.ndarray],
              concurrency: int = 16, batch_steps: int = 2000, features: bool = False) -> dict:
    """Check values d[n, s] and prediction errors e[n, s] (dB, against the
    full runs) of every instance at every stage, with no instance finished
    early (NaN where the instance had already decayed).  features=True also
    keeps the learned rule's inputs: "x" (n, s, T_WIN, 2) float16 windows and
    "s" (n, s, N_SCALAR) float32 (zeros where the instance had decayed)."""
    dt = instances[0].operator.timestep()
    horizon = max(i.max_timesteps for i in instances)
    decay_db = instances[0].energy_decay_db
    band = plan.band(freqs)
    sw = Sweep(freqs, concurrency=concurrency)
    sw.set_trace_steps(max(plan.stages))
    ids = [sw.add(i) for i in instances]
    n, ns = len(ids), len(plan.stages)
    d = np.full((n, ns), np.nan)
    e = np.full((n, ns), np.nan)
    end = np.full((n, ns), np.nan)
    em = np.full((n, ns), np.nan)
    dm = np.full((n, ns), np.nan)
    if features:
        from . import stage_net as SN
        X = np.zeros((n, ns, SN.T_WIN, 2), dtype=np.float16)
        S = np.zeros((n, ns, SN.N_SCALAR), dtype=np.float32)

    def job(trace, r, K):
        c = stage_check(trace, r, K, dt, freqs, horizon, decay_db, plan)
        f = stage_features(trace, c, K, horizon, plan) if features else None
        return c, f

    from threadpoolctl import threadpool_limits
    with _pool() as pool, threadpool_limits(1):
        for s, K in enumerate(plan.stages):
            sw.run_until(K, batch_steps)
            jobs = {}
            for k, i in enumerate(ids):
                r = sw.result(i)
                if r["paused"]:
                    jobs[k] = pool.submit(job, sw.trace(i), r, K)
            for k, j in jobs.items():
                c, f = j.result()
                d[k, s], dm[k, s], end[k, s] = c["check_max"], c["check_mean"], c["end"]
                e[k, s] = s11_db_error(c["pred"], full_s11[k], band)
                em[k, s] = s11_db_mean_error(c["pred"], full_s11[k], band)
                if features:
                    X[k, s] = f[0][:, :2].astype(np.float16)
                    S[k, s] = f[1]
    sw.close()
    out = {"check_db": d, "check_mean_db": dm, "error_db": e, "mean_error_db": em, "end": end}
    if features:
        out["x"], out["s"] = X, S
    return out


def simulate(cal: dict, tau: float, check: str = "max") -> dict:
    """Outcome of the staged rule with threshold tau on calibration records:
    per instance the stage index it stops at (-1: decayed or full run) and
    its S11 error (0 for exact)."""
    d = cal["check_mean_db"] if check == "mean" else cal["check_db"]
    e = cal["error_db"]
    em = cal.get("mean_error_db", e)
    stop = np.full(len(d), -1)
    err = np.zeros(len(d))
    merr = np.zeros(len(d))
    for k in range(len(d)):
        for s in range(d.shape[1]):
            if np.isnan(d[k, s]):
                break  # decayed before this stage: exact
            if d[k, s] < tau:
                stop[k], err[k], merr[k] = s, e[k, s], em[k, s]
                break
    return {"stop": stop, "error_db": err, "mean_error_db": merr}


def family_instances(family: str, count: int, seed: int):
    """(instances, freqs): "small" is the reduced patch family (n ~ U{40..80},
    0-12 GHz, 241 points, cap 40000 steps); "patch" the 64-instance patch
    sweep family (n ~ U{48..160}, 0-8 GHz, 801 points, cap 60000 steps)."""
    if family == "small":
        specs = P.family_specs(count, seed)
        return ([W.patch_sweep_instance(s, delta=0.5e-3, decay_db=50.0, max_steps=P.HORIZON, fmax=12e9)
                 for s in specs], P.FREQS)
    specs = W.patch_specs(count, seed=seed)
    return ([W.patch_sweep_instance(s, decay_db=50.0, max_steps=60000) for s in specs],
            np.linspace(0.0, 8e9, 801))


def main(argv=None):
    """python -m openems_b200.early_stop {calibrate,run} --family small|patch
    --count N --seed S [--tau T]: `calibrate` prints, per threshold, the
    largest and 99th-percentile S11 error and the mean steps run; `run` times
    the plain full sweep and the staged sweep of the same instances and prints
    one JSON line (errors against the full runs, instances per hour)."""
    import argparse
    import json
    p = argparse.ArgumentParser()
    p.add_argument("cmd", choices=["calibrate", "run"])
    p.add_argument("--family", choices=["small", "patch"], default="small")
    p.add_argument("--count", type=int, default=500)
    p.add_argument("--seed", type=int, default=50)
    p.add_argument("--concurrency", type=int, default=16)
    p.add_argument("--plan", choices=["standard", "dense"], default="standard",
                   help="dense: StagePlan.dense() (ten stages, 512 samples, 150 modes, max check at 0.1 dB)")
    p.add_argument("--tau", type=float, default=None, help="default 0.1")
    p.add_argument("--stages", default=None, help="default 2048,4096,8192,16384 (standard plan)")
    p.add_argument("--no-end-estimate", action="store_true",
                   help="continue every prediction to the step cap instead of the estimated end")
    p.add_argument("--check", choices=["max", "mean"], default="max",
                   help="residual statistic over the band (run)")
    p.add_argument("--save", default=None, help="calibrate: write the per-instance records to this .npz")
    a = p.parse_args(argv)
    kw = dict(end_estimate=not a.no_end_estimate)
    if a.tau is not None:
        kw["tau"] = a.tau
    if a.stages is not None:
        kw["stages"] = tuple(int(x) for x in a.stages.split(","))
    if a.plan == "dense":
        plan = StagePlan.dense(check=a.check, **kw)
    else:
        plan = StagePlan(check=a.check, **{"tau": 0.1, "stages": (2048, 4096, 8192, 16384), **kw})
    insts, freqs = family_instances(a.family, a.count, a.seed)
    band = plan.band(freqs)
    full = full_sweep(insts, freqs, a.concurrency)
    fs11 = [r["s11"] for r in full["results"]]
    steps_full = np.array([r["timesteps"] for r in full["results"]])
    head = {"family": a.family, "count": a.count, "seed": a.seed, "stages": list(plan.stages),
            "lag": plan.lag, "full_wall_s": full["wall_s"], "full_steps_mean": float(steps_full.mean()),
            "instances_per_hour_full": a.count / full["wall_s"] * 3600.0}
    if a.cmd == "calibrate":
        insts, _ = family_instances(a.family, a.count, a.seed)
        cal = calibrate(insts, freqs, plan, fs11, a.concurrency)
        # how well the continuation end matches the plain run's own end
        rel = np.abs(cal["end"] - steps_full[:, None]) / steps_full[:, None]
        head["end_rel_error_median_per_stage"] = [float(np.nanmedian(rel[:, s])) if np.isfinite(rel[:, s]).any()
                                                  else None for s in range(rel.shape[1])]
        if a.save:
            np.savez(a.save, steps_full=steps_full, stages=np.array(plan.stages), **cal)
        rows = []
        for check, tau in [("max", t) for t in (0.02, 0.05, 0.1, 0.2, 0.3, 0.5)] + \
                          [("mean", t) for t in (0.01, 0.02, 0.05, 0.1, 0.2)]:
            sim = simulate(cal, tau, check)
            steps = np.where(sim["stop"] >= 0, np.array(plan.stages)[np.maximum(sim["stop"], 0)], steps_full)
            rows.append({"check": check, "tau": tau, "max_err_db": float(sim["error_db"].max()),
                         "mean_err_db_max": float(sim["mean_error_db"].max()),
                         "p99_err_db": float(np.percentile(sim["error_db"], 99)),
                         "over_0.5db": int((sim["error_db"] > 0.5).sum()),
                         "predicted": int((sim["stop"] >= 0).sum()),
                         "steps_mean": float(steps.mean()),
                         "step_ratio": float(steps_full.mean() / steps.mean())})
        head["calibration"] = rows
        print(json.dumps(head))
        return
    insts, _ = family_instances(a.family, a.count, a.seed)
    st = staged_sweep(insts, freqs, plan, a.concurrency)
    errs = np.array([0.0 if r["how"] != "predicted" else s11_db_error(r["s11"], f, band)
                     for r, f in zip(st["results"], fs11)])
    merrs = np.array([0.0 if r["how"] != "predicted" else s11_db_mean_error(r["s11"], f, band)
                      for r, f in zip(st["results"], fs11)])
    hows = [r["how"] for r in st["results"]]
    head.update({"check": plan.check, "tau": plan.tau, "staged_wall_s": st["wall_s"], "staged_check_s_all_threads": st["check_s"],
                 "instances_per_hour_staged": a.count / st["wall_s"] * 3600.0,
                 "speedup": full["wall_s"] / st["wall_s"],
                 "predicted": hows.count("predicted"), "decayed": hows.count("decayed"),
                 "fallback_full": hows.count("full"),
                 "staged_steps_mean": float(np.mean([r["steps"] for r in st["results"]])),
                 "max_err_db": float(errs.max()), "p99_err_db": float(np.percentile(errs, 99)),
                 "median_err_db_predicted": float(np.median(errs[errs > 0])) if (errs > 0).any() else 0.0,
                 "over_0.5db": int((errs > 0.5).sum()), "mean_err_db_max": float(merrs.max()),
                 "mean_over_0.5db": int((merrs > 0.5).sum())})
    print(json.dumps(head))


if __name__ == "__main__":
    main()
