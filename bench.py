#!/usr/bin/env python
"""Benchmark: Yee FDTD throughput (MCells/s) and fraction of the HBM roofline.

Workload (default): cpml_boxes_256 -- 256^3 uniform 1 mm grid, 8-cell CPML
on all faces (m = 3, R0 = 1e-6), 40 seeded dielectric boxes (eps_r U[1,10],
sigma U[0,0.1] S/m), soft Gaussian Ez 0-10 GHz at the centre, FP32 fields and
coefficients.  The full run is 10000 timesteps.

A bench "step" is one EngineBatch of 1000 timesteps (the reference's GPU
batch size, src/fdtd/simulation.rs:219); --steps 10 is the full 10000-step
run.  Working set 1.2 GB >> 126 MB L2, so no L2 flush is needed between steps.

  value  device-resident throughput: CUDA events on the engine's stream around
         K batches (fields, coefficients and CPML state stay in HBM).
  e2e    the same metric through the public API with host buffers: operator
         upload (H2D), K batches with their sampled waveforms (H2D) and energy
         samples / probe traces (D2H), and the final read_fields (D2H).
  roofline  the H and E update kernels (each ~half the step): 60 algorithmic
         bytes per cell per launch (120 B per cell-step; --compressed 37,
         --storage f16/bf16 42, both 19: see kernel_bytes), timed with CUDA
         events around every launch on the engine's stream in a profiling
         batch of the same workload run after the timed region.
  cpu_baseline  the oracle's C++ restatements of the reference's CPU engines
         (the Rayon engine's cell loop and the SIMD engine's z-lines, OpenMP
         over x-planes, -O3 / AVX2, same arithmetic and bits): the faster of
         the two on the host cores, on a bounded sample of timesteps of the
         same workload.
  sweep  the second half of the metric, S11 sweeps per hour: the staged
         early stop (learned acceptance rule) against the plain full-length
         batched sweep of 64 seeded patch antennas (sweep_metric).

--impl reference times that CPU restatement alone (the reference is Rust and
cannot be built here) with all host threads.

Multi-GPU: one grid does not shard without a halo exchange, and the target is
one GPU, so --gpus N runs N independent replicas (weak scaling); value is the
cells*steps of all ranks over the max time across ranks.
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

def kernel_bytes(storage: str, compressed: bool) -> float:
    """Algorithmic bytes per cell of one half-step kernel: the other field
    read, its own field read and written (9 values of the storage type), and
    the coefficients (Ca/Cb or Da/Db, 6 floats; compressed: a one-byte
    material id, the table being in shared memory)."""
    elem = 4 if storage == "f32" else 2
    return 9 * elem + (1 if compressed else 24)
STEPS_PER_BENCH_STEP = 1000
METRIC = "MCells/s (Yee FDTD throughput, % of HBM roofline)"


def parse():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=10)
    p.add_argument("--warmup", type=int, default=3)
    p.add_argument("--impl", choices=("ours", "reference"), default="ours")
    p.add_argument("--n", type=int, default=256, help="grid edge (default 256)")
    p.add_argument("--timesteps-per-step", type=int, default=STEPS_PER_BENCH_STEP)
    p.add_argument("--compressed", action="store_true", help="material-id coefficient storage")
    p.add_argument("--storage", choices=("f32", "f16", "bf16"), default="f32",
                   help="field storage (arithmetic stays f32; f16 / bf16 run the register kernels)")
    p.add_argument("--no-e2e", action="store_true")
    p.add_argument("--no-cpu-baseline", action="store_true")
    p.add_argument("--kernels", choices=("auto", "register", "staged", "zsplit", "pipe"), default="auto")
    p.add_argument("--no-sweep", action="store_true",
                   help="skip the sweep half of the metric (staged vs plain S11 sweeps per hour)")
    return p.parse_args()


def peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi clocks / throttle reasons sampled during the timed region."""

    def __init__(self, device=0):
        self.device = device
        self.proc = None
        self.lines = []

    def __enter__(self):
        q = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--query-gpu={q}", "--format=csv,noheader,nounits", "-lms", "200",
                 "-i", str(self.device)], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except Exception:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *a):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            parts = [p.strip() for p in ln.split(",")]
            if len(parts) < 8:
                continue
            try:
                sm.append(float(parts[0]))
                mx = float(parts[1])
            except ValueError:
                continue
            for nm, v in zip(names, parts[4:8]):
                if v.lower() == "active":
                    reasons.add(nm)
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": mx,
                "reasons": sorted(reasons), "samples": len(sm)}


def build_engine(oe, wl, compressed=False, kernels="auto", storage="f32"):
    op = wl.operator()
    eng = oe.Engine(op, compressed=compressed, kernels=kernels, storage=storage)
    if wl.cpml_layers:
        eng.add_cpml(wl.cpml())
    for comp, pos in wl.probes:
        eng.add_point_probe(comp, pos)
    return op, eng


def batch_for(oe, wl, dt, start, n):
    sched = [oe.ScheduledExcitation.from_excitation(wl.excitation(), start, n, dt)]
    return oe.EngineBatch(num_steps=n, excitations=sched,
                          termination=oe.TerminationConfig(max_timesteps=n, check_interval=100),
                          energy_monitoring=oe.EnergyMonitorConfig(sample_interval=100,
                                                                   track_peak=True))


def run_device(oe, wl, args, torch, dist):
    """value: device-resident batches timed with CUDA events (engine stream)."""
    op, eng = build_engine(oe, wl, args.compressed, args.kernels, args.storage)
    dt = op.timestep()
    T = args.timesteps_per_step
    t = 0
    for _ in range(args.warmup):
        eng.run_batch(batch_for(oe, wl, dt, t, T))
        t += T
    torch.cuda.synchronize()
    if dist is not None:
        dist.barrier()
    dev_s, launches = 0.0, 0
    with ClockSampler(torch.cuda.current_device()) as clk:
        w0 = time.perf_counter()
        # an NVTX range around the timed batches: `ncu --nvtx --nvtx-include
        # bench_timed/` profiles exactly these launches (not the tuner's)
        torch.cuda.nvtx.range_push("bench_timed")
        for _ in range(args.steps):
            eng.run_batch(batch_for(oe, wl, dt, t, T))
            n, s = eng.last_batch_stats()
            dev_s += s
            launches += n
            t += T
        torch.cuda.synchronize()
        torch.cuda.nvtx.range_pop()
        wall = time.perf_counter() - w0
    if dist is not None:
        dist.barrier()
    # per-kernel timing of the same workload (events around every launch)
    eng.set_kernel_profiling(True)
    eng.run_batch(batch_for(oe, wl, dt, t, 200))
    hs, hn, es, en = eng.kernel_profile()
    eng.set_kernel_profiling(False)
    info = eng.launch_info()
    tune = {}
    for r in eng.tune_report():  # fastest timed shape of each kernel family
        k = ("register", "staged", "staged_split", "register_zsplit", "register_pipe")[r["kind"]]
        per = r["ms"] / max(r["reps"], 1)
        if k not in tune or per < tune[k]["ms_per_step"]:
            tune[k] = {"ms_per_step": per, "threads": r["threads"], "ichunk": r["ichunk"], "extra": r["extra"]}
    eng.close()
    return {"device_s": dev_s, "wall_s": wall, "launches": launches, "clocks": clk.summary(),
            "h_avg_s": hs / max(hn, 1), "e_avg_s": es / max(en, 1), "launch": info, "tune": tune}


def run_e2e(oe, wl, args, torch):
    """e2e: public API from host buffers, copies inside the timed region."""
    T = args.timesteps_per_step
    # warm-up on a separate engine (context, kernels, autotune cache)
    op, eng = build_engine(oe, wl, args.compressed, args.kernels, args.storage)
    dt = op.timestep()
    for w in range(max(1, args.warmup)):
        eng.run_batch(batch_for(oe, wl, dt, w * T, T))
    eng.close()
    del op
    torch.cuda.synchronize()
    nprobe = len(wl.probes)
    t0 = time.perf_counter()
    op = wl.operator()                       # host-side operator (12 host arrays)
    eng = oe.Engine(op, compressed=args.compressed, kernels=args.kernels,
                    storage=args.storage)  # H2D of the coefficients
    if wl.cpml_layers:
        eng.add_cpml(wl.cpml())
    for comp, pos in wl.probes:
        eng.add_point_probe(comp, pos)
    h2d = 12 * wl.cells * 4
    d2h = 0
    for k in range(args.steps):
        res = eng.run_batch(batch_for(oe, wl, dt, k * T, T))  # H2D samples, D2H energy
        h2d += T * 4
        d2h += len(res.energy_samples) * 32
        tr = eng.probe_traces()                                 # D2H probe traces
        d2h += tr.nbytes
    e, h = eng.read_fields()                                    # D2H final fields
    d2h += e.nbytes + h.nbytes
    torch.cuda.synchronize()
    wall = time.perf_counter() - t0
    eng.close()
    steps = args.steps * T
    return {"mcells": wl.cells * steps / wall / 1e6, "h2d": h2d / args.steps,
            "d2h": d2h / args.steps, "wall_s": wall, "nprobe": nprobe}


def sweep_metric(count=64, seed=4, concurrency=16):
    """Second half of the headline metric: S11 sweeps per hour, staged early
    stop against the plain full-length batched sweep, on the patch-antenna
    sweep family (n_{x,y,z} ~ U{48..160}, 0.5 mm, CPML 8, 50 ohm lumped feed,
    Gaussian 0-8 GHz, -50 dB energy decay or 60,000 steps, S11 at 801
    points).  Every sweep runs the same instances on this GPU, each timed on
    the host clock around the whole sweep (every instance's engine set-up,
    device runs, DFTs, checks and read-backs).  The plain sweep runs twice,
    with an engine and stream per instance and packed (all instances stepped
    together), and the faster one is the baseline.  The staged sweeps use
    the dense pencil plan, accepting a stage by the residual check alone
    (tau 0.1 dB) or by the trained acceptance network
    (openems_b200/data/stage_net.npz).  The S11 error of an instance is the
    largest |dB difference| to the plain run over f >= 0.5 GHz with both
    clipped at -30 dB (instances that decay or fall back to a full run are
    exact)."""
    from openems_b200 import early_stop as ES
    from openems_b200 import stage_net as SN
    plan = ES.StagePlan.dense()

    def fresh():
        return ES.family_instances("patch", count, seed)

    insts, freqs = fresh()
    band = plan.band(freqs)
    full = ES.full_sweep(insts, freqs, concurrency)
    fs11 = [r["s11"] for r in full["results"]]
    packed = ES.full_sweep(fresh()[0], freqs, concurrency, packed=True)
    same = all(np.array_equal(a["s11"], b["s11"]) and a["timesteps"] == b["timesteps"]
               for a, b in zip(full["results"], packed["results"]))
    plain_s = min(full["wall_s"], packed["wall_s"])
    steps_full = np.array([r["timesteps"] for r in full["results"]], dtype=np.float64)
    cells = np.array([r["cells"] for r in full["results"]], dtype=np.float64)

    def staged(net=None):
        st = ES.staged_sweep(fresh()[0], freqs, plan, concurrency, net=net)
        errs = np.array([0.0 if r["how"] != "predicted" else ES.s11_db_error(r["s11"], f, band)
                         for r, f in zip(st["results"], fs11)])
        hows = [r["how"] for r in st["results"]]
        steps = np.array([r["steps"] for r in st["results"]], dtype=np.float64)
        return {"instances_per_hour": count / st["wall_s"] * 3600.0, "wall_s": st["wall_s"],
                "speedup": plain_s / st["wall_s"], "step_ratio": float(steps_full.sum() / steps.sum()),
                "predicted": hows.count("predicted"), "decayed": hows.count("decayed"),
                "fallback_full": hows.count("full"), "max_err_db": float(errs.max()),
                "median_err_db_predicted": float(np.median(errs[errs > 0])) if (errs > 0).any() else 0.0,
                "instances_over_0.5db": int((errs > 0.5).sum())}

    check = staged()
    net = SN.load_default()
    learned = staged(net) if net is not None else None
    head = learned if learned is not None else check
    return {
        "metric": "S11 sweeps/hr learned vs plain at <= 0.5 dB",
        "workload": f"patch_sweep_{count}_seed{seed}: n ~ U{{48..160}}^3, 0.5 mm, CPML 8, 50 ohm feed, "
                    "Gaussian 0-8 GHz, -50 dB or 60000 steps, 801 S11 points",
        "plain_instances_per_hour": count / plain_s * 3600.0,
        "plain_streams_wall_s": full["wall_s"], "plain_packed_wall_s": packed["wall_s"],
        "plain_streams_mcells": float((cells * steps_full).sum() / full["wall_s"] / 1e6),
        "plain_packed_mcells": float((cells * steps_full).sum() / packed["wall_s"] / 1e6),
        "packed_equals_streams": bool(same),
        "staged_instances_per_hour": head["instances_per_hour"], "speedup": head["speedup"],
        "rule": "learned" if learned is not None else "residual check",
        "staged_learned": learned, "staged_residual_check": check,
        "plan": {"stages": list(plan.stages), "tau_db": plan.tau, "check": plan.check,
                 "samples": plan.samples, "max_modes": plan.max_modes},
        "error": "per instance: max over f >= 0.5 GHz of |dB(staged) - dB(plain)|, both clipped at -30 dB",
    }


def cpu_oracle(wl, threads, zline=False):
    """The oracle's restatement of the reference's CPU engines for the
    workload (FP32, OpenMP over x-planes): the parallel engine's cell loop,
    or with zline the SIMD engine's z-line form (same bits)."""
    import oracle
    lines = [oracle.uniform_lines(n, wl.delta) for n in wl.dims]
    dt, delta = oracle.grid_timestep(*lines)
    s = oracle.OracleSim(*wl.dims, dt, delta, precision=32, threads=threads, zline=zline)
    for b in wl.boxes:
        s.set_material(*b)
    if wl.cpml_layers:
        s.enable_cpml((wl.cpml_layers,) * 6)
    x = wl.excitation()
    s.add_excitation_analytic(x.position, x.direction, True, 0, list(x.params), 1.0, 0, 100000)
    return s


def faster_cpu_form(wl, threads):
    """(simulation, loop form name, seconds per step) of the faster of the two
    restated reference CPU engines on this host, each timed over 3 steps
    after 2 of warm-up."""
    best = None
    for zline in (False, True):
        s = cpu_oracle(wl, threads, zline)
        s.run_batch(2)
        t0 = time.perf_counter()
        s.run_batch(3)
        per = (time.perf_counter() - t0) / 3
        if best is None or per < best[2]:
            best = (s, "SIMD engine z-lines" if zline else "parallel engine cell loop", per)
    return best


def cpu_sample(wl, target_s=12.0, threads=None, max_steps=400):
    """A bounded sample of timesteps of the same workload on the host cores,
    with the faster restated CPU engine."""
    threads = threads or os.cpu_count() or 1
    s, form, per = faster_cpu_form(wl, threads)
    n = int(max(2, min(max_steps, target_s / max(per, 1e-9))))
    t0 = time.perf_counter()
    s.run_batch(n)
    el = time.perf_counter() - t0
    return {"value": wl.cells * n / el / 1e6, "steps": n, "threads": threads, "seconds": el, "form": form}


def max_over_ranks(x: float, dist, device) -> float:
    """The largest x over all ranks (x itself without a process group)."""
    if dist is None:
        return x
    import torch
    t = torch.tensor([x], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def job_mcells(world: int, cells: int, timesteps: int, seconds: float) -> float:
    """Whole-job throughput: every rank's cells x timesteps over the slowest rank's time."""
    return world * cells * timesteps / seconds / 1e6


def main():
    args = parse()
    from openems_b200 import workloads
    wl = workloads.cpml_boxes(args.n, 10000)
    hbm, peak_src = peaks()
    config = {"workload": f"{wl.name}: {args.n}^3 1 mm, CPML 8 (m=3, R0=1e-6), 40 dielectric boxes "
                          "(default_rng(2)), Gaussian Ez 0-10 GHz, FP32, 10000 timesteps",
              "timesteps_per_step": args.timesteps_per_step, "cells": wl.cells,
              "coefficients": "compressed (material id + table)" if args.compressed else "full arrays",
              "field_storage": args.storage,
              "l2": "working set 1.2 GB > 126 MB L2; no flush", "parallelism": "replicas"}

    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))

    if args.impl == "reference":
        if rank != 0:
            return
        cores = os.cpu_count() or 1
        sim, form, per = faster_cpu_form(wl, cores)
        # timesteps per bench step: about 6 s of CPU work (~400 timesteps of
        # the 256^3 grid on 16 cores), at most the GPU's step
        T = int(max(1, min(args.timesteps_per_step, 6.0 / max(per, 1e-9))))
        times = []
        for k in range(args.warmup + args.steps):
            t0 = time.perf_counter()
            sim.run_batch(T)
            if k >= args.warmup:
                times.append(time.perf_counter() - t0)
        value = wl.cells * T * len(times) / sum(times) / 1e6
        sample = (f"{T} timesteps of {wl.name} per step, C++ restatement of the reference's CPU engines "
                  f"(-O3, AVX2), the faster form on this host: {form}, OpenMP on {cores} threads "
                  "(the Rust reference is not buildable here)")
        print(json.dumps({
            "impl": "reference", "metric": METRIC, "value": value, "unit": "MCells/s",
            "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic", "config": config,
            "cpu_baseline": {"value": value, "unit": "MCells/s", "cores": cores, "kind": "port",
                             "sample": sample},
            "e2e": {"value": value, "unit": "MCells/s", "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0}}))
        return

    import torch
    import openems_b200 as oe
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist_
        local = int(os.environ.get("LOCAL_RANK", "0"))
        torch.cuda.set_device(local)
        dist_.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                 device_id=torch.device("cuda", local))
        dist = dist_
    else:
        torch.cuda.set_device(0)
    torch.cuda.init()

    d = run_device(oe, wl, args, torch, dist)
    steps_total = args.steps * args.timesteps_per_step
    t_dev = max_over_ranks(d["device_s"], dist, "cuda")
    value = job_mcells(world, wl.cells, steps_total, t_dev)
    e2e = None if args.no_e2e else run_e2e(oe, wl, args, torch)
    if dist is not None:
        if e2e is not None:
            e2e["mcells"] = job_mcells(world, wl.cells, steps_total, max_over_ranks(e2e["wall_s"], dist, "cuda"))
        dist.barrier()
    if rank != 0:
        if dist is not None:
            dist.destroy_process_group()
        return
    kernel_avg = max(d["h_avg_s"], d["e_avg_s"])
    dominant = "k_update_h" if d["h_avg_s"] >= d["e_avg_s"] else "k_update_e"
    per_kernel = kernel_bytes(args.storage, args.compressed)
    achieved = per_kernel * wl.cells / kernel_avg / 1e9
    traffic = None
    prof_path = os.path.join(ROOT, "profiles", "traffic.json")
    if os.path.exists(prof_path) and args.storage == "f32" and not args.compressed:  # captured for that variant
        try:
            with open(prof_path) as f:
                tj = json.load(f)
            traffic = tj.get(dominant, {}).get("bytes_per_cell")
            traffic = traffic * wl.cells if traffic else None
        except Exception:
            traffic = None
    cpu = None if args.no_cpu_baseline else cpu_sample(wl)
    # the sweep half of the metric: one GPU (at N > 1 the ranks would run
    # replicas of the same sweep, which adds nothing)
    sweep = None if (args.no_sweep or world > 1) else sweep_metric()
    step_gbs = 2 * per_kernel * wl.cells * steps_total / t_dev / 1e9 / world
    line = {
        "metric": METRIC, "value": value, "unit": "MCells/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": t_dev / args.steps * 1e3, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32", "data": "synthetic", "config": config,
        "hbm_fraction_step": step_gbs / hbm,
        "roofline": {"bound": "hbm", "kernel": dominant, "achieved": achieved, "peak": hbm,
                     "peak_source": peak_src, "unit": "GB/s", "frac": achieved / hbm,
                     "traffic": traffic,
                     "algorithmic_bytes_per_launch": per_kernel * wl.cells,
                     "h_kernel_ms": d["h_avg_s"] * 1e3, "e_kernel_ms": d["e_avg_s"] * 1e3},
        "gpu_launches": d["launches"],
        "clocks": d["clocks"],
        "wall_s_timed": d["wall_s"],
        "launch_shape": d["launch"],
        "tuning": d["tune"],
    }
    if e2e is not None:
        line["e2e"] = {"value": e2e["mcells"], "unit": "MCells/s",
                       "h2d_bytes_per_step": int(e2e["h2d"]), "d2h_bytes_per_step": int(e2e["d2h"])}
    if cpu is not None:
        line["cpu_baseline"] = {"value": cpu["value"], "unit": "MCells/s", "cores": cpu["threads"],
                                "kind": "port",
                                "sample": f"{cpu['steps']} timesteps of {wl.name} "
                                          f"({cpu['seconds']:.1f} s), C++ restatement of the reference's "
                                          f"CPU engines (-O3, AVX2), the faster form: {cpu['form']}"}
    if sweep is not None:
        line["sweep"] = sweep
    print(json.dumps(line))
    if dist is not None:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
