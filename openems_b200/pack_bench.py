"""Times packs (several engines stepped by shared launches) on the seeded
patch-antenna grids of the sweep family.

    python -m openems_b200.pack_bench [--count 64] [--seed 4] [--steps 100]
                                      [--shapes] [--same 4]

Builds `count` patch grids (n ~ U{48..160} per axis, 0.5 mm, CPML 8), packs
them, runs a first batch (which tunes the pack's launch shape), then
`steps` timesteps; prints one JSON line with the tuned shape and the
throughput (cells x steps / host wall time of the batch).  --shapes also
times every candidate shape family member listed below; --same N packs N
engines of the largest grid and compares them with that grid alone.
"""
from __future__ import annotations

import argparse
import json
import time

import numpy as np

SHAPES = [(128, 8, 0), (256, 8, 0), (128, 2, 1), (128, 4, 2), (256, 4, 2), (128, 4, 3)]


def main(argv=None):
    import torch

    from . import fdtd as oe
    from . import workloads as W
    p = argparse.ArgumentParser()
    p.add_argument("--count", type=int, default=64)
    p.add_argument("--seed", type=int, default=4)
    p.add_argument("--steps", type=int, default=100)
    p.add_argument("--shapes", action="store_true")
    p.add_argument("--same", type=int, default=0)
    a = p.parse_args(argv)
    specs = W.patch_specs(a.count, a.seed)
    insts = [W.patch_sweep_instance(s) for s in specs]

    def engine(inst):
        eng = oe.Engine(inst.operator)
        eng.add_cpml(inst.cpml)
        return eng

    def batch(inst, n):
        dt = inst.operator.timestep()
        return oe.EngineBatch(num_steps=n,
                              excitations=[oe.ScheduledExcitation.from_excitation(inst.waveform, 0, n, dt)],
                              termination=oe.TerminationConfig(max_timesteps=n, check_interval=100),
                              energy_monitoring=oe.EnergyMonitorConfig(sample_interval=100, track_peak=True))

    def timed(run, cells):
        # inside the NVTX range "pack_timed" (ncu --nvtx --nvtx-include "pack_timed/")
        torch.cuda.synchronize()
        torch.cuda.nvtx.range_push("pack_timed")
        t0 = time.perf_counter()
        run()
        torch.cuda.synchronize()
        dt = time.perf_counter() - t0
        torch.cuda.nvtx.range_pop()
        return cells * a.steps / dt / 1e6

    cells = np.array([float(np.prod(s.dims)) for s in specs])
    interior = np.array([float(np.prod([max(d - 2 * s.layers, 0) for d in s.dims])) for s in specs])
    engs = [engine(i) for i in insts]
    pack = oe.Pack(engs)
    t0 = time.perf_counter()
    pack.run_batch([batch(i, 20) for i in insts])
    torch.cuda.synchronize()
    out = {"grids": a.count, "cells": cells.sum(), "cpml_fraction": 1.0 - interior.sum() / cells.sum(),
           "tuned_shape": pack.shape(), "first_batch_s": time.perf_counter() - t0,
           "mcells": timed(lambda: pack.run_batch([batch(i, a.steps) for i in insts]), cells.sum())}
    if a.shapes:
        per = {}
        for sh in SHAPES:
            pack.set_shape(*sh)
            pack.run_batch([batch(i, 10) for i in insts])
            per["%dx%d/%d" % sh] = timed(lambda: pack.run_batch([batch(i, a.steps) for i in insts]), cells.sum())
        out["shapes_mcells"] = per
    pack.close()
    for e in engs:
        e.close()
    if a.same > 0:
        big = int(np.argmax(cells))
        copies = [engine(insts[big]) for _ in range(a.same)]
        pb = oe.Pack(copies)
        pb.run_batch([batch(insts[big], 20) for _ in copies])
        out["same_pack_mcells"] = timed(lambda: pb.run_batch([batch(insts[big], a.steps) for _ in copies]),
                                        a.same * cells[big])
        pb.close()
        one = copies[0]
        one.run_batch(batch(insts[big], 20))
        out["same_alone_mcells"] = timed(lambda: one.run_batch(batch(insts[big], a.steps)), cells[big])
        out["same_dims"] = specs[big].dims
        for e in copies:
            e.close()
    print(json.dumps(out, default=str))


if __name__ == "__main__":
    main()
