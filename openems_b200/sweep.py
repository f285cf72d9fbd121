"""Batched lumped-port sweeps: many independent grids run to energy decay on
one GPU, several at a time, each returning its port DFTs and S11.

The scheduler is native (csrc/sweep.cpp, oems_sweep_* in oems_host.h); this
module builds its inputs and reads its results.  S11 uses Port.CalcPort's
arithmetic (python/openEMS/ports.py:136-138).
"""
from __future__ import annotations

import ctypes
from dataclasses import dataclass
from typing import Optional

import numpy as np

from . import _native as N
from .fdtd import CpmlBoundaries, Excitation, Operator


@dataclass
class SweepInstance:
    """One grid of a sweep: its operator (materials and PEC already set), a
    lumped port on one E edge with its background material, the source
    waveform, CPML and the end condition."""

    operator: Operator
    port_position: tuple
    port_direction: int
    waveform: Excitation
    port_resistance: float = 50.0
    port_eps_r: float = 1.0
    port_sigma: float = 0.0
    cpml: Optional[CpmlBoundaries] = None
    energy_decay_db: float = 50.0
    max_timesteps: int = 60000

    def to_c(self) -> N.SweepInstanceC:
        d = N.SweepInstanceC()
        d.op = self.operator.handle
        if self.cpml is not None:
            d.cpml = self.cpml.to_c()
        for a in range(3):
            d.port_position[a] = int(self.port_position[a])
        d.port_direction = int(self.port_direction)
        d.port_resistance = float(self.port_resistance)
        d.port_eps_r = float(self.port_eps_r)
        d.port_sigma = float(self.port_sigma)
        d.waveform = self.waveform.to_c()
        d.energy_decay_db = float(self.energy_decay_db)
        d.max_timesteps = int(self.max_timesteps)
        return d


class Sweep:
    """oems_sweep: frequencies shared by every instance; `concurrency`
    engines run at a time on `device`.  packed=True: run / run_until step
    the instances that share a step count together (one launch per
    half-step over all their grids, oems_sweep_set_packed), with the same
    bits per instance; `concurrency` then only parallelises their set-up."""

    def __init__(self, freqs, concurrency: int = 4, device: int = -1, compressed: bool = False,
                 autotune: bool = False, kernels: str = "register", storage: str = "f32", packed: bool = False):
        self.freqs = np.ascontiguousarray(freqs, dtype=np.float64)
        if storage not in N.STORAGE_FLAGS:
            raise N.ConfigError(f"unknown field storage {storage!r}")
        flags = (N.ENGINE_COMPRESSED if compressed else 0) | (0 if autotune else N.ENGINE_NO_AUTOTUNE) \
            | {"auto": 0, "register": N.ENGINE_REGISTER_KERNELS, "staged": N.ENGINE_STAGED_KERNELS}[kernels] \
            | N.STORAGE_FLAGS[storage]
        h = ctypes.c_void_p()
        N.check(N.lib().oems_sweep_create(device, concurrency, flags,
                                          self.freqs.ctypes.data_as(ctypes.POINTER(N.c_f64)),
                                          len(self.freqs), ctypes.byref(h)))
        self._h = h
        self.count = 0
        if packed:
            N.check(N.lib().oems_sweep_set_packed(h, 1))

    def close(self):
        h = getattr(self, "_h", None)
        if h:
            N.lib().oems_sweep_destroy(h)
            self._h = None

    def __del__(self):
        # at interpreter exit the module globals (the library handle) may be
        # gone already; the process is ending and the driver frees the device
        try:
            self.close()
        except (TypeError, AttributeError):
            pass

    def add(self, inst: SweepInstance) -> int:
        d = inst.to_c()
        iid = N.c_i32()
        N.check(N.lib().oems_sweep_add(self._h, ctypes.byref(d), ctypes.byref(iid)))
        self.count += 1
        return iid.value

    def run(self, batch_steps: int = 2000):
        """Runs every instance that has not ended to its end."""
        N.check(N.lib().oems_sweep_run(self._h, batch_steps))

    def run_until(self, step_cap: int, batch_steps: int = 2000):
        """Runs every instance that has not ended up to `step_cap` steps in
        total; those that reach it pause and continue on the next call."""
        N.check(N.lib().oems_sweep_run_until(self._h, batch_steps, int(step_cap)))

    def advance(self, iid: int, step_cap: int, batch_steps: int = 2000):
        """One instance, on the calling thread, up to `step_cap` steps in
        total (instances may be advanced from several threads at once)."""
        N.check(N.lib().oems_sweep_advance(self._h, iid, batch_steps, int(step_cap)))

    def finish(self, iid: int):
        """Ends a paused instance with its partial result."""
        N.check(N.lib().oems_sweep_finish(self._h, iid))

    def result(self, iid: int) -> dict:
        info = N.SweepResultC()
        nf = len(self.freqs)
        bufs = [np.zeros(2 * nf) for _ in range(3)]
        ptrs = [b.ctypes.data_as(ctypes.POINTER(N.c_f64)) for b in bufs]
        N.check(N.lib().oems_sweep_get_result(self._h, iid, ctypes.byref(info), *ptrs))
        uf, if_, s11 = (b[0::2] + 1j * b[1::2] for b in bufs)
        return {"timesteps": int(info.timesteps), "termination_reason": int(info.termination_reason),
                "final_decay_db": float(info.final_decay_db), "device_seconds": float(info.device_seconds),
                "cells": float(info.cells), "setup_seconds": float(info.setup_seconds),
                "host_seconds": float(info.host_seconds), "paused": bool(info.paused),
                "uf": uf, "if": if_, "s11": s11}

    def set_trace_steps(self, steps: int):
        """Record the port u / i traces of the first `steps` timesteps."""
        N.check(N.lib().oems_sweep_set_trace_steps(self._h, int(steps)))

    def trace(self, iid: int) -> np.ndarray:
        """(steps, 2) float64: u, i per recorded timestep."""
        n = N.c_u64()
        N.check(N.lib().oems_sweep_get_trace(self._h, iid, None, 0, ctypes.byref(n)))
        out = np.zeros((n.value, 2))
        if n.value:
            N.check(N.lib().oems_sweep_get_trace(self._h, iid, out.ctypes.data_as(ctypes.POINTER(N.c_f64)),
                                                 n.value, ctypes.byref(n)))
        return out

    def stats(self):
        wall, cs = N.c_f64(), N.c_f64()
        N.check(N.lib().oems_sweep_stats(self._h, ctypes.byref(wall), ctypes.byref(cs)))
        return wall.value, cs.value


# ---------------------------------------------------------------------------
# several GPUs: instances split across ranks, results gathered once
# ---------------------------------------------------------------------------


def instance_cost(dims) -> float:
    """Relative cost of one instance: cells x (nx + ny + nz), since the
    steps to energy decay grow with the time light needs to cross the grid."""
    nx, ny, nz = dims
    return float(nx) * ny * nz * (nx + ny + nz)


def shard_instances(costs, world: int):
    """Instance indices per rank, longest first onto the least-loaded rank
    (ties to the lower index): deterministic, so every rank computes the
    same split without communicating.  Each list is in ascending order."""
    if world < 1:
        raise N.ConfigError("world size must be at least 1")
    load = [0.0] * world
    shards = [[] for _ in range(world)]
    for i in sorted(range(len(costs)), key=lambda i: (-costs[i], i)):
        r = min(range(world), key=lambda r: (load[r], r))
        shards[r].append(i)
        load[r] += costs[i]
    return [sorted(sh) for sh in shards]


def run_sharded(costs, run_local, dist=None, group=None):
    """Runs this rank's share of the instances and gathers every rank's
    results on rank 0, the only collective of the path.  `group` is the
    process group of the gather: give it a gloo group, so that a rank whose
    failure was a sticky CUDA error (its context unusable) can still report
    it; with NCCL the gather would move the objects through CUDA tensors.

    run_local(indices) -> (results {index: result}, wall_s, cell_steps).
    Rank 0 gets {"results": [result per instance, in index order], "wall_s":
    the slowest rank's wall time, "cell_steps": the sum, "shards": the
    split}; the other ranks get None.

    A rank whose share fails still joins the gather with its error, so no
    rank waits on it: rank 0 then raises OpenEMSError naming every failed
    rank, and the failed rank re-raises its own exception after the gather."""
    world = dist.get_world_size() if dist is not None else 1
    rank = dist.get_rank() if dist is not None else 0
    shards = shard_instances(costs, world)
    failure = None
    try:
        results, wall, cell_steps = run_local(shards[rank])
        if set(results) != set(shards[rank]):
            raise N.OpenEMSError(f"rank {rank} returned results for {sorted(results)}, expected {shards[rank]}")
        mine = {"results": results, "wall_s": float(wall), "cell_steps": int(cell_steps)}
    except Exception as e:  # reported through the gather, re-raised below
        failure = e
        mine = {"error": f"{type(e).__name__}: {e}"}
    if dist is None:
        if failure is not None:
            raise failure
        parts = [mine]
    else:
        parts = [None] * world if rank == 0 else None
        dist.gather_object(mine, parts, dst=0, group=group)
        if rank != 0:
            if failure is not None:
                raise failure
            return None
        failed = [(r, part["error"]) for r, part in enumerate(parts) if "error" in part]
        if failed:
            raise N.OpenEMSError("sweep failed on " + "; ".join(f"rank {r}: {msg}" for r, msg in failed))
    merged = {}
    for part in parts:
        merged.update(part["results"])
    return {"results": [merged[i] for i in range(len(costs))],
            "wall_s": max(part["wall_s"] for part in parts),
            "cell_steps": sum(part["cell_steps"] for part in parts), "shards": shards}


def main(argv=None):
    """Runs the seeded patch-antenna sweep and prints one JSON line:
    python -m openems_b200.sweep [--count 64] [--seed 4] [--concurrency 6]
    Under torchrun (WORLD_SIZE > 1) each rank runs its share of the
    instances on GPU LOCAL_RANK and rank 0 prints the whole job's line."""
    import argparse
    import datetime
    import json
    import os
    import time

    from . import workloads as W

    p = argparse.ArgumentParser(description="batched lumped-port sweep of seeded patch antennas")
    p.add_argument("--count", type=int, default=64)
    p.add_argument("--seed", type=int, default=4)
    p.add_argument("--concurrency", type=int, default=6)
    p.add_argument("--freqs", type=int, default=801, help="S11 points over 0-8 GHz")
    p.add_argument("--decay-db", type=float, default=50.0)
    p.add_argument("--max-steps", type=int, default=60000)
    p.add_argument("--batch-steps", type=int, default=2000)
    p.add_argument("--out", default=None, help="write S11 per instance to this .npz")
    p.add_argument("--storage", choices=("f32", "f16", "bf16"), default="f32", help="field storage")
    p.add_argument("--dist-timeout", type=float, default=900.0,
                   help="seconds a rank waits at the final gather (several GPUs)")
    a = p.parse_args(argv)
    freqs = np.linspace(0.0, 8e9, a.freqs)
    specs = W.patch_specs(a.count, seed=a.seed)
    world = int(os.environ.get("WORLD_SIZE", "1"))
    dist, device = None, -1
    if world > 1:
        import torch
        import torch.distributed as dist
        device = int(os.environ.get("LOCAL_RANK", "0"))
        torch.cuda.set_device(device)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=a.dist_timeout),
                                device_id=torch.device("cuda", device))
        # the results travel over gloo: host memory only, so a rank with a
        # broken CUDA context still delivers its error report
        gather_group = dist.new_group(backend="gloo", timeout=datetime.timedelta(seconds=a.dist_timeout))
    else:
        gather_group = None
    setup = [0.0]

    def run_local(indices):
        t0 = time.perf_counter()
        sw = Sweep(freqs, concurrency=a.concurrency, device=device, storage=a.storage)
        ids = {i: sw.add(W.patch_sweep_instance(specs[i], decay_db=a.decay_db, max_steps=a.max_steps))
               for i in indices}
        setup[0] = time.perf_counter() - t0
        sw.run(a.batch_steps)
        wall, cell_steps = sw.stats()
        out = {i: sw.result(iid) for i, iid in ids.items()}
        sw.close()
        return out, wall, cell_steps

    try:
        job = run_sharded([instance_cost(sp.dims) for sp in specs], run_local, dist, gather_group)
    finally:
        if dist is not None:
            dist.destroy_process_group()
    if job is None:
        return
    res, wall, cell_steps = job["results"], job["wall_s"], job["cell_steps"]
    s11_db = [20 * np.log10(np.maximum(np.abs(r["s11"][1:]), 1e-30)) for r in res]
    line = {
        "workload": f"patch_sweep_{a.count}_seed{a.seed}", "field_storage": a.storage,
        "instances": a.count, "concurrency": a.concurrency, "freqs": a.freqs, "ranks": world,
        "cell_steps": cell_steps, "wall_s": wall, "setup_s": setup[0],
        "mcells_per_s": cell_steps / wall / 1e6, "instances_per_hour": a.count / wall * 3600.0,
        "device_seconds_sum": sum(r["device_seconds"] for r in res),
        "decayed": sum(r["termination_reason"] == 1 for r in res),
        "timesteps_mean": float(np.mean([r["timesteps"] for r in res])),
        "timesteps_max": int(max(r["timesteps"] for r in res)),
        "min_s11_db_median": float(np.median([d.min() for d in s11_db])),
        "max_abs_s11": float(max(np.abs(r["s11"]).max() for r in res)),
        "instances_abs_s11_above_1.01": int(sum(np.abs(r["s11"]).max() > 1.01 for r in res)),
    }
    print(json.dumps(line))
    if a.out:
        np.savez(a.out, freqs=freqs, s11=np.array([r["s11"] for r in res]),
                 timesteps=np.array([r["timesteps"] for r in res]))


if __name__ == "__main__":
    main()
