"""Writes the golden fixtures of this directory: the oracle's results for a
few small scenarios of tests/scenarios.py, one .npz each, plus
manifest.json (dims, steps, SHA-256 of the field bytes).

    python tests/golden/make_golden.py

The reference (Rust) cannot be built or run here and stores no field arrays
of its own, so these are the oracle's outputs: they pin the oracle against
drift (tests/test_golden.py, CPU) and give the engine's GPU parity test
committed data to match (tests/test_gpu_golden.py).
"""
import hashlib
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(HERE))  # tests/
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))  # repository root

# small cases covering PEC, split batches, odd sizes, point probes, CPML, Mur and dispersive media
NAMES = ("small_grid", "batch_consistency", "odd_5x7x9", "nz_odd_33", "cpml_odd_asym", "mur2_partial",
         "drude_debye_cpml")


def scenarios_by_name():
    import scenarios as S
    all_sc = (S.reference_scenarios() + S.odd_scenarios() + S.cpml_scenarios() + [S.probe_scenario()]
              + S.mur_scenarios() + S.dispersive_scenarios())
    return {sc.name: sc for sc in all_sc}


def field_digest(fields: np.ndarray) -> str:
    return hashlib.sha256(np.ascontiguousarray(fields, dtype="<f4").tobytes()).hexdigest()


def main():
    import oracle
    import scenarios as S
    oracle.build()
    by_name = scenarios_by_name()
    manifest = {}
    for name in NAMES:
        sc = by_name[name]
        r = S.run_oracle(sc)
        energy = np.array(r["energy"], dtype=np.float64).reshape(-1, 4)
        arrays = {"fields": np.asarray(r["fields"], dtype=np.float32), "energy": energy,
                  "timestep": np.int64(r["timestep"])}
        if r["traces"] is not None:
            arrays["traces"] = np.asarray(r["traces"])
        np.savez_compressed(os.path.join(HERE, f"{name}.npz"), **arrays)
        manifest[name] = {"dims": list(sc.dims), "num_steps": sc.num_steps, "timestep": int(r["timestep"]),
                          "fields_sha256": field_digest(arrays["fields"]), "energy_samples": len(energy),
                          "traces": None if r["traces"] is None else list(np.shape(r["traces"]))}
        print(name, manifest[name]["fields_sha256"][:16])
    with open(os.path.join(HERE, "manifest.json"), "w") as f:
        json.dump({"generator": "python tests/golden/make_golden.py", "source": "oracle (FP32, BasicEngine semantics)",
                   "cases": manifest}, f, indent=1)
        f.write("\n")


if __name__ == "__main__":
    main()
