"""The oracle against the committed golden fixtures (tests/golden, written
by tests/golden/make_golden.py): fields, probe traces, energy samples and
the step counter bit for bit, and the field digests of the manifest."""
import json
import os

import numpy as np
import pytest

from scenarios import run_oracle

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
with open(os.path.join(GOLDEN, "manifest.json")) as _f:
    MANIFEST = json.load(_f)["cases"]


def load(name):
    with np.load(os.path.join(GOLDEN, f"{name}.npz")) as z:
        return {k: z[k] for k in z.files}


def scenario(name):
    import sys
    sys.path.insert(0, GOLDEN)
    from make_golden import scenarios_by_name
    return scenarios_by_name()[name]


@pytest.mark.parametrize("name", sorted(MANIFEST))
def test_fixture_matches_manifest(name):
    import hashlib
    g = load(name)
    m = MANIFEST[name]
    assert list(g["fields"].shape[1:]) == m["dims"] and g["fields"].shape[0] == 6
    assert hashlib.sha256(g["fields"].astype("<f4").tobytes()).hexdigest() == m["fields_sha256"]
    assert int(g["timestep"]) == m["timestep"] and len(g["energy"]) == m["energy_samples"]


@pytest.mark.parametrize("name", sorted(MANIFEST))
def test_oracle_reproduces_fixture(name):
    g = load(name)
    r = run_oracle(scenario(name))
    assert np.array_equal(np.asarray(r["fields"], np.float32).view(np.uint32), g["fields"].view(np.uint32))
    assert r["timestep"] == int(g["timestep"])
    assert np.array_equal(np.array(r["energy"], np.float64).reshape(-1, 4), g["energy"])
    if "traces" in g:
        assert np.array_equal(np.asarray(r["traces"]), g["traces"])
    else:
        assert r["traces"] is None
