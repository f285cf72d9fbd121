"""Staged early termination replayed on oracle runs (CPU): three short
patches of the small family run to -50 dB on the oracle, then the standard
and dense plans decide on them as staged_sweep would.  Also: the check's
shared pencil (one fit of the port voltage serving the end estimate and the
prediction) gives the same numbers as separate fits."""
import numpy as np
import pytest

from early_stop_offline import replay, run_instance
from openems_b200 import early_stop as ES
from openems_b200 import predictor as P

INDICES = (1, 7, 17)  # seed 5: 1801, 1901 and 2701 steps to -50 dB


@pytest.fixture(scope="module")
def records():
    specs = P.family_specs(max(INDICES) + 1, 5)
    return [run_instance(specs[i], threads=4) for i in INDICES]


def test_runs_are_complete(records):
    for rec in records:
        assert rec["trace"].shape == (rec["steps"], 2) and rec["steps"] < 4000
        assert rec["energy"][-1, 0] <= rec["steps"] and np.all(np.abs(rec["s11"]) <= 1.0 + 5e-3)


@pytest.mark.parametrize("plan", [ES.StagePlan(tau=0.05), ES.StagePlan.dense()], ids=["standard", "dense"])
def test_replay_stops_only_within_half_a_db(records, plan):
    r = replay(records, plan)
    assert r["predicted"] + r["decayed"] + r["full"] == len(records)
    assert all(s <= rec["steps"] for s, rec in zip(r["steps"], records))
    assert r["max_err_db"] < 0.5 and r["step_ratio"] >= 1.0


def test_shared_pencil_matches_separate_fits(records):
    rec = max(records, key=lambda x: x["steps"])
    tr, dt, K = rec["trace"], rec["dt"], 1536
    plan = ES.StagePlan.dense()
    pen = plan.pencil(K)
    r = {"uf": P.head_dft(tr[:K, 0], 1, dt, P.FREQS, 0.0), "if": P.head_dft(tr[:K, 1], 1, dt, P.FREQS, 0.5),
         "final_decay_db": -20.0}
    pred, d, end = ES.check_instance(tr, r, K, dt, P.FREQS, P.HORIZON, 50.0, plan)
    end2 = max(ES.plain_end(tr[:, 0], K, -20.0, dt, 50.0, P.HORIZON, **pen), K)
    a = ES.pencil_s11(tr, r["uf"], r["if"], K, dt, P.FREQS, end2, 0, **pen)
    b = ES.pencil_s11(tr, r["uf"], r["if"], K, dt, P.FREQS, end2, plan.lag, **pen)
    assert end == end2 and np.array_equal(pred, a)
    assert d == ES.s11_db_error(a, b, plan.band(P.FREQS))


def test_dense_plan():
    p = ES.StagePlan.dense()
    assert p.stages[0] == 1024 and p.stages[-1] == 24576 and len(p.stages) == 10
    assert (p.samples, p.max_modes, p.tau, p.check) == (512, 150, 0.1, "max")
    assert ES.StagePlan.dense(tau=0.2, check="mean").tau == 0.2
    assert p.pencil(24576) == {"window": 12288, "decimate": 24, "max_modes": 150}
