"""The learned part of the staged early stop: a network that predicts, at a
stage K, how far the matrix-pencil continuation's S11 is from the full run.

The staged early stop (early_stop.py) pauses every instance at K steps and
continues its port traces with the pencil's damped sinusoids.  Whether to
trust that continuation was decided by a residual check alone: predictions
from windows ending K and K - 256 steps agree within tau dB.  This network
makes the decision from more of what is known at K:

    input   the pencil window of the port voltage and current (the last
            0.75 K steps, at most 12288, decimated to 256 samples, each
            channel divided by its largest magnitude), channels padded to 8
    tcn     4 causal conv layers, kernel 5, dilations 1 4 16 64, 128
            channels, ReLU (receptive field 341 samples: the whole window),
            read at the last sample
    scalars the residual check (largest and mean |dB| difference over the
            band, and the largest against the prediction from a window 1024
            steps earlier), the prediction's sensitivity to its tail (its
            largest |dB| change when the continuation is scaled by 1.1), the
            energy level below the peak, log K, the continuation's end step
            over K
    mlp     (128 + 8) -> 256 (ReLU) -> 8; output 0 is log10(error + 0.01),
            error = the largest |dB(S11_pred) - dB(S11_full)| over the band

An instance is accepted at the first stage whose predicted error is below a
threshold chosen on held-back validation instances of the training family
(the largest one that keeps every validation instance within 0.5 dB, assessed
on the network's out-of-sample predictions).  Every product (forward, input and weight
gradients) is oems_tc_gemm_bf16 (tcgen05, bf16 operands, f32 accumulation);
the causal convolutions are oems_pk_im2col_causal / col2im_causal, the rest
oems_pk_* kernels; torch only holds device buffers.  The float64 restatement
is oracle/tailnet_ref.StageNetRef (tests only).

The network of predictor_net.py maps the head of the traces to the tail's
modal amplitudes directly; trained on 2,000 small patches it ended up worse
than plain truncation, while the pencil's continuation is accurate for most
instances and fails for a few.  Telling those apart is what the learning is
for here.
"""
from __future__ import annotations

from dataclasses import dataclass
from typing import Optional

import numpy as np

from . import predictor as P
from .predictor_net import Dense, _chk, _p, _torch, bf16, relu_, relu_bwd_

T_WIN = 256        # samples of the decimated pencil window fed to the TCN
C_IN = 8           # input channels: u, i, padding
N_SCALAR = 8
LOG_FLOOR = 0.01   # dB added before the log10 of the error


def window_input(trace: np.ndarray, K: int, window: int) -> np.ndarray:
    """(T_WIN, C_IN) float32: the window of u and i that ends at K,
    decimated to T_WIN samples ending at K - 1 (zeros before its start),
    each channel divided by its largest magnitude there."""
    dec = max(1, window // T_WIN)
    w = trace[max(0, K - window):K]
    w = w[::-1][::dec][::-1][-T_WIN:]
    out = np.zeros((T_WIN, C_IN), dtype=np.float32)
    sc = np.maximum(np.abs(w).max(axis=0), 1e-30)
    out[T_WIN - len(w):, :2] = (w / sc).astype(np.float32)
    return out


def scalar_input(check_max: float, check_mean: float, check_far: float, tail_sens: float, level_db: float,
                 K: int, end: int) -> np.ndarray:
    """(N_SCALAR,) float32 of the pencil diagnostics at stage K: the
    residual check (largest and mean |dB| over the band, and the largest
    against a window 1024 steps earlier), the prediction's sensitivity to
    its continuation (largest |dB| change when the tail is scaled by 1.1),
    the energy level below the peak, log K and the estimated remaining run."""
    lg = lambda v: np.log10(v + LOG_FLOOR)  # noqa: E731
    return np.array([lg(check_max), lg(check_mean), lg(check_far), lg(tail_sens), level_db / 50.0,
                     np.log2(K / 1024.0) / 5.0, min(end / K, 32.0) / 8.0, 1.0], dtype=np.float32)


class CausalConv:
    """Causal dilated conv1d over (B, T, C) f32 as im2col + Dense; the output
    keeps the length T."""

    def __init__(self, cin, cout, ks, dil, rng):
        self.cin, self.cout, self.ks, self.dil = cin, cout, ks, dil
        self.width = ks * cin
        assert self.width % 8 == 0
        self.fc = Dense(self.width, cout, rng)

    def forward(self, x):
        torch = _torch()
        B, T, C = x.shape
        from . import _native as N
        cols = torch.empty(B * T, self.width, dtype=torch.bfloat16, device="cuda")
        _chk(N.lib().oems_pk_im2col_causal(_p(x), _p(cols), B, T, C, self.ks, self.dil, self.width, None))
        y = self.fc.forward(cols)
        return y.view(B, T, self.cout), cols

    def backward(self, dy, cols, x_shape, need_dx=True):
        torch = _torch()
        from . import _native as N
        B, T, C = x_shape
        dcols = self.fc.backward(dy.reshape(-1, self.cout), cols, need_dx)
        if not need_dx:
            return None
        dx = torch.empty(B, T, C, dtype=torch.float32, device="cuda")
        _chk(N.lib().oems_pk_col2im_causal(_p(dcols), self.width, _p(dx), B, T, C, self.ks, self.dil, None))
        return dx


@dataclass
class StageNetConfig:
    channels: int = 128
    layers: int = 4
    kernel: int = 5
    hidden: int = 256
    batch: int = 256
    lr: float = 1e-3
    epochs: int = 60
    seed: int = 0


class StageNet:
    def __init__(self, cfg: StageNetConfig = StageNetConfig()):
        rng = np.random.default_rng(cfg.seed)
        self.cfg = cfg
        cin = [C_IN] + [cfg.channels] * (cfg.layers - 1)
        self.convs = [CausalConv(cin[l], cfg.channels, cfg.kernel, 4 ** l, rng) for l in range(cfg.layers)]
        self.fc1 = Dense(cfg.channels + N_SCALAR, cfg.hidden, rng)
        self.fc2 = Dense(cfg.hidden, 8, rng, scale=1e-2)
        self.step_no = 0
        self.threshold: Optional[float] = None  # log10 error below which a stage is accepted
        self._partial = _torch().zeros(256, dtype=_torch().float64, device="cuda")

    def dense_layers(self):
        return [c.fc for c in self.convs] + [self.fc1, self.fc2]

    def forward(self, x, s):
        """x (B, T_WIN, C_IN) f32, s (B, N_SCALAR) f32 -> (B, 8) f32; keeps
        the activations for backward."""
        torch = _torch()
        acts = []
        h = x
        for c in self.convs:
            y, cols = c.forward(h)
            relu_(y)
            acts.append((h.shape, cols, y))
            h = y
        B = x.shape[0]
        feat = torch.cat([h[:, -1, :], s], dim=1).contiguous()
        fb = bf16(feat)
        z1 = self.fc1.forward(fb)
        z1b = relu_(z1)
        out = self.fc2.forward(z1b)
        self._cache = (acts, fb, z1, z1b, B)
        return out

    def backward(self, dout):
        torch = _torch()
        acts, fb, z1, z1b, B = self._cache
        dz1 = self.fc2.backward(dout, z1b)
        relu_bwd_(dz1, z1)
        dfeat = self.fc1.backward(dz1, fb)
        # only the last time step of the TCN output reaches the head
        shape_last = acts[-1][2].shape
        dh = torch.zeros(shape_last, dtype=torch.float32, device="cuda")
        dh[:, -1, :] = dfeat[:, :self.cfg.channels]
        for idx in range(len(self.convs) - 1, -1, -1):
            shape, cols, y = acts[idx]
            relu_bwd_(dh, y)
            dh = self.convs[idx].backward(dh, cols, shape, need_dx=idx > 0)

    def predict(self, x: np.ndarray, s: np.ndarray) -> np.ndarray:
        """Predicted log10(error dB + 0.01) per row (numpy in, numpy out)."""
        torch = _torch()
        out = []
        for a in range(0, len(x), 1024):
            xt = torch.tensor(x[a:a + 1024], dtype=torch.float32, device="cuda")
            st = torch.tensor(s[a:a + 1024], dtype=torch.float32, device="cuda")
            out.append(self.forward(xt, st)[:, 0].cpu().numpy())
        return np.concatenate(out) if out else np.zeros(0)

    # -- weights ------------------------------------------------------------
    def state(self) -> dict:
        d = {}
        for k, layer in enumerate(self.dense_layers()):
            d[f"w{k}"] = layer.w.cpu().numpy()
            d[f"b{k}"] = layer.b.cpu().numpy()
        d["threshold"] = np.array([np.nan if self.threshold is None else self.threshold])
        return d

    def load(self, d: dict):
        torch = _torch()
        for k, layer in enumerate(self.dense_layers()):
            layer.w.copy_(torch.tensor(np.asarray(d[f"w{k}"], dtype=np.float32)))
            layer.b.copy_(torch.tensor(np.asarray(d[f"b{k}"], dtype=np.float32)))
            bf16(layer.w, out=layer.wb)
        t = float(np.asarray(d["threshold"]).reshape(-1)[0])
        self.threshold = None if np.isnan(t) else t
        return self


def train(x, s, y, cfg: StageNetConfig = StageNetConfig(), log=print, val=None) -> StageNet:
    """Fits the network to log10(error + 0.01) targets y (n,) on the GPU:
    Adam on the squared error of output 0 (outputs 1..7 carry no loss).
    With val = (x, s, y) of held-out instances, keeps the weights of the
    epoch with the lowest validation loss (early stopping)."""
    torch = _torch()
    net = StageNet(cfg)
    n = len(x)
    xt = torch.tensor(x, dtype=torch.float32, device="cuda")
    st = torch.tensor(s, dtype=torch.float32, device="cuda")
    yt = torch.tensor(y, dtype=torch.float32, device="cuda")
    rng = np.random.default_rng(cfg.seed + 1)
    B = min(cfg.batch, n)
    best, best_loss = None, np.inf
    for ep in range(cfg.epochs):
        perm = rng.permutation(n)
        losses = []
        for a in range(0, n - B + 1, B):
            idx = torch.tensor(perm[a:a + B], device="cuda")
            losses.append(train_step(net, xt[idx].contiguous(), st[idx].contiguous(), yt[idx].contiguous()))
        vloss = None
        if val is not None:
            vloss = float(np.mean((net.predict(val[0], val[1]) - val[2]) ** 2))
            if vloss < best_loss:
                best_loss, best = vloss, net.state()
        if log and (ep % 10 == 0 or ep == cfg.epochs - 1):
            log(f"epoch {ep}: loss {np.mean(losses):.4f}" + ("" if vloss is None else f", validation {vloss:.4f}"))
    if best is not None:
        net.load(best)
        net.best_validation_loss = best_loss
    return net


def train_step(net: StageNet, x, s, y):
    """One Adam step on the mean squared error of output 0; returns it."""
    from . import _native as N
    torch = _torch()
    out = net.forward(x, s)
    # outputs 1..7 are unused: their target is the output itself (no gradient)
    t = out.detach().clone()
    t[:, 0] = y
    g = torch.empty_like(out)
    _chk(N.lib().oems_pk_mse(_p(out), _p(t), None, _p(g), out.shape[0], out.shape[1], _p(net._partial), 256, None))
    net.backward(g)
    net.step_no += 1
    for layer in net.dense_layers():
        layer.step(net.cfg.lr, net.step_no)
    return float(net._partial.sum().item()) / out.shape[0]


def choose_threshold(pred: np.ndarray, err: np.ndarray, stage_of: np.ndarray, inst_of: np.ndarray,
                     limit_db: float = 0.5, n_cand: int = 400) -> float:
    """Largest threshold on the predicted log error (over n_cand quantiles
    of the predictions) whose first-accept rule keeps every instance's
    error within limit_db; -inf if none does."""
    best = -np.inf
    for thr in np.unique(np.quantile(pred, np.linspace(0.0, 1.0, n_cand))):
        if first_accept(pred, err, stage_of, inst_of, thr)[1] <= limit_db:
            best = max(best, float(thr))
    return best


def first_accept(pred, err, stage_of, inst_of, thr):
    """({instance: first accepted stage index}, worst error of the accepted
    predictions); rows are (instance, stage) records with a prediction."""
    acc = {}
    worst = 0.0
    for r in np.lexsort((stage_of, inst_of)):
        i = int(inst_of[r])
        if i in acc:
            continue
        if pred[r] < thr:
            acc[i] = int(stage_of[r])
            worst = max(worst, float(err[r]))
    return acc, worst


# ---------------------------------------------------------------------------
# data, training and evaluation on a patch family (GPU)
# ---------------------------------------------------------------------------


def rows(cal: dict):
    """Flattens calibration records (early_stop.calibrate with features) to
    the (instance, stage) pairs that have a prediction: inputs x (m, T_WIN,
    C_IN), s (m, N_SCALAR), the prediction's error (dB), stage and instance."""
    e = cal["error_db"]
    inst, stage = np.nonzero(~np.isnan(e))
    x = np.zeros((len(inst), T_WIN, C_IN), dtype=np.float32)
    x[:, :, :2] = cal["x"][inst, stage].astype(np.float32)
    return x, cal["s"][inst, stage].astype(np.float32), e[inst, stage], stage, inst


def evaluate(score, thr, err, stage_of, inst_of, stages, steps_full, limit_db: float = 0.5) -> dict:
    """Outcome of accepting at the first stage with score < thr: the step
    ratio against the plain runs, how many were accepted, the largest
    accepted error and how many exceed limit_db."""
    acc, worst = first_accept(score, err, stage_of, inst_of, thr)
    n = len(steps_full)
    steps = np.array([stages[acc[k]] if k in acc else steps_full[k] for k in range(n)], dtype=np.float64)
    by = {(int(i), int(s)): float(e) for e, s, i in zip(err, stage_of, inst_of)}
    errs = np.array([by[(k, acc[k])] for k in acc]) if acc else np.zeros(0)
    return {"threshold": float(thr), "step_ratio": float(np.sum(steps_full) / np.sum(steps)),
            "accepted": len(acc), "max_err_db": float(worst),
            "over_limit": int((errs > limit_db).sum()), "steps_mean": float(steps.mean())}


def tradeoff(score, err, stage_of, inst_of, stages, steps_full, budgets=(0, 0.01, 0.02, 0.05)) -> list:
    """For each violation budget (fraction of instances allowed above 0.5
    dB), the largest threshold that meets it on these records and the step
    ratio it gives: a rule's operating curve, for comparing rules at equal
    error."""
    n = len(steps_full)
    out = []
    cands = np.unique(np.quantile(score, np.linspace(0.0, 1.0, 400)))
    for b in budgets:
        allowed = int(np.floor(b * n + 1e-9))
        best = None
        for thr in cands:
            r = evaluate(score, thr, err, stage_of, inst_of, stages, steps_full)
            if r["over_limit"] <= allowed and (best is None or r["step_ratio"] > best["step_ratio"]):
                best = r
        out.append({"budget": b, "allowed": allowed, **(best or {"step_ratio": 1.0})})
    return out


def records(family, count, seed, plan, concurrency, log, t0):
    """Records of `count` instances of `family` (seed `seed`): the full runs
    give each instance's reference S11 and step count ("steps_full"), then
    early_stop.calibrate with features runs them through every stage of
    `plan`.  log(msg) reports the elapsed time since perf_counter() t0."""
    import time
    from . import early_stop as ES
    insts, freqs = ES.family_instances(family, count, seed)
    full = ES.full_sweep(insts, freqs, concurrency)
    fs11 = [r["s11"] for r in full["results"]]
    insts, _ = ES.family_instances(family, count, seed)
    cal = ES.calibrate(insts, freqs, plan, fs11, concurrency, features=True)
    cal["steps_full"] = np.array([r["timesteps"] for r in full["results"]], dtype=np.float64)
    if log:
        log(f"{family} seed {seed}: {count} instances recorded ({time.perf_counter() - t0:.0f} s)")
    return cal


def _concat(a: dict, b: dict) -> dict:
    """Records of two families as one (instances of b after those of a;
    they share the stage list)."""
    return {k: np.concatenate([a[k], b[k]]) for k in a}


def learn(train_count: int = 1500, test_count: int = 400, family: str = "small", train_seed: int = 5,
          test_seed: int = 50, extra_patch: int = 0, val_frac: float = 0.2,
          cfg: StageNetConfig = StageNetConfig(), concurrency: int = 16, log=print, reuse: Optional[str] = None,
          patch_seed: Optional[int] = None):
    """Generates the records with the batched engine (full runs for the
    reference S11, then every instance through every stage of the dense
    plan): train_count instances of `family` (plus extra_patch of the
    64-patch sweep family, seed train_seed + 1) for training and test_count
    held out.  A val_frac share of the training instances is held back for
    validation: early stopping, and both rules' thresholds are chosen on the
    validation instances' out-of-sample scores (the largest threshold
    keeping every validation instance within 0.5 dB, and within a 1%
    budget).  reuse: a directory with the records an earlier run saved
    (stage_records_train.npz / _test.npz), used instead of recording them
    again; extra_patch instances (seed patch_seed, default train_seed + 1)
    are then recorded and added to its training records.  Returns (net,
    report, train records, test records)."""
    import time
    from . import early_stop as ES
    plan = ES.StagePlan.dense()
    t0 = time.perf_counter()
    if reuse:
        import os
        with np.load(os.path.join(reuse, "stage_records_train.npz")) as d:
            rtr = {k: d[k] for k in d.files}
        with np.load(os.path.join(reuse, "stage_records_test.npz")) as d:
            rte = {k: d[k] for k in d.files}
    else:
        rtr = records(family, train_count, train_seed, plan, concurrency, log, t0)
    if extra_patch:
        ps = train_seed + 1 if patch_seed is None else patch_seed
        rtr = _concat(rtr, records("patch", extra_patch, ps, plan, concurrency, log, t0))
    if not reuse:
        rte = records(family, test_count, test_seed, plan, concurrency, log, t0)
    x, sc, e, sg, it = rows(rtr)
    n_inst = len(rtr["steps_full"])
    rng = np.random.default_rng(cfg.seed + 7)
    val_inst = rng.permutation(n_inst)[:int(round(val_frac * n_inst))]
    is_val = np.isin(it, val_inst)
    y = np.log10(e + LOG_FLOOR)
    t1 = time.perf_counter()
    net = train(x[~is_val], sc[~is_val], y[~is_val], cfg, log=log, val=(x[is_val], sc[is_val], y[is_val]))
    train_s = time.perf_counter() - t1
    stages = list(plan.stages)
    # validation records, instances renumbered 0..v-1
    vmap = {int(k): j for j, k in enumerate(sorted(val_inst))}
    vi = np.array([vmap[int(k)] for k in it[is_val]])
    vsteps = rtr["steps_full"][sorted(val_inst)]
    pv = net.predict(x[is_val], sc[is_val])
    cv = np.log10(rtr["check_db"][it[is_val], sg[is_val]] + LOG_FLOOR)
    ev, sv = e[is_val], sg[is_val]

    def thr_for(score, budget):
        allowed = int(np.floor(budget * len(vsteps) + 1e-9))
        best = -np.inf
        for thr in np.unique(np.quantile(score, np.linspace(0.0, 1.0, 400))):
            if evaluate(score, thr, ev, sv, vi, stages, vsteps)["over_limit"] <= allowed:
                best = max(best, float(thr))
        return best

    xte, ste, ete, sgte, itte = rows(rte)
    pte = net.predict(xte, ste)
    cte = np.log10(rte["check_db"][itte, sgte] + LOG_FLOOR)
    sf = rte["steps_full"]
    deployed = {}
    for budget in (0.0, 0.01):
        tn, tc = thr_for(pv, budget), thr_for(cv, budget)
        deployed[str(budget)] = {"network": evaluate(pte, tn, ete, sgte, itte, stages, sf),
                                 "residual_check": evaluate(cte, tc, ete, sgte, itte, stages, sf)}
    net.threshold = thr_for(pv, 0.0)
    report = {
        "family": family, "train": train_count, "extra_patch": extra_patch, "test": test_count,
        "reused_records": reuse is not None, "patch_seed": train_seed + 1 if patch_seed is None else patch_seed,
        "train_seed": train_seed, "test_seed": test_seed, "validation_instances": int(len(val_inst)),
        "stages": stages, "records_train": int((~is_val).sum()), "records_validation": int(is_val.sum()),
        "records_test": int(len(ete)), "train_seconds": train_s, "epochs": cfg.epochs,
        "best_validation_loss": float(getattr(net, "best_validation_loss", np.nan)),
        "deployed_thresholds_from_validation": deployed,
        "tradeoff_test": {"network": tradeoff(pte, ete, sgte, itte, stages, sf),
                          "residual_check": tradeoff(cte, ete, sgte, itte, stages, sf)},
        # the best any rule can do: accept each instance at its first stage within 0.5 dB
        "perfect_rule_test": evaluate(np.where(ete <= 0.5, -1.0, 1.0), 0.0, ete, sgte, itte, stages, sf),
        "pred_corr_test": float(np.corrcoef(pte, np.log10(ete + LOG_FLOOR))[0, 1]),
    }
    return net, report, rtr, rte


def default_weights_path() -> str:
    import os
    return os.path.join(os.path.dirname(os.path.abspath(__file__)), "data", "stage_net.npz")


def load_default() -> Optional[StageNet]:
    """The committed trained network, or None if there is none."""
    import os
    path = default_weights_path()
    if not os.path.exists(path):
        return None
    with np.load(path) as d:
        return StageNet().load({k: d[k] for k in d.files})


def main(argv=None):
    """python -m openems_b200.stage_net learn [--train N] [--test M]
    [--out DIR]: records, trains and evaluates on the GPU; prints one JSON
    line and writes DIR/stage_net.npz (weights and threshold, float32)."""
    import argparse
    import json
    import os
    p = argparse.ArgumentParser()
    p.add_argument("cmd", choices=["learn"])
    p.add_argument("--train", type=int, default=1500)
    p.add_argument("--test", type=int, default=400)
    p.add_argument("--family", choices=["small", "patch"], default="small")
    p.add_argument("--extra-patch", type=int, default=0,
                   help="also train on this many instances of the 64-patch sweep family")
    p.add_argument("--epochs", type=int, default=StageNetConfig.epochs)
    p.add_argument("--concurrency", type=int, default=16)
    p.add_argument("--out", default=".")
    p.add_argument("--save-records", action="store_true", help="also write the records (.npz, float16 windows)")
    p.add_argument("--reuse", default=None, help="directory of an earlier run's saved records, used instead")
    p.add_argument("--patch-seed", type=int, default=None, help="seed of the --extra-patch instances")
    a = p.parse_args(argv)
    cfg = StageNetConfig(epochs=a.epochs)
    net, report, rtr, rte = learn(a.train, a.test, a.family, extra_patch=a.extra_patch, cfg=cfg,
                                  concurrency=a.concurrency, log=lambda m: print(m, flush=True), reuse=a.reuse,
                                  patch_seed=a.patch_seed)
    os.makedirs(a.out, exist_ok=True)
    np.savez(os.path.join(a.out, "stage_net.npz"), **net.state())
    if a.save_records:
        for name, r in (("train", rtr), ("test", rte)):
            np.savez_compressed(os.path.join(a.out, f"stage_records_{name}.npz"), **r)
    print(json.dumps(report))


if __name__ == "__main__":
    main()
