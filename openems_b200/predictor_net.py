"""The early-termination network on the engine library's tensor-core kernels.

    input  (B, K, 2)  port u and i of the first K steps, each channel scaled by
                      its largest magnitude in those steps
    conv   k 8 / s 4: 2 -> 32 -> 64 -> 64 channels, ReLU   (B, 30, 64 at K 2048)
    mlp    1920 -> 512 (ReLU) -> 256: 64 complex modal coefficients per channel
    fixed  256 -> 4 F: the tail's DFT at F frequencies (predictor.tail_matrix)

Training minimises the mean squared error of the scaled tail DFT.  Every
product (forward, input gradients and weight gradients) is a call of
oems_tc_gemm_bf16 (tcgen05, bf16 operands, f32 accumulation); the other steps
are the oems_pk_* kernels.  torch provides device buffers only.
"""
from __future__ import annotations

import ctypes
import time
from dataclasses import dataclass

import numpy as np

from . import _native as N
from . import predictor as P


def _torch():
    import torch
    return torch


def _p(t):
    return ctypes.c_void_p(t.data_ptr()) if t is not None else None


def _chk(st):
    N.check(st)


def gemm(a, b, c, bias=None, beta=0.0):
    """c[M, n] = a[M, K] b[n, K]^T (+ beta c) (+ bias); a, b bf16 row-major."""
    M, K = a.shape
    n = b.shape[0]
    _chk(N.lib().oems_tc_gemm_bf16(_p(a), a.stride(0), _p(b), b.stride(0), _p(c), c.stride(0), M, n, K,
                                   float(beta), _p(bias), None))


def bf16(x, out=None):
    torch = _torch()
    if out is None:
        out = torch.empty(x.shape, dtype=torch.bfloat16, device=x.device)
    _chk(N.lib().oems_pk_f32_to_bf16(_p(x), _p(out), x.numel(), None))
    return out


def transpose(xb):
    torch = _torch()
    R, C = xb.shape
    out = torch.empty(C, R, dtype=torch.bfloat16, device=xb.device)
    _chk(N.lib().oems_pk_transpose_bf16(_p(xb), xb.stride(0), _p(out), out.stride(0), R, C, None))
    return out


class Dense:
    """y = x W^T + b with f32 master weights, bf16 copies and Adam state."""

    def __init__(self, n_in, n_out, rng, scale=None, trainable=True, weight=None):
        torch = _torch()
        if weight is None:
            s = scale if scale is not None else np.sqrt(2.0 / n_in)
            weight = rng.normal(0.0, s, size=(n_out, n_in))
        self.w = torch.tensor(weight, dtype=torch.float32, device="cuda")
        self.b = torch.zeros(n_out, dtype=torch.float32, device="cuda")
        self.wb = bf16(self.w)
        self.trainable = trainable
        if trainable:
            self.state = [torch.zeros_like(self.w), torch.zeros_like(self.w), torch.zeros_like(self.b),
                          torch.zeros_like(self.b)]
            self.gw = torch.zeros_like(self.w)
            self.gb = torch.zeros_like(self.b)

    def forward(self, xb):
        torch = _torch()
        y = torch.empty(xb.shape[0], self.w.shape[0], dtype=torch.float32, device="cuda")
        gemm(xb, self.wb, y, bias=self.b if self.trainable else None)
        return y

    def backward(self, dy, xb, need_dx=True):
        """Weight gradients from dy (rows x out, f32) and the layer input xb
        (rows x in, bf16); returns dx (rows x in, f32) when asked."""
        torch = _torch()
        dyb = bf16(dy)
        if self.trainable:
            gemm(transpose(dyb), transpose(xb), self.gw)           # dW = dy^T x
            _chk(N.lib().oems_pk_colsum(_p(dy), dy.shape[0], dy.shape[1], _p(self.gb), None))
        if not need_dx:
            return None
        dx = torch.empty(xb.shape[0], self.w.shape[1], dtype=torch.float32, device="cuda")
        gemm(dyb, transpose(self.wb), dx)                           # dx = dy W
        return dx

    def step(self, lr, t, wd=1e-4):
        if not self.trainable:
            return
        mw, vw, mb, vb = self.state
        _chk(N.lib().oems_pk_adam(_p(self.w), _p(self.wb), _p(self.gw), _p(mw), _p(vw), self.w.numel(), lr, 0.9,
                                  0.999, 1e-8, wd, t, None))
        _chk(N.lib().oems_pk_adam(_p(self.b), None, _p(self.gb), _p(mb), _p(vb), self.b.numel(), lr, 0.9, 0.999,
                                  1e-8, 0.0, t, None))


class Conv:
    """Strided valid conv1d over (B, T, C) activations as im2col + Dense."""

    def __init__(self, cin, cout, ks, stride, rng):
        self.cin, self.cout, self.ks, self.s = cin, cout, ks, stride
        self.width = ks * cin
        assert self.width % 8 == 0
        self.fc = Dense(self.width, cout, rng)

    def tout(self, T):
        return (T - self.ks) // self.s + 1

    def forward(self, x):
        """x: (B, T, C) f32 -> (B, Tout, Cout) f32 (before the activation)."""
        torch = _torch()
        B, T, C = x.shape
        To = self.tout(T)
        cols = torch.empty(B * To, self.width, dtype=torch.bfloat16, device="cuda")
        _chk(N.lib().oems_pk_im2col(_p(x), _p(cols), B, T, C, self.ks, self.s, self.width, None))
        y = self.fc.forward(cols)
        return y.view(B, To, self.cout), cols

    def backward(self, dy, cols, x_shape, need_dx=True):
        torch = _torch()
        B, T, C = x_shape
        dcols = self.fc.backward(dy.reshape(-1, self.cout), cols, need_dx)
        if not need_dx:
            return None
        dx = torch.empty(B, T, C, dtype=torch.float32, device="cuda")
        _chk(N.lib().oems_pk_col2im(_p(dcols), self.width, _p(dx), B, T, C, self.ks, self.s, None))
        return dx


def relu_(y):
    """In place; returns the bf16 copy."""
    torch = _torch()
    flat = y.reshape(-1, y.shape[-1])
    yb = torch.empty(flat.shape, dtype=torch.bfloat16, device="cuda")
    _chk(N.lib().oems_pk_relu(_p(flat), _p(yb), flat.shape[0], flat.shape[1], yb.stride(0), None))
    return yb


def relu_bwd_(dy, y):
    _chk(N.lib().oems_pk_relu_bwd(_p(dy), _p(y), dy.numel(), None))


@dataclass
class NetConfig:
    K: int = P.K_DEFAULT
    channels: tuple = (32, 64, 64)
    hidden: int = 512
    modes: int = 64
    batch: int = 256
    lr: float = 1e-3
    epochs: int = 300
    seed: int = 0


class TailNet:
    def __init__(self, cfg: NetConfig, freqs: np.ndarray, horizon: int = P.HORIZON, row_scale=None,
                 fmin_loss: float = 0.0):
        torch = _torch()
        rng = np.random.default_rng(cfg.seed)
        self.cfg = cfg
        ch = (2,) + tuple(cfg.channels)
        self.convs = [Conv(ch[i], ch[i + 1], 8, 4, rng) for i in range(len(cfg.channels))]
        T = cfg.K
        for c in self.convs:
            T = c.tout(T)
        self.T_last = T
        self.flat = T * ch[-1]
        self.fc1 = Dense(self.flat, cfg.hidden, rng)
        self.fc2 = Dense(cfg.hidden, 4 * cfg.modes, rng, scale=1e-3)
        # fixed spectral layer: block-diagonal (u, i) tail matrices, rows padded to a multiple of 8
        dt = P.grid_dt()
        poles = P.PoleGrid().poles()[:cfg.modes]
        self.F = len(freqs)
        Tu = P.tail_matrix(poles, cfg.K, dt, freqs, 0.0, horizon)
        Ti = P.tail_matrix(poles, cfg.K, dt, freqs, 0.5, horizon)
        rows = 4 * self.F
        self.rows = (rows + 7) // 8 * 8
        Tm = np.zeros((self.rows, 4 * cfg.modes))
        Tm[:2 * self.F, :2 * cfg.modes] = Tu
        Tm[2 * self.F:4 * self.F, 2 * cfg.modes:] = Ti
        # output rows: frequencies below fmin_loss carry no weight; the rest
        # are divided by row_scale (the RMS of each row's target over the
        # training set) so that every frequency counts alike in the loss
        keep = np.tile(np.asarray(freqs) >= fmin_loss, 4)
        self.row_scale = np.ones(self.rows)
        if row_scale is not None:
            self.row_scale[:4 * self.F] = row_scale
        self.row_w = np.zeros(self.rows)
        self.row_w[:4 * self.F] = keep / self.row_scale[:4 * self.F]
        Tw = Tm * self.row_w[:, None]
        self.t_scale = float(np.abs(Tw).max())
        self.spec = Dense(4 * cfg.modes, self.rows, rng, trainable=False, weight=Tw / self.t_scale)
        self.step_no = 0
        self._partial = torch.zeros(256, dtype=torch.float64, device="cuda")

    def layers(self):
        return self.convs + [self.fc1, self.fc2]

    def forward(self, x):
        """x: (B, K, 2) f32 -> (B, rows) predicted scaled tail DFT; keeps the
        activations for backward."""
        acts = []
        h = x
        for c in self.convs:
            y, cols = c.forward(h)
            relu_(y)
            acts.append((h.shape, cols, y))
            h = y
        hb = bf16(h.reshape(h.shape[0], -1).contiguous())
        z1 = self.fc1.forward(hb)
        z1b = relu_(z1)
        coef = self.fc2.forward(z1b)
        coefb = bf16(coef)
        out = self.spec.forward(coefb)
        self._cache = (acts, hb, z1, z1b, coefb)
        return out

    def backward(self, dout):
        acts, hb, z1, z1b, coefb = self._cache
        dcoef = self.spec.backward(dout, coefb)
        dz1 = self.fc2.backward(dcoef, z1b)
        relu_bwd_(dz1, z1)
        dh = self.fc1.backward(dz1, hb).view(acts[-1][2].shape)
        for idx in range(len(self.convs) - 1, -1, -1):
            shape, cols, y = acts[idx]
            relu_bwd_(dh, y)
            dh = self.convs[idx].backward(dh, cols, shape, need_dx=idx > 0)

    def train_step(self, x, target):
        torch = _torch()
        out = self.forward(x)
        g = torch.empty_like(out)
        _chk(N.lib().oems_pk_mse(_p(out), _p(target), None, _p(g), out.shape[0], out.shape[1], _p(self._partial),
                                 256, None))
        self.backward(g)
        self.step_no += 1
        for layer in self.layers():
            (layer.fc if isinstance(layer, Conv) else layer).step(self.cfg.lr, self.step_no)
        return float(self._partial.sum().item()) / out.numel()


def scaled_tails(ds: dict, K: int):
    """Inputs (n, K, 2), each channel divided by its largest |value| in the
    first K steps, the tail DFTs (n, 4 F) in the same scale, and the scales."""
    head = ds["head"][:, :, :K].astype(np.float64)
    sc = np.maximum(np.abs(head).max(axis=2), 1e-30)          # (n, 2)
    x = (head / sc[:, :, None]).transpose(0, 2, 1).astype(np.float32)
    F = ds["tail"].shape[2]
    t = np.zeros((len(head), 4 * F))
    for ch in range(4):
        t[:, ch * F:(ch + 1) * F] = ds["tail"][:, ch] / sc[:, ch // 2:ch // 2 + 1]
    return x, t, sc


def prepare(ds: dict, K: int, net: "TailNet"):
    """Network inputs and targets (n, rows): scaled tails times the output
    rows' weights, over the spectral layer's scale."""
    x, t, sc = scaled_tails(ds, K)
    tgt = np.zeros((len(x), net.rows), np.float32)
    tgt[:, :t.shape[1]] = t * net.row_w[None, :t.shape[1]] / net.t_scale
    return x, tgt, sc


def s11_error_db(ds: dict, pred_tail: np.ndarray, band_min: float = 0.5e9):
    """Mean |S11 dB| error over the band for: predicted tail, no tail
    (truncated at K) -- per instance, against the full runs."""
    freqs = ds["freqs"]
    band = freqs > band_min
    F = len(freqs)

    def db(s):
        return 20 * np.log10(np.maximum(np.abs(s), 1e-6))

    hf = ds["headf"]
    u_h = hf[:, 0] + 1j * hf[:, 1]
    i_h = hf[:, 2] + 1j * hf[:, 3]
    full = db(ds["s11_full"])
    trunc = np.abs(db(P.s11(u_h, i_h)) - full)[:, band].mean(1)
    u_t = pred_tail[:, 0:F] + 1j * pred_tail[:, F:2 * F]
    i_t = pred_tail[:, 2 * F:3 * F] + 1j * pred_tail[:, 3 * F:4 * F]
    pred = np.abs(db(P.s11(u_h + u_t, i_h + i_t)) - full)[:, band].mean(1)
    return pred, trunc


def train(train_ds: dict, test_ds: dict, cfg: NetConfig = NetConfig(), log=print):
    """Trains on train_ds and reports the S11 error on test_ds."""
    torch = _torch()
    _, t_train, _ = scaled_tails(train_ds, cfg.K)
    rms = np.sqrt((t_train ** 2).mean(0)) + 1e-30
    net = TailNet(cfg, train_ds["freqs"], int(train_ds["horizon"]), row_scale=rms, fmin_loss=0.5e9)
    x, y, _ = prepare(train_ds, cfg.K, net)
    xt, yt, sct = prepare(test_ds, cfg.K, net)
    X = torch.tensor(x, device="cuda")
    Y = torch.tensor(y, device="cuda")
    n = (len(x) // cfg.batch) * cfg.batch
    rng = np.random.default_rng(cfg.seed)
    t0 = time.perf_counter()
    losses = []
    for ep in range(cfg.epochs):
        perm = torch.tensor(rng.permutation(len(x))[:n], device="cuda")
        tot = 0.0
        for b0 in range(0, n, cfg.batch):
            idx = perm[b0:b0 + cfg.batch]
            tot += net.train_step(X[idx].contiguous(), Y[idx].contiguous())
        losses.append(tot / (n // cfg.batch))
        if log and (ep % 50 == 0 or ep == cfg.epochs - 1):
            log(f"epoch {ep} loss {losses[-1]:.4e}")
    _chk(N.lib().oems_tc_check(None))
    train_s = time.perf_counter() - t0
    pred = predict(net, xt, sct)
    err_pred, err_trunc = s11_error_db(test_ds, pred)
    sub = {k: (v[:500] if isinstance(v, np.ndarray) and v.ndim and len(v) == len(x) else v)
           for k, v in train_ds.items()}
    xs, _, scs = prepare(sub, cfg.K, net)
    err_tr, _ = s11_error_db(sub, predict(net, xs, scs))
    return net, {"train_seconds": train_s, "epochs": cfg.epochs, "final_loss": losses[-1],
                 "train_s11_db_err_pred_median": float(np.median(err_tr)),
                 "test_s11_db_err_pred_median": float(np.median(err_pred)),
                 "test_s11_db_err_pred_mean": float(np.mean(err_pred)),
                 "test_s11_db_err_trunc_median": float(np.median(err_trunc)),
                 "test_s11_db_err_trunc_mean": float(np.mean(err_trunc))}


def predict(net: TailNet, x: np.ndarray, sc: np.ndarray) -> np.ndarray:
    """Unscaled predicted tail DFTs (n, 4 F) for scaled inputs x."""
    torch = _torch()
    out = []
    B = net.cfg.batch
    for b0 in range(0, len(x), B):
        xb = x[b0:b0 + B]
        pad = B - len(xb)
        if pad:
            xb = np.concatenate([xb, np.zeros((pad,) + xb.shape[1:], np.float32)])
        o = net.forward(torch.tensor(xb, device="cuda")).cpu().numpy()[:B - pad]
        out.append(o)
    F = net.F
    w = net.row_w[:4 * F]
    o = np.concatenate(out)[:, :4 * F] * net.t_scale
    o = np.where(w > 0, o / np.where(w > 0, w, 1.0), 0.0)
    o[:, :2 * F] *= sc[:, :1]
    o[:, 2 * F:] *= sc[:, 1:]
    return o


def early_sweep(specs, K: int, freqs: np.ndarray, concurrency: int = 16):
    """Runs every spec for K steps only; returns the sweep (its results hold
    the head DFTs), the wall time and the K-step traces."""
    from . import workloads as W
    from .sweep import Sweep
    sw = Sweep(freqs, concurrency=concurrency)
    sw.set_trace_steps(K)
    ids = [sw.add(W.patch_sweep_instance(s, delta=0.5e-3, decay_db=0.0, max_steps=K, fmax=12e9)) for s in specs]
    sw.run(K)
    wall, _ = sw.stats()
    heads = np.stack([sw.trace(i)[:K].T for i in ids]).astype(np.float32)
    return sw, ids, wall, heads


def main(argv=None):
    """python -m openems_b200.predictor_net --train TRAIN.npz --test TEST.npz
    trains the network and prints one JSON line: S11 error against the full
    runs of the network's tails, of the matrix-pencil continuation and of
    plain truncation at K, and instances per hour of early-terminated vs
    full sweeps."""
    import argparse
    import json
    p = argparse.ArgumentParser()
    p.add_argument("--train", required=True)
    p.add_argument("--test", required=True)
    p.add_argument("--epochs", type=int, default=300)
    p.add_argument("--lr", type=float, default=1e-3)
    a = p.parse_args(argv)
    tr = dict(np.load(a.train))
    te = dict(np.load(a.test))
    cfg = NetConfig(epochs=a.epochs, lr=a.lr)
    net, rep = train(tr, te, cfg)
    # throughput: the held-out family early-terminated at K (+ inference) vs full runs
    specs = P.family_specs(len(te["steps"]), int(te["seed"]))
    sw, ids, wall_k, heads = early_sweep(specs, cfg.K, te["freqs"])
    # the K-step runs reproduce the full runs' heads
    rep["head_consistency_max_rel"] = float(np.abs(heads - te["head"]).max() / np.abs(te["head"]).max())
    x, _, sc = prepare({"head": heads, "tail": te["tail"]}, cfg.K, net)
    t0 = time.perf_counter()
    predict(net, x, sc)
    infer_s = time.perf_counter() - t0
    # matrix-pencil continuation of the same K-step heads (one host core)
    dt = P.grid_dt()
    freqs = te["freqs"]
    F = len(freqs)
    t0 = time.perf_counter()
    pen = np.zeros((len(heads), 4 * F))
    for k in range(len(heads)):
        ut = P.pencil_tail_dft(heads[k, 0].astype(np.float64), cfg.K, dt, freqs, 0.0, int(te["horizon"]))
        it = P.pencil_tail_dft(heads[k, 1].astype(np.float64), cfg.K, dt, freqs, 0.5, int(te["horizon"]))
        pen[k] = np.concatenate([ut.real, ut.imag, it.real, it.imag])
    pencil_s = time.perf_counter() - t0
    err_pen, _ = s11_error_db(te, pen)
    n = len(te["steps"])
    rep.update({"K": cfg.K, "test_instances": n, "train_instances": int(len(tr["steps"])),
                "test_s11_db_err_pencil_median": float(np.median(err_pen)),
                "test_s11_db_err_pencil_mean": float(np.mean(err_pen)),
                "test_s11_db_err_pencil_p90": float(np.percentile(err_pen, 90)),
                "full_wall_s": float(te["wall"]), "full_steps_mean": float(te["steps"].mean()),
                "early_wall_s": wall_k, "inference_s": infer_s, "pencil_s_one_core": pencil_s,
                "instances_per_hour_full": n / float(te["wall"]) * 3600,
                "instances_per_hour_early_net": n / (wall_k + infer_s) * 3600,
                "instances_per_hour_early_pencil": n / (wall_k + pencil_s) * 3600})
    print(json.dumps(rep))


if __name__ == "__main__":
    main()
