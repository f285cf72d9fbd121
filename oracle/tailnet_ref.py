"""CPU restatement of the early-termination network -- TEST INFRASTRUCTURE ONLY.

Only ``tests/`` may use this module: it checks the tensor-core forward and
backward kernels of openems_b200/predictor_net.py, it is never the product.

The network has no counterpart in the reference (it is new); this is a
numpy float64 statement of the same layers from the weights of a network
instance: strided valid conv1d as im2col + dense, ReLU, the two dense layers
and the fixed spectral layer, with hand-written backward passes.  With
``bf16=True`` every GEMM operand is rounded to bfloat16 (round to nearest
even) at the points where the kernels convert (activations, weights and the
output gradients fed to the weight and input products); the rest stays
float64, so the kernels agree with it up to their float32 accumulation.  The
restatement itself is pinned by central finite differences of its own
forward pass (tests/test_predictor_host.py).
"""
from __future__ import annotations

import numpy as np


def round_bf16(x) -> np.ndarray:
    """float -> bfloat16 (round to nearest even) -> float64."""
    a = np.ascontiguousarray(x, dtype=np.float32)
    b = a.view(np.uint32).astype(np.uint64)
    b = ((b + 0x7FFF + ((b >> 16) & 1)) >> 16) << 16
    return (b & 0xFFFFFFFF).astype(np.uint32).view(np.float32).astype(np.float64)


def _ident(x):
    return np.asarray(x, dtype=np.float64)


def im2col(x: np.ndarray, ks: int, s: int) -> np.ndarray:
    """(B, T, C) -> (B * Tout, ks * C): row (b, t) holds x[b, t s + k, c] at k C + c."""
    B, T, C = x.shape
    To = (T - ks) // s + 1
    idx = np.arange(To)[:, None] * s + np.arange(ks)[None, :]
    return x[:, idx, :].reshape(B * To, ks * C)


def col2im(dcols: np.ndarray, B: int, T: int, C: int, ks: int, s: int) -> np.ndarray:
    """Adjoint of im2col."""
    To = (T - ks) // s + 1
    d = dcols.reshape(B, To, ks, C)
    dx = np.zeros((B, T, C))
    for k in range(ks):
        dx[:, k:k + s * (To - 1) + 1:s, :] += d[:, :, k, :]
    return dx


class TailNetRef:
    """convs: [(w (cout, ks cin), b)], fc1, fc2: (w, b), spec: w (no bias)."""

    def __init__(self, convs, fc1, fc2, spec, ks: int = 8, stride: int = 4):
        self.convs = [(np.asarray(w, np.float64), np.asarray(b, np.float64)) for w, b in convs]
        self.fc1 = tuple(np.asarray(a, np.float64) for a in fc1)
        self.fc2 = tuple(np.asarray(a, np.float64) for a in fc2)
        self.spec = np.asarray(spec, np.float64)
        self.ks, self.s = ks, stride

    @classmethod
    def from_net(cls, net):
        """Weights of a predictor_net.TailNet (device tensors)."""
        def pair(d):
            return d.w.cpu().numpy(), d.b.cpu().numpy()
        return cls([pair(c.fc) for c in net.convs], pair(net.fc1), pair(net.fc2), net.spec.w.cpu().numpy(),
                   net.convs[0].ks, net.convs[0].s)

    def forward(self, x: np.ndarray, bf16: bool = False) -> np.ndarray:
        R = round_bf16 if bf16 else _ident
        h = np.asarray(x, np.float64)
        self._acts = []
        for w, b in self.convs:
            B, T, C = h.shape
            cols = R(im2col(h, self.ks, self.s))
            y = np.maximum(cols @ R(w).T + b, 0.0)
            self._acts.append((h.shape, cols, y))
            h = y.reshape(B, -1, w.shape[0])
        hb = R(h.reshape(h.shape[0], -1))
        z1 = np.maximum(hb @ R(self.fc1[0]).T + self.fc1[1], 0.0)
        z1b = R(z1)
        coef = z1b @ R(self.fc2[0]).T + self.fc2[1]
        coefb = R(coef)
        self._cache = (hb, z1, z1b, coefb, bf16)
        return coefb @ R(self.spec).T

    def backward(self, dout: np.ndarray):
        """Gradients [(dW, db)] of conv layers, fc1, fc2 for output gradient dout."""
        hb, z1, z1b, coefb, bf16 = self._cache
        R = round_bf16 if bf16 else _ident
        grads = []
        dcoef = R(dout) @ R(self.spec)
        d2 = R(dcoef)
        grads.append((d2.T @ z1b, dcoef.sum(0)))
        dz1 = (d2 @ R(self.fc2[0])) * (z1 > 0)
        d1 = R(dz1)
        grads.append((d1.T @ hb, dz1.sum(0)))
        dh = d1 @ R(self.fc1[0])
        conv_grads = []
        for idx in range(len(self.convs) - 1, -1, -1):
            w, _ = self.convs[idx]
            shape, cols, y = self._acts[idx]
            dy = dh.reshape(y.shape) * (y > 0)
            db_ = R(dy)
            conv_grads.append((db_.T @ cols, dy.sum(0)))
            if idx > 0:
                dh = col2im(db_ @ R(w), *shape, self.ks, self.s)
        return conv_grads[::-1] + grads[::-1]


# ---------------------------------------------------------------------------
# the staged early stop's acceptance network (openems_b200/stage_net.py)
# ---------------------------------------------------------------------------


def im2col_causal(x: np.ndarray, ks: int, dil: int) -> np.ndarray:
    """(B, T, C) -> (B * T, ks * C): row (b, t) holds x[b, t - (ks-1-k) dil, c]
    at k C + c, 0 before the start."""
    B, T, C = x.shape
    pad = (ks - 1) * dil
    xp = np.concatenate([np.zeros((B, pad, C)), x], axis=1)
    idx = np.arange(T)[:, None] + np.arange(ks)[None, :] * dil
    return xp[:, idx, :].reshape(B * T, ks * C)


def col2im_causal(dcols: np.ndarray, B: int, T: int, C: int, ks: int, dil: int) -> np.ndarray:
    """Adjoint of im2col_causal."""
    pad = (ks - 1) * dil
    d = dcols.reshape(B, T, ks, C)
    dxp = np.zeros((B, T + pad, C))
    for k in range(ks):
        dxp[:, k * dil:k * dil + T, :] += d[:, :, k, :]
    return dxp[:, pad:, :]


class StageNetRef:
    """convs [(w (cout, ks cin), b)] with dilations 4**l, fc1, fc2 (w, b):
    causal TCN read at the last step, concatenated with the scalars, MLP."""

    def __init__(self, convs, fc1, fc2, ks: int = 5):
        self.convs = [(np.asarray(w, np.float64), np.asarray(b, np.float64)) for w, b in convs]
        self.fc1 = tuple(np.asarray(a, np.float64) for a in fc1)
        self.fc2 = tuple(np.asarray(a, np.float64) for a in fc2)
        self.ks = ks

    @classmethod
    def from_net(cls, net):
        """Weights of a stage_net.StageNet (device tensors)."""
        def pair(d):
            return d.w.cpu().numpy(), d.b.cpu().numpy()
        return cls([pair(c.fc) for c in net.convs], pair(net.fc1), pair(net.fc2), net.convs[0].ks)

    def forward(self, x: np.ndarray, s: np.ndarray, bf16: bool = False) -> np.ndarray:
        R = round_bf16 if bf16 else _ident
        h = np.asarray(x, np.float64)
        self._acts = []
        for l, (w, b) in enumerate(self.convs):
            B, T, C = h.shape
            cols = R(im2col_causal(h, self.ks, 4 ** l))
            y = np.maximum(cols @ R(w).T + b, 0.0)
            self._acts.append((h.shape, cols, y))
            h = y.reshape(B, T, w.shape[0])
        feat = np.concatenate([h[:, -1, :], np.asarray(s, np.float64)], axis=1)
        fb = R(feat)
        z1 = np.maximum(fb @ R(self.fc1[0]).T + self.fc1[1], 0.0)
        z1b = R(z1)
        self._cache = (fb, z1, z1b, h.shape, bf16)
        return z1b @ R(self.fc2[0]).T + self.fc2[1]

    def backward(self, dout: np.ndarray):
        """Gradients [(dW, db)] of the conv layers, fc1, fc2 for dout."""
        fb, z1, z1b, hshape, bf16 = self._cache
        R = round_bf16 if bf16 else _ident
        d2 = R(dout)
        g2 = (d2.T @ z1b, dout.sum(0))
        dz1 = (d2 @ R(self.fc2[0])) * (z1 > 0)
        d1 = R(dz1)
        g1 = (d1.T @ fb, dz1.sum(0))
        dfeat = d1 @ R(self.fc1[0])
        B, T, Ch = hshape
        dh = np.zeros(hshape)
        dh[:, -1, :] = dfeat[:, :Ch]
        conv_grads = []
        for idx in range(len(self.convs) - 1, -1, -1):
            w, _ = self.convs[idx]
            shape, cols, y = self._acts[idx]
            dy = dh.reshape(-1, w.shape[0]) * (y > 0)
            db_ = R(dy)
            conv_grads.append((db_.T @ cols, dy.sum(0)))
            if idx > 0:
                dh = col2im_causal(db_ @ R(w), *shape, self.ks, 4 ** idx)
        return conv_grads[::-1] + [g1, g2]
