"""Early termination of port sweeps: the tail of a run stopped at K steps.

A run is stopped after K timesteps and the rest of its port voltage /
current is predicted as damped sinusoids, whose DFT is added in closed form
to the DFT of the K simulated steps to give S11.  Two predictors use this
module: the learned network (predictor_net.py; modal coefficients on a fixed
pole grid, trained on the engine library's BF16 tensor-core kernels) and the
matrix pencil (Hua & Sarkar), which finds the modes of the last window of
the trace itself and drives the staged early stop (early_stop.py).

Here: the seeded patch family the network is trained on (the patch-antenna
sweep family at a reduced size, n ~ U{40..80} cells of 0.5 mm), the runs
that produce training traces, the pole grid and the least-squares fit of a
trace tail onto it, the closed-form DFT of a tail and the matrix pencil.
"""
from __future__ import annotations

from dataclasses import dataclass
from typing import List

import numpy as np

from . import workloads as W

K_DEFAULT = 2048        # simulated steps before the prediction
HORIZON = 40000         # steps of a full run (cap); the tail spans [K, HORIZON)
FREQS = np.linspace(0.0, 12e9, 241)


def family_specs(count: int, seed: int, layers: int = 6) -> List[W.PatchSpec]:
    """Seeded patches of the reduced family: n_{x,y,z} ~ U{40..80}, substrate
    eps_r ~ U[2.2, 10.2], thickness 2-6 cells, W, L ~ U{12..n-2(layers+4)},
    feed at a seeded fraction U[0.2, 0.7] of L/2 from the centre."""
    rng = np.random.default_rng(seed)
    out = []
    for _ in range(count):
        dims = tuple(int(v) for v in rng.integers(40, 81, size=3))
        eps_r = float(rng.uniform(2.2, 10.2))
        h = int(rng.integers(2, 7))
        margin = layers + 4
        W_ = int(rng.integers(12, max(13, dims[0] - 2 * margin + 1)))
        L_ = int(rng.integers(12, max(13, dims[1] - 2 * margin + 1)))
        frac = float(rng.uniform(0.2, 0.7))
        x0, y0 = (dims[0] - W_) // 2, (dims[1] - L_) // 2
        fx, fy = x0 + W_ // 2, y0 + L_ // 2 - int(round(frac * (L_ // 2)))
        out.append(W.PatchSpec(dims, eps_r, h, W_, L_, x0, y0, fx, fy, k_ground=layers + 2, layers=layers))
    return out


@dataclass
class PoleGrid:
    """Fixed poles p = -omega / (2 Q) + j omega on nf frequencies x the Q
    values: 64 modes by default (32 frequencies 0.25-12 GHz, Q 8 and 40)."""

    fmin: float = 0.25e9
    fmax: float = 12e9
    nf: int = 32
    qs: tuple = (8.0, 40.0)

    def poles(self) -> np.ndarray:
        w = 2 * np.pi * np.geomspace(self.fmin, self.fmax, self.nf)
        return np.concatenate([-w / (2 * q) + 1j * w for q in self.qs])

    @property
    def modes(self) -> int:
        return self.nf * len(self.qs)


def tail_basis(poles: np.ndarray, n: int, dt: float) -> np.ndarray:
    """(n, 2 m) real basis: Re and -Im of exp(p t), t = k dt, k < n."""
    t = np.arange(n) * dt
    e = np.exp(np.outer(t, poles))
    return np.concatenate([e.real, -e.imag], axis=1)


def fit_tail(tail: np.ndarray, poles: np.ndarray, dt: float, ridge: float = 1e-8) -> np.ndarray:
    """Least-squares coefficients c (complex, per pole) with
    tail(k dt) ~ Re sum c_m exp(p_m k dt), Tikhonov-regularised by `ridge`
    times the mean Gram diagonal (the basis is far from orthogonal)."""
    m = len(poles)
    if len(tail) == 0:
        return np.zeros(m, dtype=complex)
    B = tail_basis(poles, len(tail), dt)
    G = B.T @ B
    G[np.diag_indices_from(G)] += ridge * max(np.trace(G) / len(G), 1e-300)
    x = np.linalg.solve(G, B.T @ tail)
    return x[:m] + 1j * x[m:]


def tail_dft(c: np.ndarray, poles: np.ndarray, t0: float, dt: float, freqs: np.ndarray,
             n: int = 0) -> np.ndarray:
    """2 dt sum_{0<=k<n} Re(sum c_m exp(p_m k dt)) exp(-j 2 pi f (t0 + k dt)),
    the engine's single-sided DFT scaling, in closed form (geometric series;
    n = 0 sums to infinity)."""
    w = 2 * np.pi * np.asarray(freqs)[:, None]
    out = np.zeros(len(freqs), dtype=complex)
    for sign in (1, -1):  # Re(z) = (z + conj z) / 2
        p = poles[None, :] if sign == 1 else np.conj(poles)[None, :]
        cc = c[None, :] if sign == 1 else np.conj(c)[None, :]
        r = np.exp((p - 1j * w) * dt)
        part = (1.0 - r ** n) if n else 1.0
        out += (0.5 * cc * part / (1.0 - r)).sum(1)
    return 2 * dt * out * np.exp(-1j * 2 * np.pi * np.asarray(freqs) * t0)


def head_dft(x: np.ndarray, t_after0: int, dt: float, freqs: np.ndarray, half: float = 0.0) -> np.ndarray:
    """The engine's probe DFT of samples x[k] taken after timestep t_after0 + k."""
    t = (t_after0 + np.arange(len(x)) - half) * dt
    return 2 * dt * (np.exp(-2j * np.pi * np.outer(freqs, t)) @ x)


def s11(uf: np.ndarray, if_: np.ndarray, R: float = 50.0) -> np.ndarray:
    uinc = 0.5 * (uf + if_ * R)
    return (uf - uinc) / uinc


# ---------------------------------------------------------------------------
# matrix-pencil extrapolation
# ---------------------------------------------------------------------------


def matrix_pencil(y: np.ndarray, max_modes: int, rel_sv: float = 1e-7):
    """Poles z (per sample of y) and complex residues r with
    y[k] ~ sum r_m z_m^k (Hua & Sarkar's matrix pencil: SVD of the Hankel
    matrix of y, eigenvalues of the shifted signal subspace, residues by
    least squares); only decaying modes (|z| < 1) are kept."""
    n = len(y)
    L = n // 2
    Y = np.lib.stride_tricks.sliding_window_view(y, L + 1)
    _, S, Vh = np.linalg.svd(Y, full_matrices=False)
    M = int(min(max_modes, (S > S[0] * rel_sv).sum())) if S[0] > 0 else 0
    if M == 0:
        return np.zeros(0, complex), np.zeros(0, complex)
    V = Vh[:M].conj().T
    z = np.linalg.eigvals(np.linalg.pinv(V[:-1]) @ V[1:])
    z = z[np.abs(z) < 1.0]
    if len(z) == 0:
        return z, z
    Z = np.vander(z, n, increasing=True).T
    r = np.linalg.lstsq(Z, y.astype(complex), rcond=None)[0]
    return z, r


def pencil_modes(x: np.ndarray, K: int, dt: float, window: int = 1536, decimate: int = 4, max_modes: int = 40):
    """Continuous-time poles p and residues c (at sample K) of the modes the
    matrix pencil finds in x[K - window : K] (clipped to the samples there
    are) decimated by `decimate`: x[K + k] ~ sum c exp(p k dt)."""
    start = max(0, K - window)
    y = np.asarray(x[start:K:decimate], dtype=np.float64)
    if len(y) < 8:
        return np.zeros(0, complex), np.zeros(0, complex)
    z, r = matrix_pencil(y, max_modes)
    if len(z) == 0:
        return z, r
    p = np.log(z) / (decimate * dt)
    return p, r * np.exp(p * (K - start) * dt)


def pencil_tail_dft(x: np.ndarray, K: int, dt: float, freqs: np.ndarray, half: float, horizon: int = HORIZON,
                    window: int = 1536, decimate: int = 4, max_modes: int = 40, modes=None) -> np.ndarray:
    """DFT of the continuation of x after sample K (to `horizon`), from the
    modes the matrix pencil finds in x[K - window : K] decimated by
    `decimate` (or `modes` = (p, c) of pencil_modes, already computed); the
    engine's DFT scaling and sample times (x[k] taken after timestep k + 1,
    minus `half`)."""
    p, c = modes if modes is not None else pencil_modes(x, K, dt, window, decimate, max_modes)
    if len(p) == 0:
        return np.zeros(len(freqs), complex)
    # the modes come in conjugate pairs: Re(sum) is the real continuation
    return tail_dft(c, p, (K + 1 - half) * dt, dt, freqs, horizon - K)


# ---------------------------------------------------------------------------
# dataset
# ---------------------------------------------------------------------------

def grid_dt(delta: float = 0.5e-3) -> float:
    """dt of the uniform cubic grid (src/fdtd/operator.rs:82-89)."""
    return 0.99 * (1.0 / (299792458.0 * np.sqrt(3.0 / (delta * delta))))


def tail_matrix(poles: np.ndarray, K: int, dt: float, freqs: np.ndarray, half: float,
                horizon: int = HORIZON) -> np.ndarray:
    """Real (2F, 2m) matrix T with [Re X; Im X] = T [Re c; Im c] for the tail
    DFT X of the modal coefficients c (the network's last, fixed layer)."""
    m = len(poles)
    T = np.zeros((2 * len(freqs), 2 * m))
    for j in range(m):
        for part, c in ((0, 1.0 + 0j), (1, 1j)):
            e = np.zeros(m, dtype=complex)
            e[j] = c
            x = tail_dft(e, poles, (K + 1 - half) * dt, dt, freqs, horizon - K)
            T[:len(freqs), part * m + j] = x.real
            T[len(freqs):, part * m + j] = x.imag
    return T


def build_dataset(count: int, seed: int, K: int = K_DEFAULT, concurrency: int = 16,
                  freqs: np.ndarray = FREQS, horizon: int = HORIZON) -> dict:
    """Runs `count` seeded patches to -50 dB (cap `horizon` steps) on the GPU
    and returns per instance: the first K samples of u and i, the DFTs of the
    tails [K, end) and of the heads, and the full-run S11."""
    from .sweep import Sweep
    specs = family_specs(count, seed)
    sw = Sweep(freqs, concurrency=concurrency)
    sw.set_trace_steps(K)
    ids = [sw.add(W.patch_sweep_instance(s, delta=0.5e-3, decay_db=50.0, max_steps=horizon, fmax=12e9))
           for s in specs]
    sw.run(2000)
    wall, cell_steps = sw.stats()
    dt = grid_dt()
    F = len(freqs)
    head = np.zeros((count, 2, K), np.float32)
    tail = np.zeros((count, 4, F), np.float64)      # Re U, Im U, Re I, Im I of the tail
    headf = np.zeros((count, 4, F), np.float64)
    s11_full = np.zeros((count, F), complex)
    steps = np.zeros(count, np.int64)
    for k, iid in enumerate(ids):
        r = sw.result(iid)
        x = sw.trace(iid)
        steps[k] = r["timesteps"]
        head[k, :, :min(K, len(x))] = x[:K].T
        # the sweep's running DFTs cover the whole run: tail = full - head
        for ch, half, full in ((0, 0.0, r["uf"]), (1, 0.5, r["if"])):
            hd = head_dft(x[:K, ch], 1, dt, freqs, half)
            td = full - hd if steps[k] > K else np.zeros(F, complex)
            headf[k, 2 * ch], headf[k, 2 * ch + 1] = hd.real, hd.imag
            tail[k, 2 * ch], tail[k, 2 * ch + 1] = td.real, td.imag
        s11_full[k] = r["s11"]
    return {"head": head, "tail": tail, "headf": headf, "s11_full": s11_full, "steps": steps,
            "freqs": freqs, "K": K, "horizon": horizon, "wall": wall, "cell_steps": cell_steps, "seed": seed}


def main(argv=None):
    """python -m openems_b200.predictor generate --count N --seed S --out FILE"""
    import argparse
    import json
    p = argparse.ArgumentParser()
    p.add_argument("cmd", choices=["generate"])
    p.add_argument("--count", type=int, default=2000)
    p.add_argument("--seed", type=int, default=5)
    p.add_argument("--concurrency", type=int, default=16)
    p.add_argument("--out", required=True)
    a = p.parse_args(argv)
    d = build_dataset(a.count, a.seed, concurrency=a.concurrency)
    # compact storage: the network scales its inputs anyway
    d["head"] = d["head"].astype(np.float16 if np.abs(d["head"]).max() < 6e4 else np.float32)
    for k in ("tail", "headf"):
        d[k] = d[k].astype(np.float32)
    d["s11_full"] = d["s11_full"].astype(np.complex64)
    np.savez_compressed(a.out, **{k: v for k, v in d.items()})
    print(json.dumps({"count": a.count, "seed": a.seed, "wall_s": d["wall"], "cell_steps": d["cell_steps"],
                      "instances_per_hour": a.count / d["wall"] * 3600, "steps_mean": float(d["steps"].mean())}))


if __name__ == "__main__":
    main()
