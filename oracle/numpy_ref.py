"""Independent numpy restatement of the reference Yee update -- TEST INFRASTRUCTURE.

A second oracle, written separately from ``oems_oracle.cpp``, used only to
cross-check it.  It follows src/fdtd/basic_engine.rs:191-306 (H over all
cells with zero forward differences at the max faces; E over i, j, k >= 1) and
:313-395 (soft ``+=`` / hard ``=`` after the E update).  numpy rounds every
elementwise product and sum separately, which is the same arithmetic as the
Rust code.  Small grids only: each step allocates temporaries.
"""
from __future__ import annotations

import numpy as np


def _fwd(a: np.ndarray, axis: int) -> np.ndarray:
    """a[idx+1] - a[idx] along axis, 0 at the last index."""
    d = np.zeros_like(a)
    sl_hi = [slice(None)] * 3
    sl_lo = [slice(None)] * 3
    sl_hi[axis] = slice(1, None)
    sl_lo[axis] = slice(0, -1)
    d[tuple(sl_lo)] = a[tuple(sl_hi)] - a[tuple(sl_lo)]
    return d


def _bwd(a: np.ndarray, axis: int) -> np.ndarray:
    """a[idx] - a[idx-1] along axis (garbage-free 0 at index 0, never used)."""
    d = np.zeros_like(a)
    sl_hi = [slice(None)] * 3
    sl_lo = [slice(None)] * 3
    sl_hi[axis] = slice(1, None)
    sl_lo[axis] = slice(0, -1)
    d[tuple(sl_hi)] = a[tuple(sl_hi)] - a[tuple(sl_lo)]
    return d


def run(coeffs12: np.ndarray, fields6: np.ndarray, num_steps: int, excitations=()) -> np.ndarray:
    """Advance ``fields6`` (Ex Ey Ez Hx Hy Hz) by ``num_steps``.

    ``excitations``: iterable of (pos (i,j,k), dir, soft, samples) with
    samples indexed by batch step.  Returns the new fields (float32).
    """
    c = [np.asarray(x, dtype=np.float32) for x in coeffs12]
    ca, cb, da, db = c[0:3], c[3:6], c[6:9], c[9:12]
    ex, ey, ez, hx, hy, hz = (np.array(f, dtype=np.float32) for f in fields6)
    for step in range(num_steps):
        dez_dy, dey_dz = _fwd(ez, 1), _fwd(ey, 2)
        dex_dz, dez_dx = _fwd(ex, 2), _fwd(ez, 0)
        dey_dx, dex_dy = _fwd(ey, 0), _fwd(ex, 1)
        hx = da[0] * hx + db[0] * (dez_dy - dey_dz)
        hy = da[1] * hy + db[1] * (dex_dz - dez_dx)
        hz = da[2] * hz + db[2] * (dey_dx - dex_dy)
        inner = (slice(1, None),) * 3
        cx = _bwd(hz, 1) - _bwd(hy, 2)
        cy = _bwd(hx, 2) - _bwd(hz, 0)
        cz = _bwd(hy, 0) - _bwd(hx, 1)
        nex = ca[0] * ex + cb[0] * cx
        ney = ca[1] * ey + cb[1] * cy
        nez = ca[2] * ez + cb[2] * cz
        ex[inner] = nex[inner]
        ey[inner] = ney[inner]
        ez[inner] = nez[inner]
        comps = (ex, ey, ez)
        for pos, d, soft, samples in excitations:
            if step >= len(samples):
                continue
            v = np.float32(samples[step])
            if soft:
                comps[d][tuple(pos)] += v
            else:
                comps[d][tuple(pos)] = v
    return np.stack([ex, ey, ez, hx, hy, hz])


def round_to_storage(a: np.ndarray, store: str) -> np.ndarray:
    """float32 values rounded to nearest (even) in the 2-byte storage type
    and back: "f16" IEEE half, "bf16" bfloat16 (the top 16 bits of a float32),
    "f32" unchanged."""
    a = np.asarray(a, dtype=np.float32)
    if store == "f32":
        return a
    if store == "f16":
        return a.astype(np.float16).astype(np.float32)
    b = a.view(np.uint32).astype(np.uint64)
    b = ((b + 0x7FFF + ((b >> 16) & 1)) >> 16) << 16
    return (b & 0xFFFFFFFF).astype(np.uint32).view(np.float32).reshape(a.shape)


def run_stored(coeffs12: np.ndarray, fields6: np.ndarray, num_steps: int, excitations=(), store: str = "f16",
               h_scale: float = 512.0) -> np.ndarray:
    """The update of ``run`` with 2-byte field storage: arithmetic in float32,
    every stored field value rounded to ``store``, H kept multiplied by
    ``h_scale`` (a power of two, folded into Cb / s and Db * s, so the
    float32 arithmetic is exactly the scaled one).  Returns unscaled fields.
    This restates the engine's OEMS_ENGINE_FIELDS_F16 / _BF16 modes (no
    counterpart in the reference)."""
    s = np.float32(h_scale)
    c = [np.asarray(x, dtype=np.float32) for x in coeffs12]
    ca, cb, da, db = c[0:3], [x / s for x in c[3:6]], c[6:9], [x * s for x in c[9:12]]
    R = lambda a: round_to_storage(a, store)  # noqa: E731
    f = [R(np.asarray(x, dtype=np.float32) * (s if k >= 3 else np.float32(1.0))) for k, x in enumerate(fields6)]
    ex, ey, ez, hx, hy, hz = f
    for step in range(num_steps):
        dez_dy, dey_dz = _fwd(ez, 1), _fwd(ey, 2)
        dex_dz, dez_dx = _fwd(ex, 2), _fwd(ez, 0)
        dey_dx, dex_dy = _fwd(ey, 0), _fwd(ex, 1)
        hx = R(da[0] * hx + db[0] * (dez_dy - dey_dz))
        hy = R(da[1] * hy + db[1] * (dex_dz - dez_dx))
        hz = R(da[2] * hz + db[2] * (dey_dx - dex_dy))
        inner = (slice(1, None),) * 3
        cx = _bwd(hz, 1) - _bwd(hy, 2)
        cy = _bwd(hx, 2) - _bwd(hz, 0)
        cz = _bwd(hy, 0) - _bwd(hx, 1)
        ex[inner] = R(ca[0] * ex + cb[0] * cx)[inner]
        ey[inner] = R(ca[1] * ey + cb[1] * cy)[inner]
        ez[inner] = R(ca[2] * ez + cb[2] * cz)[inner]
        comps = (ex, ey, ez)
        for pos, d, soft, samples in excitations:
            if step >= len(samples):
                continue
            v = np.float32(samples[step])
            p = tuple(pos)
            comps[d][p] = R(np.array(comps[d][p] + v if soft else v, dtype=np.float32))
    return np.stack([ex, ey, ez, hx / s, hy / s, hz / s])


# ---------------------------------------------------------------------------
# per-cell extensions, written separately from oems_oracle.cpp
# ---------------------------------------------------------------------------

EPS0 = 8.854187817e-12  # src/constants.rs
f32 = np.float32


def dispersive_coeffs(kind: int, params, dt: float, eps_inf: float = 1.0):
    """(a, b, c, c2) as float32.  Drude: DrudeMaterial::new
    (src/extensions/dispersive.rs:476-498); Lorentz: LorentzMaterial::new
    (:134-159, kind 1 as the reference, kind 3 the same a, b, c with the
    second-order update); Debye: DebyeMaterial::new (:570-592).  eps_inf = 1
    gives the reference's c."""
    p = list(params) + [0.0] * (3 - len(params))
    c2 = 0.0
    if kind == 0:
        den = 1.0 + p[1] * dt / 2.0
        a, b, c = (1.0 - p[1] * dt / 2.0) / den, EPS0 * p[0] * p[0] * dt / den, dt / (EPS0 * eps_inf)
    elif kind == 4:  # Drude as a polarisation recursion (omega_0 = 0)
        den = 1.0 + p[1] * dt / 2.0
        a, b, c = 2.0 / den, (p[1] * dt / 2.0 - 1.0) / den, EPS0 * p[0] * p[0] * dt * dt / den
        c2 = 1.0 / (EPS0 * eps_inf)
    elif kind in (1, 3):
        den = 1.0 + p[1] * dt / 2.0
        a = (2.0 - p[0] * p[0] * dt * dt) / den
        b = (p[1] * dt / 2.0 - 1.0) / den
        c = EPS0 * p[2] * p[0] * p[0] * dt * dt / den
        c2 = 1.0 / (EPS0 * eps_inf)
    else:
        den = 2.0 * p[0] + dt
        a, b, c = (2.0 * p[0] - dt) / den, 2.0 * EPS0 * p[1] * dt / den, dt / (EPS0 * eps_inf)
    return f32(a), f32(b), f32(c), f32(c2)


def dispersive_step(kind, coeffs, e, state, prev, dt):
    """One post_update_e of one field value (float32 scalars); returns
    (e', state', prev').  Drude :510-535, Lorentz :171-196, Debye :604-630;
    kinds 3 / 4 are driven by the field before the E update, which on a grid
    without curl (one cell) is the e passed here."""
    a, b, c, c2 = coeffs
    e, state, prev = f32(e), f32(state), f32(prev)
    if kind == 0:
        jn = a * state + b * e
        return e - c * jn, jn, prev
    if kind == 1:
        jn = a * state + c * e
        return e - b * jn, jn, prev
    if kind == 2:
        pn = a * state + b * e
        return e - c * ((pn - state) / f32(dt)), pn, prev
    pn = (a * state + b * prev) + c * e
    return e - c2 * (pn - state), pn, state


def rlc_coeffs(rlc_type, r, l, c, dl, dt):
    """(v_vv, v_il) as float32: calc_parallel_coeffs / calc_series_coeffs
    (src/extensions/lumped_rlc.rs:190-250)."""
    da = dl * dl
    if rlc_type == 0:
        g = 1.0 / r if r > 0 else 0.0
        inv_l = dt / l if l > 0 else 0.0
        cc = c if c > 0 else 0.0
        g_eff = g * dl / da
        c_eff = cc * dl / da + EPS0 * dl / da
        den = 2.0 * c_eff + g_eff * dt
        return f32((2.0 * c_eff - g_eff * dt) / den), f32(inv_l * dl / da)
    rr = r if r > 0 else 0.0
    ll = l if l > 0 else 0.0
    inv_c = dt / c if c > 0 else 0.0
    den = 2.0 * (ll * da / dl) + (rr * da / dl) * dt
    return f32(1.0), f32(0.0 if abs(den) < 1e-20 else inv_c * da / dl)


def rlc_step(coeffs, e, i_int, dt):
    """LumpedRlc::post_update_e for one element (lumped_rlc.rs:263-286)."""
    v_vv, v_il = coeffs
    e, i_int = f32(e), f32(i_int)
    return v_vv * e + v_il * i_int, i_int + e * f32(dt)
