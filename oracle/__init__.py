"""CPU oracle for the Yee FDTD hot path -- TEST INFRASTRUCTURE ONLY.

Only ``tests/``, ``__graft_entry__.smoke()`` and the CPU-baseline leg of
``bench.py`` may import this package.  It is the checker, never the product.

``liboems_oracle.so`` (built by ``oracle/Makefile``) restates the Rust openEMS
rewrite's scalar reference engine (src/fdtd/basic_engine.rs:56-395), its
operator (src/fdtd/operator.rs:82-263) and excitation sampling
(src/fdtd/excitation.rs:150-200, src/fdtd/batch.rs:110-129) in C++ compiled
with -ffp-contract=off.  ``numpy_ref`` is a second, independent restatement of
the same update in numpy used to cross-check it bit for bit.

Parity status: pinned to the reference's known-answer unit tests and scenario
physics checks; the reference ships no golden field arrays and cannot be built
here (no Rust toolchain).
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "liboems_oracle.so")

# Excitation kinds (src/fdtd/excitation.rs:9-42)
EXC_GAUSSIAN = 0
EXC_SINUSOIDAL = 1
EXC_GAUSSIAN_MODULATED = 2
EXC_DIRAC = 3
EXC_STEP = 4


class EnergySample(ctypes.Structure):
    _fields_ = [("timestep", ctypes.c_uint64), ("e_energy", ctypes.c_double),
                ("h_energy", ctypes.c_double), ("total_energy", ctypes.c_double)]


class BatchResult(ctypes.Structure):
    _fields_ = [("timesteps_executed", ctypes.c_uint64), ("termination_reason", ctypes.c_int32),
                ("pad_", ctypes.c_int32), ("final_decay_db", ctypes.c_double),
                ("num_energy_samples", ctypes.c_uint64), ("peak_energy", ctypes.c_double)]


def build() -> str:
    """Compile the oracle library with its Makefile; return the library path."""
    subprocess.run(["make", "-s", "-C", _HERE], check=True)
    return _LIB_PATH


_lib = None


def lib() -> ctypes.CDLL:
    global _lib
    if _lib is None:
        if not os.path.exists(_LIB_PATH):
            build()
        L = ctypes.CDLL(_LIB_PATH)
        P, I64, I32, D, U64 = ctypes.c_void_p, ctypes.c_int64, ctypes.c_int32, ctypes.c_double, ctypes.c_uint64
        L.orc_new.restype = P
        L.orc_new.argtypes = [I32, I64, I64, I64, D, D, D, D]
        L.orc_free.argtypes = [P]
        L.orc_set_threads.argtypes = [P, I32]
        L.orc_set_zline.argtypes = [P, I32]
        L.orc_set_material.argtypes = [P, D, D, D, D, P]
        L.orc_set_pec.argtypes = [P, P]
        L.orc_get_coefficients.argtypes = [P, P]
        L.orc_set_coefficients.argtypes = [P, P]
        L.orc_get_fields.argtypes = [P, P]
        L.orc_set_fields.argtypes = [P, P]
        L.orc_reset.argtypes = [P]
        L.orc_timestep.restype = U64
        L.orc_timestep.argtypes = [P]
        L.orc_clear_excitations.argtypes = [P]
        L.orc_add_excitation_sampled.argtypes = [P, P, I32, I32, P, I64]
        L.orc_add_excitation_analytic.argtypes = [P, P, I32, I32, I32, P, D, U64, I64]
        L.orc_add_point_probe.argtypes = [P, I32, P]
        L.orc_get_probe_traces.argtypes = [P, P, I64]
        L.orc_add_probe.restype = I32
        L.orc_add_probe.argtypes = [P, P, P, P, I64, I32]
        L.orc_add_probe_dft.restype = I32
        L.orc_add_probe_dft.argtypes = [P, I32, P, I64]
        L.orc_get_probe_dft.argtypes = [P, I32, P]
        L.orc_eval_probes.argtypes = [P, P]
        L.orc_enable_cpml.restype = I32
        L.orc_enable_cpml.argtypes = [P, P, D, D, D, D]
        L.orc_cpml_profile.restype = I32
        L.orc_cpml_profile.argtypes = [P, I32, P]
        L.orc_enable_mur.restype = I32
        L.orc_enable_mur.argtypes = [P, P, I32, D]
        L.orc_enable_tfsf.restype = I32
        L.orc_enable_tfsf.argtypes = [P, I32, I32, D, D, I64, D, I32]
        L.orc_add_dispersive.restype = I32
        L.orc_add_dispersive.argtypes = [P, I32, P, D, P, I64]
        L.orc_add_lumped_rlc.restype = I32
        L.orc_add_lumped_rlc.argtypes = [P, P, I32, I32, D, D, D]
        L.orc_set_lumped.restype = D
        L.orc_set_lumped.argtypes = [P, P, I32, D, D, D, D]
        L.orc_add_field_dft.restype = I32
        L.orc_add_field_dft.argtypes = [P, P, P, ctypes.c_uint32, P, I64, U64]
        L.orc_field_dft_points.restype = I64
        L.orc_field_dft_points.argtypes = [P, I32]
        L.orc_get_field_dft.argtypes = [P, I32, I64, I64, P]
        L.orc_add_nf2ff_box.restype = I32
        L.orc_add_nf2ff_box.argtypes = [P, P, P, P, P, I64, U64]
        L.orc_get_nf2ff_face.restype = I64
        L.orc_get_nf2ff_face.argtypes = [P, I32, I32, I64, P]
        L.orc_enable_upml.restype = I32
        L.orc_enable_upml.argtypes = [P, P, D, D, I32]
        L.orc_upml_kappa.argtypes = [P, I32, I32, P, I32, I64, D, D, D, ctypes.POINTER(D),
                                     ctypes.POINTER(D)]
        L.orc_run_batch.restype = I32
        L.orc_run_batch.argtypes = [P, U64, U64, I32, U64, I32, D, D, ctypes.POINTER(BatchResult)]
        L.orc_get_energy_samples.argtypes = [P, ctypes.POINTER(EnergySample), U64]
        L.orc_energy.argtypes = [P, ctypes.POINTER(D), ctypes.POINTER(D)]
        L.orc_grid_timestep.argtypes = [P, I64, P, I64, P, I64, D, ctypes.POINTER(D), P]
        L.orc_excitation_eval.restype = D
        L.orc_excitation_eval.argtypes = [I32, P, D, D]
        _lib = L
    return _lib


def _ptr(a: np.ndarray) -> ctypes.c_void_p:
    return ctypes.c_void_p(a.ctypes.data)


def grid_timestep(xl, yl, zl, unit=1.0):
    """dt and (dx, dy, dz) per src/fdtd/operator.rs:82-89."""
    xl, yl, zl = (np.ascontiguousarray(v, dtype=np.float64) for v in (xl, yl, zl))
    dt = ctypes.c_double()
    d = np.zeros(3)
    lib().orc_grid_timestep(_ptr(xl), len(xl), _ptr(yl), len(yl), _ptr(zl), len(zl), unit,
                            ctypes.byref(dt), _ptr(d))
    return dt.value, tuple(d)


def uniform_lines(n, delta):
    """Grid::uniform mesh lines (src/geometry/mod.rs:60-66)."""
    return np.arange(n + 1, dtype=np.float64) * delta


def excitation_eval(kind, params, amplitude, t):
    p = np.zeros(3)
    p[:len(params)] = params
    return lib().orc_excitation_eval(kind, _ptr(p), amplitude, t)


class OracleSim:
    """One oracle simulation (BasicEngine semantics) in FP32 or FP64."""

    def __init__(self, nx, ny, nz, dt, delta, precision=32, threads=1, zline=False):
        self.shape = (nx, ny, nz)
        self.n = nx * ny * nz
        self.dt = dt
        self.precision = precision
        self.dtype = np.float32 if precision == 32 else np.float64
        self._h = lib().orc_new(precision, nx, ny, nz, dt, *delta)
        if not self._h:
            raise ValueError("invalid oracle dimensions")
        self.num_probes = 0
        self._last_steps = 0
        lib().orc_set_threads(self._h, threads)
        lib().orc_set_zline(self._h, int(bool(zline)))

    def set_zline(self, on: bool):
        """Switch the H / E loops to the SIMD engine's z-line form (same bits)."""
        lib().orc_set_zline(self._h, int(bool(on)))

    def __del__(self):
        h = getattr(self, "_h", None)
        if h:
            lib().orc_free(h)
            self._h = None

    @staticmethod
    def _region(r):
        return np.ascontiguousarray(r, dtype=np.int64)

    def set_material(self, eps_r, mu_r, sigma_e, sigma_m, region):
        r = self._region(region)
        lib().orc_set_material(self._h, eps_r, mu_r, sigma_e, sigma_m, _ptr(r))

    def set_pec(self, region):
        r = self._region(region)
        lib().orc_set_pec(self._h, _ptr(r))

    def coefficients(self):
        out = np.zeros((12,) + self.shape, dtype=self.dtype)
        lib().orc_get_coefficients(self._h, _ptr(out))
        return out

    def set_coefficients(self, c12):
        c = np.ascontiguousarray(c12, dtype=self.dtype).reshape((12,) + self.shape)
        lib().orc_set_coefficients(self._h, _ptr(c))

    def fields(self):
        out = np.zeros((6,) + self.shape, dtype=self.dtype)
        lib().orc_get_fields(self._h, _ptr(out))
        return out

    def set_fields(self, f6):
        f = np.ascontiguousarray(f6, dtype=self.dtype).reshape((6,) + self.shape)
        lib().orc_set_fields(self._h, _ptr(f))

    def reset(self):
        lib().orc_reset(self._h)

    @property
    def timestep(self):
        return int(lib().orc_timestep(self._h))

    def clear_excitations(self):
        lib().orc_clear_excitations(self._h)

    def add_excitation_sampled(self, pos, direction, soft, samples):
        p = np.ascontiguousarray(pos, dtype=np.int64)
        s = np.ascontiguousarray(samples, dtype=self.dtype)
        lib().orc_add_excitation_sampled(self._h, _ptr(p), direction, int(soft), _ptr(s), len(s))

    def add_excitation_analytic(self, pos, direction, soft, kind, params, amplitude, start, n):
        p = np.ascontiguousarray(pos, dtype=np.int64)
        par = np.zeros(3)
        par[:len(params)] = params
        lib().orc_add_excitation_analytic(self._h, _ptr(p), direction, int(soft), kind, _ptr(par),
                                          amplitude, start, n)

    def add_point_probe(self, comp, pos):
        p = np.ascontiguousarray(pos, dtype=np.int64)
        lib().orc_add_point_probe(self._h, comp, _ptr(p))
        self.num_probes += 1

    def add_probe(self, terms, mode):
        """terms: [(component, (i, j, k), weight)]; mode 0 f32 ordered sum, 1 f64."""
        c = np.ascontiguousarray([t[0] for t in terms] or [0], dtype=np.int32)
        p = np.ascontiguousarray([list(t[1]) for t in terms] or [[0, 0, 0]], dtype=np.int64)
        w = np.ascontiguousarray([t[2] for t in terms] or [0.0], dtype=np.float64)
        pid = lib().orc_add_probe(self._h, _ptr(c), _ptr(p), _ptr(w), len(terms), mode)
        self.num_probes += 1
        return pid

    def probe_traces(self):
        out = np.zeros((self._last_steps, self.num_probes), dtype=np.float64)
        lib().orc_get_probe_traces(self._h, _ptr(out), self._last_steps)
        return out

    def eval_probes(self):
        out = np.zeros(max(1, self.num_probes))
        lib().orc_eval_probes(self._h, _ptr(out))
        return out[:self.num_probes]

    def add_probe_dft(self, probe, freqs):
        f = np.ascontiguousarray(freqs, dtype=np.float64)
        self._dft_sizes = getattr(self, "_dft_sizes", [])
        self._dft_sizes.append(len(f))
        return lib().orc_add_probe_dft(self._h, probe, _ptr(f), len(f))

    def probe_dft(self, dft):
        out = np.zeros(2 * self._dft_sizes[dft])
        lib().orc_get_probe_dft(self._h, dft, _ptr(out))
        return out[0::2] + 1j * out[1::2]

    def enable_cpml(self, layers=(8,) * 6, grading_order=3.0, reflection_coeff=1e-6,
                    alpha_max=0.0, kappa_max=1.0):
        l6 = np.ascontiguousarray(layers, dtype=np.int32)
        rc = lib().orc_enable_cpml(self._h, _ptr(l6), grading_order, reflection_coeff, alpha_max,
                                   kappa_max)
        if rc != 0:
            raise ValueError(f"invalid CPML configuration ({rc})")

    def enable_tfsf(self, direction, polarization, frequency, amplitude, boundary_layer=10, phase_velocity=0.0,
                    kind=0):
        rc = lib().orc_enable_tfsf(self._h, int(direction), int(polarization), float(frequency),
                                   float(amplitude), int(boundary_layer), float(phase_velocity), int(kind))
        if rc != 0:
            raise ValueError(f"TF/SF configuration rejected ({rc})")

    def enable_mur(self, enabled=(1,) * 6, order=1, phase_velocity=0.0):
        e = np.ascontiguousarray([int(bool(v)) for v in enabled], dtype=np.int32)
        rc = lib().orc_enable_mur(self._h, _ptr(e), order, phase_velocity or 0.0)
        if rc != 0:
            raise ValueError(f"invalid Mur configuration ({rc})")

    def add_dispersive(self, kind, params, cells, eps_inf=1.0):
        p = np.zeros(3)
        p[:len(params)] = params
        c = np.ascontiguousarray(cells, dtype=np.int64).reshape(-1, 3)
        rc = lib().orc_add_dispersive(self._h, int(kind), _ptr(p), float(eps_inf), _ptr(c), len(c))
        if rc != 0:
            raise ValueError(f"invalid dispersive material ({rc})")

    def add_lumped_rlc(self, pos, direction, type_, r=0.0, l=0.0, c=0.0):
        q = np.ascontiguousarray(pos, dtype=np.int64)
        rc = lib().orc_add_lumped_rlc(self._h, _ptr(q), int(direction), int(type_), r, l, c)
        if rc != 0:
            raise ValueError(f"invalid lumped RLC element ({rc})")

    def set_lumped(self, pos, direction, r=0.0, c=0.0, eps_r=1.0, sigma=0.0):
        q = np.ascontiguousarray(pos, dtype=np.int64)
        return lib().orc_set_lumped(self._h, _ptr(q), int(direction), r, c, eps_r, sigma)

    def add_field_dft(self, region, freqs, comp_mask=0x3F, sub_sample=(1, 1, 1), interval=1):
        r = np.ascontiguousarray(region, dtype=np.int64)
        ss = np.ascontiguousarray(sub_sample, dtype=np.int64)
        f = np.ascontiguousarray(freqs, dtype=np.float64)
        did = lib().orc_add_field_dft(self._h, _ptr(r), _ptr(ss), comp_mask, _ptr(f), len(f), interval)
        self._fd = getattr(self, "_fd", {})
        self._fd[did] = (len(f), [c for c in range(6) if comp_mask >> c & 1])
        return did

    def field_dft(self, did, f, comp):
        """Complex accumulator of component comp (0..5) at frequency index f."""
        n = lib().orc_field_dft_points(self._h, did)
        out = np.zeros(2 * n)
        lib().orc_get_field_dft(self._h, did, f, self._fd[did][1].index(comp), _ptr(out))
        return out[0::2] + 1j * out[1::2]

    def add_nf2ff_box(self, lo, hi, freqs, directions=(1,) * 6, interval=1):
        l3 = np.ascontiguousarray(lo, dtype=np.int64)
        h3 = np.ascontiguousarray(hi, dtype=np.int64)
        d6 = np.ascontiguousarray([int(bool(v)) for v in directions], dtype=np.int32)
        f = np.ascontiguousarray(freqs, dtype=np.float64)
        bid = lib().orc_add_nf2ff_box(self._h, _ptr(l3), _ptr(h3), _ptr(d6), _ptr(f), len(f), interval)
        if bid < 0:
            raise ValueError("invalid NF2FF box")
        return bid

    def nf2ff_face(self, bid, face, f, lo, hi):
        """(4, nb, nc) complex: Eb, Ec, Hb, Hc of one face at frequency index f."""
        a = face // 2
        b, c = (a + 1) % 3, (a + 2) % 3
        nb, nc = hi[b] - lo[b] + 1, hi[c] - lo[c] + 1
        out = np.zeros(8 * nb * nc)
        n = lib().orc_get_nf2ff_face(self._h, bid, face, f, _ptr(out))
        if n == 0:
            return None
        z = out[0::2] + 1j * out[1::2]
        return z.reshape(4, nb, nc)

    def enable_upml(self, layers=(8,) * 6, grading_order=3.0, reflection_coeff=1e-6, kind=0):
        """kind 0: the reference's UPML; kind 1: the corrected uniaxial PML."""
        l6 = np.ascontiguousarray(layers, dtype=np.int64)
        n = lib().orc_enable_upml(self._h, _ptr(l6), grading_order, reflection_coeff, int(kind))
        if n < 0:
            raise ValueError(f"invalid UPML kind {kind}")
        return n

    def upml_kappa(self, comp, direction, pos, is_min, layers, width, sigma_max, m):
        p = np.ascontiguousarray(pos, dtype=np.int64)
        kv, ki = ctypes.c_double(), ctypes.c_double()
        lib().orc_upml_kappa(self._h, comp, direction, _ptr(p), int(is_min), layers, width, sigma_max, m,
                             ctypes.byref(kv), ctypes.byref(ki))
        return kv.value, ki.value

    def cpml_profile(self, face):
        out = np.zeros((6, 256))
        L = lib().orc_cpml_profile(self._h, face, _ptr(out))
        flat = out.reshape(-1)[:6 * L].reshape(6, L) if L else np.zeros((6, 0))
        return {"b_e": flat[0], "c_e": flat[1], "ik_e": flat[2],
                "b_h": flat[3], "c_h": flat[4], "ik_h": flat[5]}

    def run_batch(self, num_steps, sample_interval=0, track_peak=False, check_interval=100,
                  energy_decay_db=None, initial_peak=0.0):
        res = BatchResult()
        has = energy_decay_db is not None
        lib().orc_run_batch(self._h, num_steps, sample_interval, int(track_peak), check_interval,
                            int(has), float(energy_decay_db or 0.0), initial_peak, ctypes.byref(res))
        self._last_steps = int(res.timesteps_executed)
        samples = (EnergySample * max(1, res.num_energy_samples))()
        lib().orc_get_energy_samples(self._h, samples, res.num_energy_samples)
        energy = [(s.timestep, s.e_energy, s.h_energy, s.total_energy)
                  for s in samples[:res.num_energy_samples]]
        return {"timesteps_executed": int(res.timesteps_executed),
                "termination_reason": int(res.termination_reason),
                "final_decay_db": float(res.final_decay_db),
                "energy_samples": energy, "peak_energy": float(res.peak_energy)}

    def energy(self):
        e, h = ctypes.c_double(), ctypes.c_double()
        lib().orc_energy(self._h, ctypes.byref(e), ctypes.byref(h))
        return e.value, h.value
