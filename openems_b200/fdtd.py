"""Python mirror of the reference's src/fdtd surface, over liboems_b200.so.

Names and argument meanings follow the Rust openEMS rewrite:

  Grid                       src/geometry/mod.rs:20-255
  Operator                   src/fdtd/operator.rs:42-263
  Excitation/ExcitationType  src/fdtd/excitation.rs:9-200
  ScheduledExcitation        src/fdtd/batch.rs:71-147
  EngineBatch, TerminationConfig, EnergyMonitorConfig,
  BatchResult, TerminationReason, EnergySample
                             src/fdtd/batch.rs:17-228
  Engine / EngineType        src/fdtd/new_engine.rs:20-153, src/fdtd/mod.rs:69-79
  BoundaryConditions         src/fdtd/mod.rs:82-167
  Simulation, EndCondition, SimulationStats
                             src/fdtd/simulation.rs:36-360

The engine is CUDA only (one GPU, no CPU fallback).  Fields are returned as
numpy float32 arrays of shape (3, nx, ny, nz), z fastest.
"""
from __future__ import annotations

import ctypes
import math
import enum
from dataclasses import dataclass, field
from typing import List, Optional, Sequence, Tuple

import numpy as np

from . import _native as N

# ---------------------------------------------------------------------------
# geometry
# ---------------------------------------------------------------------------


class Grid:
    """Cartesian mesh lines per axis (cells = lines - 1), scaled by `unit`."""

    def __init__(self, x_lines, y_lines, z_lines, unit: float = 1.0):
        self.x_lines = np.asarray(x_lines, dtype=np.float64)
        self.y_lines = np.asarray(y_lines, dtype=np.float64)
        self.z_lines = np.asarray(z_lines, dtype=np.float64)
        self.unit = float(unit)

    @classmethod
    def uniform(cls, nx: int, ny: int, nz: int, delta: float) -> "Grid":
        """Grid::uniform (src/geometry/mod.rs:60-66): lines = i * delta."""
        return cls(np.arange(nx + 1) * delta, np.arange(ny + 1) * delta,
                   np.arange(nz + 1) * delta)

    @classmethod
    def cartesian(cls, x_lines, y_lines, z_lines) -> "Grid":
        return cls(x_lines, y_lines, z_lines)

    def dimensions(self) -> Tuple[int, int, int]:
        return tuple(max(len(v) - 1, 1) for v in (self.x_lines, self.y_lines, self.z_lines))

    @staticmethod
    def _min_delta(lines) -> float:
        if len(lines) < 2:
            return 1.0
        d = np.diff(lines)
        d = d[d > 0]
        return float(d.min())

    def cell_size(self) -> Tuple[float, float, float]:
        """Minimum line spacing per axis (src/geometry/mod.rs:113-119)."""
        return tuple(self._min_delta(v) * self.unit
                     for v in (self.x_lines, self.y_lines, self.z_lines))

    def set_unit(self, unit: float):
        """Grid::set_unit: the lines are in units of `unit` metres."""
        self.unit = float(unit)


# ---------------------------------------------------------------------------
# boundaries
# ---------------------------------------------------------------------------


@dataclass(frozen=True)
class BoundaryCondition:
    """One face: kind in {'pec', 'pmc', 'mur', 'pml', 'periodic'}; layers for 'pml'."""

    kind: str = "pec"
    layers: int = 0

    @staticmethod
    def pec():
        return BoundaryCondition("pec")

    @staticmethod
    def pml(layers: int = 8):
        return BoundaryCondition("pml", layers)


@dataclass
class BoundaryConditions:
    """Six faces xmin xmax ymin ymax zmin zmax (src/fdtd/mod.rs:102-167).

    The reference's default is PML with 8 layers on every face
    (src/fdtd/mod.rs:117-128); its Operator stores but never applies it.  Here
    a 'pml' face attaches a CPML with that many layers; 'pec' faces keep the
    reference's stencil truncation.
    """

    faces: Tuple[BoundaryCondition, ...] = field(
        default_factory=lambda: tuple(BoundaryCondition.pml(8) for _ in range(6)))

    @classmethod
    def all_pec(cls):
        return cls(tuple(BoundaryCondition.pec() for _ in range(6)))

    @classmethod
    def all_pml(cls, layers: int):
        return cls(tuple(BoundaryCondition.pml(layers) for _ in range(6)))

    @classmethod
    def from_array(cls, bc: Sequence[BoundaryCondition]):
        return cls(tuple(bc))

    def cpml_layers(self) -> Tuple[int, ...]:
        return tuple(f.layers if f.kind == "pml" else 0 for f in self.faces)


@dataclass
class CpmlBoundaries:
    """CpmlBoundaries (src/extensions/cpml.rs:27-73); defaults of :41-51."""

    layers: Tuple[int, ...] = (8, 8, 8, 8, 8, 8)
    grading_order: float = 3.0
    reflection_coeff: float = 1e-6
    alpha_max: float = 0.0
    kappa_max: float = 1.0

    @classmethod
    def uniform(cls, layers: int):
        return cls(layers=(layers,) * 6)

    def to_c(self) -> N.CpmlDescC:
        d = N.CpmlDescC()
        for f in range(6):
            d.layers[f] = int(self.layers[f])
        d.grading_order = self.grading_order
        d.reflection_coeff = self.reflection_coeff
        d.alpha_max = self.alpha_max
        d.kappa_max = self.kappa_max
        return d


class PropagationDirection(enum.IntEnum):
    """PropagationDirection (src/extensions/tfsf.rs:11-41)."""
    XPlus = 0
    XMinus = 1
    YPlus = 2
    YMinus = 3
    ZPlus = 4
    ZMinus = 5

    def axis(self) -> int:
        return int(self) // 2

    def is_positive(self) -> bool:
        return int(self) % 2 == 0


class Polarization(enum.IntEnum):
    """Polarization (src/extensions/tfsf.rs:44-50)."""
    Transverse1 = 0
    Transverse2 = 1


@dataclass
class TfsfConfig:
    """TfsfConfig (src/extensions/tfsf.rs:54-103): defaults Transverse1,
    boundary layer 10, phase velocity c0.  corrected=False reproduces the
    reference's update (its 1D grid grows exponentially); True is the stable
    plane-wave source (positive directions, boundary_layer >= 1)."""

    direction: PropagationDirection
    frequency: float
    amplitude: float
    polarization: Polarization = Polarization.Transverse1
    boundary_layer: int = 10
    phase_velocity: Optional[float] = None
    corrected: bool = False

    def to_c(self) -> N.TfsfDescC:
        d = N.TfsfDescC()
        d.direction = int(self.direction)
        d.polarization = int(self.polarization)
        d.frequency = float(self.frequency)
        d.amplitude = float(self.amplitude)
        d.boundary_layer = int(self.boundary_layer)
        d.phase_velocity = float(self.phase_velocity or 0.0)
        d.kind = 1 if self.corrected else 0
        return d


@dataclass
class MurAbcConfig:
    """MurAbcConfig (src/extensions/mur_abc.rs:13-58); order 2 selects the
    second-order Mur condition (no counterpart in the reference)."""

    enabled: Tuple[bool, ...] = (True,) * 6
    phase_velocity: Optional[float] = None
    order: int = 1

    @classmethod
    def all(cls, order: int = 1):
        return cls(order=order)

    @classmethod
    def none(cls):
        return cls(enabled=(False,) * 6)

    def set_enabled(self, face: int, on: bool):
        """Face 0..5 = x-min, x-max, y-min, y-max, z-min, z-max."""
        e = list(self.enabled)
        e[face] = bool(on)
        self.enabled = tuple(e)

    def num_faces(self) -> int:
        return sum(bool(e) for e in self.enabled)

    def to_c(self) -> N.MurDescC:
        d = N.MurDescC()
        for f in range(6):
            d.enabled[f] = int(bool(self.enabled[f]))
        d.order = int(self.order)
        d.phase_velocity = float(self.phase_velocity or 0.0)
        return d


@dataclass
class PmlBoundaries:
    """PmlBoundaries (src/extensions/pml.rs:85-135) for the UPML
    (Engine.add_upml).  kind 0 is the reference's: its coefficients make the
    scheme grow without bound.  kind 1 is the corrected uniaxial PML
    (Taflove & Hagness 7.8 in the same flux form), which absorbs as well as
    CpmlBoundaries."""

    layers: Tuple[int, ...] = (8,) * 6
    grading_order: float = 3.0
    reflection_coeff: float = 1e-6
    kind: int = 0

    @classmethod
    def uniform(cls, layers: int, kind: int = 0):
        return cls(layers=(int(layers),) * 6, kind=int(kind))

    def disable(self, face: int) -> "PmlBoundaries":
        lay = list(self.layers)
        lay[face] = 0
        self.layers = tuple(lay)
        return self

    def any_enabled(self) -> bool:
        return any(v > 0 for v in self.layers)

    def to_c(self) -> N.UpmlDescC:
        d = N.UpmlDescC()
        for f in range(6):
            d.layers[f] = int(self.layers[f])
        d.grading_order = float(self.grading_order)
        d.reflection_coeff = float(self.reflection_coeff)
        d.kind = int(self.kind)
        return d


@dataclass
class DrudeMaterial:
    """DrudeMaterial (src/extensions/dispersive.rs:450-535): omega_p, gamma
    in rad/s; eps_inf divides the E correction (1 = the reference).
    second_order False reproduces the reference's update, which grows when
    gamma << omega_p in a 3D grid; True runs the polarisation recursion
    P'' + gamma P' = eps0 omega_p^2 E driven by the field before the E
    update, which stays bounded."""

    plasma_frequency: float
    collision_frequency: float
    eps_inf: float = 1.0
    second_order: bool = False

    def to_c(self) -> N.DispersiveDescC:
        return _disp_desc(4 if self.second_order else 0, (self.plasma_frequency, self.collision_frequency),
                          self.eps_inf)


@dataclass
class LorentzMaterial:
    """LorentzMaterial (src/extensions/dispersive.rs:107-196).  second_order
    False reproduces the reference's update, which keeps no P^{n-1} and
    grows without bound; True runs the full second-order recursion."""

    resonance_frequency: float
    damping: float
    delta_eps: float
    eps_inf: float = 1.0
    second_order: bool = False

    def to_c(self) -> N.DispersiveDescC:
        return _disp_desc(3 if self.second_order else 1,
                          (self.resonance_frequency, self.damping, self.delta_eps), self.eps_inf)


@dataclass
class DebyeMaterial:
    """DebyeMaterial (src/extensions/dispersive.rs:545-630): tau in s."""

    relaxation_time: float
    delta_eps: float
    eps_inf: float = 1.0

    def to_c(self) -> N.DispersiveDescC:
        return _disp_desc(2, (self.relaxation_time, self.delta_eps), self.eps_inf)


def _disp_desc(kind, params, eps_inf) -> N.DispersiveDescC:
    d = N.DispersiveDescC()
    d.kind = kind
    for a, v in enumerate(params):
        d.params[a] = float(v)
    d.eps_inf = float(eps_inf)
    return d


class RlcType(enum.IntEnum):
    """RlcType (src/extensions/lumped_rlc.rs:10-16)."""

    Parallel = 0
    Series = 1


@dataclass
class RlcElement:
    """RlcElement (src/extensions/lumped_rlc.rs:20-112) on one E edge."""

    position: Tuple[int, int, int]
    direction: int
    rlc_type: RlcType = RlcType.Parallel
    resistance: float = 0.0
    inductance: float = 0.0
    capacitance: float = 0.0

    @classmethod
    def resistor(cls, position, direction, r):
        return cls(tuple(position), direction, RlcType.Parallel, resistance=r)

    @classmethod
    def capacitor(cls, position, direction, c):
        return cls(tuple(position), direction, RlcType.Parallel, capacitance=c)

    @classmethod
    def inductor(cls, position, direction, l):
        return cls(tuple(position), direction, RlcType.Parallel, inductance=l)

    @classmethod
    def parallel_rlc(cls, position, direction, r=None, l=None, c=None):
        return cls(tuple(position), direction, RlcType.Parallel, r or 0.0, l or 0.0, c or 0.0)

    @classmethod
    def series_rlc(cls, position, direction, r=None, l=None, c=None):
        return cls(tuple(position), direction, RlcType.Series, r or 0.0, l or 0.0, c or 0.0)

    def to_c(self) -> N.LumpedRlcDescC:
        d = N.LumpedRlcDescC()
        for a in range(3):
            d.position[a] = int(self.position[a])
        d.direction = int(self.direction)
        d.type = int(self.rlc_type)
        d.resistance, d.inductance, d.capacitance = (float(self.resistance), float(self.inductance),
                                                     float(self.capacitance))
        return d


# ---------------------------------------------------------------------------
# operator
# ---------------------------------------------------------------------------


class Operator:
    """Coefficient precompute (src/fdtd/operator.rs:42-263), in the native library."""

    def __init__(self, grid: Grid, boundaries: Optional[BoundaryConditions] = None):
        self.grid = grid
        self.boundaries = boundaries if boundaries is not None else BoundaryConditions()
        h = ctypes.c_void_p()
        xl, yl, zl = (np.ascontiguousarray(v, dtype=np.float64)
                      for v in (grid.x_lines, grid.y_lines, grid.z_lines))
        N.check(N.lib().oems_operator_create(xl.ctypes.data, len(xl), yl.ctypes.data, len(yl),
                                             zl.ctypes.data, len(zl), grid.unit, ctypes.byref(h)))
        self._h = h

    def __del__(self):
        # at interpreter exit the module globals (the library handle) may be
        # gone already; the process is ending and the driver frees the device
        try:
            h = getattr(self, "_h", None)
            if h:
                N.lib().oems_operator_destroy(h)
                self._h = None
        except (TypeError, AttributeError):
            pass

    @property
    def handle(self):
        return self._h

    def clone(self) -> "Operator":
        """An independent copy: grid, dt and every coefficient (the
        reference's coefficient structs are Clone, operator.rs:21-38)."""
        h = ctypes.c_void_p()
        N.check(N.lib().oems_operator_clone(self._h, ctypes.byref(h)))
        out = Operator.__new__(Operator)
        out.grid, out.boundaries, out._h = self.grid, self.boundaries, h
        return out

    def _info(self):
        dims = (N.c_u64 * 3)()
        dt = N.c_f64()
        delta = (N.c_f64 * 3)()
        N.check(N.lib().oems_operator_info(self._h, dims, ctypes.byref(dt), delta))
        return tuple(dims), dt.value, tuple(delta)

    def timestep(self) -> float:
        return self._info()[1]

    def nyquist_timesteps(self, freq: float) -> int:
        """Operator::nyquist_timesteps (src/fdtd/operator.rs:266-270): steps
        in one period of freq, rounded up."""
        return int(math.ceil((1.0 / freq) / self.timestep()))

    def dimensions(self) -> Tuple[int, int, int]:
        return tuple(int(v) for v in self._info()[0])

    def cell_size(self) -> Tuple[float, float, float]:
        return self._info()[2]

    @staticmethod
    def _region(region):
        r = (N.c_u64 * 6)()
        for a in range(6):
            r[a] = int(region[a])
        return r

    def set_material(self, eps_r, mu_r, sigma_e, sigma_m, region):
        """region = (i0, i1, j0, j1, k0, k1), half-open."""
        N.check(N.lib().oems_operator_set_material(self._h, eps_r, mu_r, sigma_e, sigma_m,
                                                   self._region(region)))

    def set_pec(self, region):
        N.check(N.lib().oems_operator_set_pec(self._h, self._region(region)))

    def set_material_cells(self, eps_r, mu_r, sigma_e, sigma_m, cells):
        """set_material on a list of cells (n, 3)."""
        c = np.ascontiguousarray(cells, dtype=np.uint64).reshape(-1, 3)
        N.check(N.lib().oems_operator_set_material_cells(self._h, eps_r, mu_r, sigma_e, sigma_m,
                                                         c.ctypes.data, len(c)))

    def set_lumped(self, position, direction, resistance=0.0, capacitance=0.0, eps_r=1.0,
                   sigma=0.0) -> float:
        """Lumped R and/or C folded into the Ca/Cb of one E edge; returns the
        factor that turns a series source voltage into that edge's soft-source
        sample (0 without R)."""
        scale = N.c_f64()
        N.check(N.lib().oems_operator_set_lumped(self._h, _u3(position), int(direction),
                                                 float(resistance), float(capacitance), float(eps_r),
                                                 float(sigma), ctypes.byref(scale)))
        return scale.value

    def coefficients(self) -> np.ndarray:
        """Copy of the 12 arrays: (12, nx, ny, nz) = ca0..2, cb0..2, da0..2, db0..2."""
        ptrs = (N.PF * 12)()
        N.check(N.lib().oems_operator_coefficients(self._h, ptrs))
        nx, ny, nz = self.dimensions()
        n = nx * ny * nz
        out = np.empty((12, nx, ny, nz), dtype=np.float32)
        for a in range(12):
            out[a] = np.ctypeslib.as_array(ptrs[a], shape=(n,)).reshape(nx, ny, nz)
        return out

    def e_coefficients(self):
        c = self.coefficients()
        return c[0:3], c[3:6]

    def h_coefficients(self):
        c = self.coefficients()
        return c[6:9], c[9:12]

    def nyquist_timesteps(self, freq: float) -> int:
        """src/fdtd/operator.rs:266-270."""
        return int(np.ceil((1.0 / freq) / self.timestep()))


# ---------------------------------------------------------------------------
# excitation
# ---------------------------------------------------------------------------


@dataclass
class ProbeTerms:
    """A probe's term list [(component, (i, j, k), weight)] and its mode:
    0 = f32 ordered sum (VoltageProbe / CurrentProbe::sample), 1 = f64
    weighted sum (EngineInterface integrals, port V / I)."""

    terms: List[Tuple[int, Tuple[int, int, int], float]]
    mode: int


def _terms_from(fn, *args, mode):
    n = N.c_u64()
    N.check(fn(*args, None, 0, ctypes.byref(n)))
    arr = (N.ProbeTermC * max(1, n.value))()
    N.check(fn(*args, arr, n.value, ctypes.byref(n)))
    return ProbeTerms([(arr[i].component, tuple(arr[i].position), arr[i].weight)
                       for i in range(n.value)], mode)


def _u3(v):
    return (N.c_u64 * 3)(*[int(x) for x in v])


def voltage_probe(start, end, direction) -> ProbeTerms:
    """VoltageProbe (src/processing/probes.rs:63-131)."""
    return _terms_from(N.lib().oems_probe_voltage_terms, _u3(start), _u3(end), direction,
                       mode=N.PROBE_SUM_F32)


def current_probe(start, end, normal_direction) -> ProbeTerms:
    """CurrentProbe (src/processing/probes.rs:155-239)."""
    return _terms_from(N.lib().oems_probe_current_terms, _u3(start), _u3(end), normal_direction,
                       mode=N.PROBE_SUM_F32)


def voltage_integral(op: "Operator", start, stop) -> ProbeTerms:
    """EngineInterface::calc_voltage_integral between cell indices."""
    return _terms_from(N.lib().oems_probe_voltage_integral_terms, op.handle, _u3(start), _u3(stop),
                       mode=N.PROBE_SUM_F64)


def current_integral(op: "Operator", start, stop, normal_dir) -> ProbeTerms:
    """EngineInterface::calc_current_integral between cell indices."""
    return _terms_from(N.lib().oems_probe_current_integral_terms, op.handle, _u3(start), _u3(stop),
                       normal_dir, mode=N.PROBE_SUM_F64)


def port_probe(op: "Operator", position, direction, kind) -> ProbeTerms:
    """Lumped-port voltage (kind 0) or loop current (kind 1) at an E edge."""
    return _terms_from(N.lib().oems_probe_port_terms, op.handle, _u3(position), direction, kind,
                       mode=N.PROBE_SUM_F64)


class LumpedPort:
    """Lumped port on one E edge (python/openEMS/ports.py:155-209).

    A resistor R sits across the edge (folded into its Ca/Cb); with excite
    != 0 a voltage source excite * waveform drives it in series with R.  The
    port voltage is u = +E . dl and the port current i is the current the port
    delivers into the structure (minus the loop integral of H around the
    edge), so that an open port reads u = excite * waveform and a matched
    load reads half of it.  calc_port follows Port.CalcPort
    (python/openEMS/ports.py:115-153) on the engine's running DFTs, which use
    the single-sided 2 dt scaling of utilities.DFT_time2freq (:21-35).
    """

    def __init__(self, port_nr: int, R: float, position, direction: int, excite: float = 0.0,
                 eps_r: float = 1.0):
        if direction not in (0, 1, 2):
            raise N.ConfigError("LumpedPort direction must be 0, 1 or 2")
        if R <= 0:
            raise N.ConfigError("LumpedPort needs a positive resistance")
        self.number = port_nr
        self.R = float(R)
        self.Z_ref = float(R)
        self.position = tuple(int(v) for v in position)
        self.direction = int(direction)
        self.excite = float(excite)
        self.eps_r = float(eps_r)
        self.source_scale = None
        self.freqs = None

    def apply(self, op: Operator) -> "LumpedPort":
        """Writes the port resistor into the operator's coefficients."""
        self.source_scale = op.set_lumped(self.position, self.direction, resistance=self.R,
                                          eps_r=self.eps_r)
        self._op = op
        return self

    def excitation(self, waveform: Excitation) -> Excitation:
        """waveform's time signal as this port's soft source."""
        if self.source_scale is None:
            raise N.ConfigError("LumpedPort.apply(operator) must run first")
        return Excitation(waveform.excitation_type, tuple(waveform.params), self.direction,
                          self.position, waveform.amplitude * self.excite * self.source_scale, True)

    def add_probes(self, engine: "Engine", freqs) -> "LumpedPort":
        """u / i probes and their running DFTs at freqs (Hz)."""
        u = port_probe(self._op, self.position, self.direction, 0)
        i = port_probe(self._op, self.position, self.direction, 1)
        u = ProbeTerms([(c, q, -w) for c, q, w in u.terms], u.mode)
        i = ProbeTerms([(c, q, -w) for c, q, w in i.terms], i.mode)
        self.u_probe = engine.add_probe(u)
        self.i_probe = engine.add_probe(i)
        self.freqs = np.asarray(freqs, dtype=np.float64)
        self.u_dft = engine.add_probe_dft(self.u_probe, self.freqs)
        self.i_dft = engine.add_probe_dft(self.i_probe, self.freqs)
        return self

    def calc_port(self, engine: "Engine", ref_impedance: Optional[float] = None) -> "LumpedPort":
        """Port.CalcPort (python/openEMS/ports.py:115-153) without the
        reference-plane shift, which a lumped port does not support."""
        if ref_impedance is not None:
            self.Z_ref = float(ref_impedance)
        Z = self.Z_ref
        self.uf_tot = engine.probe_dft(self.u_dft)
        self.if_tot = engine.probe_dft(self.i_dft)
        self.uf_inc = 0.5 * (self.uf_tot + self.if_tot * Z)
        self.if_inc = 0.5 * (self.if_tot + self.uf_tot / Z)
        self.uf_ref = self.uf_tot - self.uf_inc
        self.if_ref = self.if_inc - self.if_tot
        self.P_inc = 0.5 * np.real(self.uf_inc * np.conj(self.if_inc))
        self.P_ref = 0.5 * np.real(self.uf_ref * np.conj(self.if_ref))
        self.P_acc = 0.5 * np.real(self.uf_tot * np.conj(self.if_tot))
        return self

    def s11(self) -> np.ndarray:
        return self.uf_ref / self.uf_inc

    def z_in(self) -> np.ndarray:
        return self.uf_tot / self.if_tot


class ExcitationType(enum.IntEnum):
    Gaussian = 0
    Sinusoidal = 1
    GaussianModulated = 2
    Dirac = 3
    Step = 4
    Custom = 5  # sampled (times, values), linearly interpolated


@dataclass
class Excitation:
    """Excitation (src/fdtd/excitation.rs:46-226).

    params: Gaussian (t0, tau); Sinusoidal (frequency,); GaussianModulated
    (frequency, t0, tau); Dirac / Step (); Custom (): its waveform is
    `times` / `values` (seconds, amplitudes), evaluated here on the host
    and passed to the engine as a sampled ScheduledExcitation like every
    other kind.
    """

    excitation_type: ExcitationType
    params: Tuple[float, ...]
    direction: int
    position: Tuple[int, int, int]
    amplitude: float = 1.0
    soft_source: bool = True
    times: Tuple[float, ...] = ()
    values: Tuple[float, ...] = ()

    @classmethod
    def _from_c(cls, c: N.ExcitationC):
        kind = ExcitationType(c.kind)
        npar = {0: 2, 1: 1, 2: 3, 3: 0, 4: 0}[int(kind)]
        return cls(kind, tuple(c.params[:npar]), int(c.direction), tuple(int(v) for v in c.position),
                   float(c.amplitude), bool(c.soft_source))

    @staticmethod
    def _pos(position):
        p = (N.c_u64 * 3)()
        for a in range(3):
            p[a] = int(position[a])
        return p

    @classmethod
    def gaussian(cls, center_freq, bandwidth, direction, position):
        c = N.ExcitationC()
        N.check(N.lib().oems_excitation_gaussian(center_freq, bandwidth, direction,
                                                 cls._pos(position), ctypes.byref(c)))
        return cls._from_c(c)

    @classmethod
    def gaussian_pulse(cls, tau, t0, direction, position, amplitude=1.0):
        """ExcitationType::Gaussian { t0, tau } built directly."""
        return cls(ExcitationType.Gaussian, (t0, tau), direction, tuple(position), amplitude, True)

    @classmethod
    def gaussian_modulated(cls, center_freq, bandwidth, direction, position):
        c = N.ExcitationC()
        N.check(N.lib().oems_excitation_gaussian_modulated(center_freq, bandwidth, direction,
                                                           cls._pos(position), ctypes.byref(c)))
        return cls._from_c(c)

    @classmethod
    def sinusoidal(cls, frequency, direction, position):
        c = N.ExcitationC()
        N.check(N.lib().oems_excitation_sinusoidal(frequency, direction, cls._pos(position),
                                                   ctypes.byref(c)))
        return cls._from_c(c)

    @classmethod
    def dirac(cls, amplitude, direction, position):
        c = N.ExcitationC()
        N.check(N.lib().oems_excitation_dirac(amplitude, direction, cls._pos(position),
                                              ctypes.byref(c)))
        return cls._from_c(c)

    @classmethod
    def custom(cls, times, values, direction, position, amplitude=1.0):
        """ExcitationType::Custom { times, values } (src/fdtd/excitation.rs:35-41)."""
        if len(times) != len(values):
            raise N.ConfigError("custom waveform: times and values differ in length")
        return cls(ExcitationType.Custom, (), direction, tuple(position), float(amplitude), True,
                   tuple(float(t) for t in times), tuple(float(v) for v in values))

    def with_amplitude(self, amplitude):
        self.amplitude = float(amplitude)
        return self

    def hard_source(self):
        self.soft_source = False
        return self

    def to_c(self) -> N.ExcitationC:
        if self.excitation_type == ExcitationType.Custom:
            raise N.ConfigError("a custom waveform runs as a sampled ScheduledExcitation (EngineBatch), "
                                "not through the analytic host excitation")
        c = N.ExcitationC()
        c.kind = int(self.excitation_type)
        c.direction = int(self.direction)
        for a in range(3):
            c.position[a] = int(self.position[a])
        for a, v in enumerate(self.params):
            c.params[a] = float(v)
        c.amplitude = float(self.amplitude)
        c.soft_source = int(bool(self.soft_source))
        return c

    def _custom_value(self, t: float) -> float:
        """Linear interpolation of the custom waveform, clamped at both ends
        (excitation.rs:177-197, the same bracketing loop)."""
        ts, vs = self.times, self.values
        if not ts:
            raise N.ConfigError("custom waveform without samples")
        if t <= ts[0]:
            return vs[0]
        if t >= ts[-1]:
            return vs[-1]
        i = 0
        while i < len(ts) - 1 and ts[i + 1] < t:
            i += 1
        alpha = (t - ts[i]) / (ts[i + 1] - ts[i])
        return vs[i] + alpha * (vs[i + 1] - vs[i])

    def evaluate(self, t: float) -> float:
        if self.excitation_type == ExcitationType.Custom:
            return self.amplitude * self._custom_value(float(t))
        c = self.to_c()
        return N.lib().oems_excitation_evaluate(ctypes.byref(c), t)

    def sample(self, start_timestep: int, num_timesteps: int, dt: float) -> np.ndarray:
        """(f32) evaluate((start + n) dt), t in f64 (batch.rs:110-129)."""
        if self.excitation_type == ExcitationType.Custom:
            return np.array([self.evaluate((start_timestep + n) * dt) for n in range(num_timesteps)],
                            dtype=np.float32)
        out = np.empty(num_timesteps, dtype=np.float32)
        c = self.to_c()
        N.check(N.lib().oems_excitation_sample(ctypes.byref(c), start_timestep, num_timesteps, dt,
                                               N.fptr(out)))
        return out

    def duration(self) -> float:
        """src/fdtd/excitation.rs:203-213."""
        if self.excitation_type in (ExcitationType.Gaussian, ExcitationType.GaussianModulated):
            t0, tau = self.params[-2], self.params[-1]
            return t0 + 6.0 * tau
        if self.excitation_type == ExcitationType.Custom:
            return self.times[-1] if self.times else 0.0
        return float("inf")

    def is_active(self, t: float) -> bool:
        """src/fdtd/excitation.rs:216-225."""
        k = self.excitation_type
        if k in (ExcitationType.Gaussian, ExcitationType.GaussianModulated):
            return t <= self.params[-2] + 6.0 * self.params[-1]
        if k == ExcitationType.Dirac:
            return abs(t) < 1e-15
        if k == ExcitationType.Custom:
            return t <= (self.times[-1] if self.times else 0.0)
        return True


def waveguide_te10(a: float, freq: float, position: int, ny: int) -> List[Excitation]:
    """waveguide_te10 (src/fdtd/excitation.rs:229-252): y-directed sinusoidal
    point sources at (0, j, position), j = 1 .. ny - 2, with amplitude
    sin(pi j / (ny - 1)) where that exceeds 0.01 (`a` is unused there too)."""
    out = []
    for j in range(1, ny - 1):
        amp = float(np.sin(np.pi * (j / (ny - 1))))
        if amp > 0.01:
            out.append(Excitation.sinusoidal(freq, 1, (0, j, position)).with_amplitude(amp))
    return out


@dataclass
class ScheduledExcitation:
    """ScheduledExcitation with a Sampled waveform (src/fdtd/batch.rs:71-129)."""

    position: Tuple[int, int, int]
    direction: int
    soft_source: bool
    samples: np.ndarray

    @classmethod
    def from_excitation(cls, exc: Excitation, start_timestep: int, num_timesteps: int, dt: float):
        return cls(tuple(exc.position), exc.direction, exc.soft_source,
                   exc.sample(start_timestep, num_timesteps, dt))


# ---------------------------------------------------------------------------
# batch protocol
# ---------------------------------------------------------------------------


@dataclass
class TerminationConfig:
    max_timesteps: Optional[int] = None
    energy_decay_db: Optional[float] = None
    check_interval: int = 100


@dataclass
class EnergyMonitorConfig:
    sample_interval: int = 0
    track_peak: bool = False
    decay_threshold: Optional[float] = None


@dataclass
class EngineBatch:
    """EngineBatch (src/fdtd/batch.rs:17-32).  Extensions are attached to the
    engine (Engine.add_cpml) instead of being passed per batch."""

    num_steps: Optional[int] = None
    excitations: List[ScheduledExcitation] = field(default_factory=list)
    termination: TerminationConfig = field(default_factory=TerminationConfig)
    energy_monitoring: EnergyMonitorConfig = field(default_factory=EnergyMonitorConfig)
    initial_peak_energy: float = 0.0


class TerminationReason(enum.IntEnum):
    StepsCompleted = 0
    EnergyDecay = 1
    ExtensionStop = 2


@dataclass
class EnergySample:
    timestep: int
    e_energy: float
    h_energy: float
    total_energy: float


@dataclass
class BatchResult:
    timesteps_executed: int
    termination_reason: TerminationReason
    final_decay_db: float
    energy_samples: List[EnergySample]
    peak_energy: float
    elapsed_time: float


# ---------------------------------------------------------------------------
# engine
# ---------------------------------------------------------------------------


def _request(theta, phi, radius, center, lines, keep):
    th = np.ascontiguousarray(theta, dtype=np.float64).reshape(-1)
    ph = np.ascontiguousarray(phi, dtype=np.float64).reshape(-1)
    keep += [th, ph]
    q = N.Nf2ffRequestC()
    q.theta = th.ctypes.data_as(ctypes.POINTER(N.c_f64))
    q.ntheta = len(th)
    q.phi = ph.ctypes.data_as(ctypes.POINTER(N.c_f64))
    q.nphi = len(ph)
    q.radius = float(radius)
    for a in range(3):
        q.center[a] = float(center[a])
        if lines is not None and lines[a] is not None:
            la = np.ascontiguousarray(lines[a], dtype=np.float64)
            keep.append(la)
            q.lines[a] = la.ctypes.data_as(ctypes.POINTER(N.c_f64))
    return q, len(th), len(ph)


def _result(nt, np_, keep):
    et = np.zeros(2 * nt * np_)
    ep = np.zeros(2 * nt * np_)
    pr = np.zeros(nt * np_)
    keep += [et, ep, pr]
    r = N.Nf2ffResultC()
    r.e_theta = et.ctypes.data_as(ctypes.POINTER(N.c_f64))
    r.e_phi = ep.ctypes.data_as(ctypes.POINTER(N.c_f64))
    r.p_rad = pr.ctypes.data_as(ctypes.POINTER(N.c_f64))
    return r, et, ep, pr


@dataclass
class Nf2ffResults:
    """nf2ff_results (python/openEMS/nf2ff.py:167-220): per frequency
    E_theta, E_phi, E_norm, E_cprh, E_cplh, P_rad (ntheta x nphi) and Dmax,
    Prad; theta / phi in radians, r the observation radius (m)."""

    theta: np.ndarray
    phi: np.ndarray
    r: float
    freq: np.ndarray
    E_theta: List[np.ndarray] = field(default_factory=list)
    E_phi: List[np.ndarray] = field(default_factory=list)
    E_norm: List[np.ndarray] = field(default_factory=list)
    E_cprh: List[np.ndarray] = field(default_factory=list)
    E_cplh: List[np.ndarray] = field(default_factory=list)
    P_rad: List[np.ndarray] = field(default_factory=list)
    Dmax: List[float] = field(default_factory=list)
    Prad: List[float] = field(default_factory=list)

    def _append(self, et, ep, pr, nt, np_, prad, dmax):
        Et = (et[0::2] + 1j * et[1::2]).reshape(nt, np_)
        Ep = (ep[0::2] + 1j * ep[1::2]).reshape(nt, np_)
        _, PHI = np.meshgrid(self.theta, self.phi, indexing="ij")
        self.E_theta.append(Et)
        self.E_phi.append(Ep)
        self.E_norm.append(np.sqrt(np.abs(Et) ** 2 + np.abs(Ep) ** 2))
        self.E_cprh.append((np.cos(PHI) + 1j * np.sin(PHI)) * (Et + 1j * Ep) / np.sqrt(2.0))
        self.E_cplh.append((np.cos(PHI) - 1j * np.sin(PHI)) * (Et - 1j * Ep) / np.sqrt(2.0))
        self.P_rad.append(pr.reshape(nt, np_))
        self.Prad.append(prad)
        self.Dmax.append(dmax)


class Nf2ffBox:
    """nf2ff recording box (python/openEMS/nf2ff.py:26-97) with
    frequency-domain recording on an engine; start / stop are node planes
    (cell indices) with 1 <= start < stop <= n - 1."""

    def __init__(self, engine: "Engine", start, stop, frequency, directions=(True,) * 6,
                 interval: int = 1, name: str = "nf2ff"):
        self.engine = engine
        self.name = name
        self.start = tuple(int(v) for v in start)
        self.stop = tuple(int(v) for v in stop)
        self.freq = np.atleast_1d(np.asarray(frequency, dtype=np.float64))
        self.directions = tuple(bool(v) for v in directions)
        d = N.Nf2ffBoxDescC()
        for a in range(3):
            d.start[a], d.stop[a] = self.start[a], self.stop[a]
        for f in range(6):
            d.directions[f] = int(self.directions[f])
        d.interval = int(interval)
        bid = N.c_i32()
        N.check(N.lib().oems_engine_add_nf2ff_box(engine.handle, ctypes.byref(d),
                                                  self.freq.ctypes.data_as(ctypes.POINTER(N.c_f64)),
                                                  len(self.freq), ctypes.byref(bid)))
        self.box_id = bid.value

    def face(self, face: int, freq_index: int) -> np.ndarray:
        """Raw accumulators (4, nb, nc) = Eb, Ec, Hb, Hc of one face."""
        a = face // 2
        b, c = (a + 1) % 3, (a + 2) % 3
        nb, nc = self.stop[b] - self.start[b] + 1, self.stop[c] - self.start[c] + 1
        out = np.zeros(8 * nb * nc)
        N.check(N.lib().oems_engine_read_nf2ff_face(self.engine.handle, self.box_id, face, freq_index,
                                                    out.ctypes.data_as(ctypes.POINTER(N.c_f64)),
                                                    len(out), None))
        return (out[0::2] + 1j * out[1::2]).reshape(4, nb, nc)

    def calc_nf2ff(self, freq, theta, phi, radius=1.0, center=(0.0, 0.0, 0.0), lines=None,
                   degrees=True) -> Nf2ffResults:
        """CalcNF2FF (python/openEMS/nf2ff.py:98-165): freq one or several of
        the recorded frequencies; theta / phi in degrees unless degrees=False;
        lines: mesh lines in metres per axis (default: uniform cells)."""
        th = np.deg2rad(theta) if degrees else np.asarray(theta, dtype=np.float64)
        ph = np.deg2rad(phi) if degrees else np.asarray(phi, dtype=np.float64)
        th, ph = np.atleast_1d(th).astype(np.float64), np.atleast_1d(ph).astype(np.float64)
        freqs = np.atleast_1d(np.asarray(freq, dtype=np.float64))
        res = Nf2ffResults(th, ph, float(radius), freqs)
        for f in freqs:
            hit = np.nonzero(np.isclose(self.freq, f, rtol=1e-9, atol=0))[0]
            if len(hit) == 0:
                raise N.ConfigError(f"frequency {f} is not recorded by this NF2FF box")
            keep = []
            q, nt, np_ = _request(th, ph, radius, center, lines, keep)
            r, et, ep, pr = _result(nt, np_, keep)
            N.check(N.lib().oems_engine_nf2ff(self.engine.handle, self.box_id, int(hit[0]),
                                              ctypes.byref(q), ctypes.byref(r)))
            res._append(et, ep, pr, nt, np_, r.prad, r.dmax)
        return res


def nf2ff_surface(points: np.ndarray, freq: float, theta, phi, radius=1.0, center=(0.0, 0.0, 0.0),
                  device: int = -1) -> Nf2ffResults:
    """Far field of a point list (n, 16): x y z weight, J (re, im) x 3,
    M (re, im) x 3; theta / phi in radians."""
    pts = np.ascontiguousarray(points, dtype=np.float64).reshape(-1, 16)
    th, ph = np.atleast_1d(theta).astype(np.float64), np.atleast_1d(phi).astype(np.float64)
    keep = []
    q, nt, np_ = _request(th, ph, radius, center, None, keep)
    r, et, ep, pr = _result(nt, np_, keep)
    N.check(N.lib().oems_nf2ff_surface(device, pts.ctypes.data_as(ctypes.POINTER(N.c_f64)), len(pts),
                                       float(freq), ctypes.byref(q), ctypes.byref(r)))
    res = Nf2ffResults(th, ph, float(radius), np.array([freq]))
    res._append(et, ep, pr, nt, np_, r.prad, r.dmax)
    return res


class EngineType(enum.Enum):
    """The engine is CUDA-only; `Cuda` is the single implementation."""

    Cuda = "cuda"


def compress_coefficients(coef) -> Tuple[np.ndarray, np.ndarray]:
    """CompressedCoefficients::from_fields (src/fdtd/compressed.rs:125-192)
    as the engine's compressed storage does it (oems_compress_coefficients):
    coef holds the 12 per-cell arrays ca0..2, cb0..2, da0..2, db0..2 (first
    axis; e.g. Operator.coefficients()); returns (ids, table): a uint16 set
    per cell (C order of the other axes) and the unique sets (n, 12) float32,
    compared bit for bit."""
    c = np.ascontiguousarray(coef, dtype=np.float32)
    if c.shape[0] != 12:
        raise N.ConfigError("12 coefficient arrays expected")
    flat = c.reshape(12, -1)
    n = flat.shape[1]
    ptrs = (ctypes.c_void_p * 12)(*[flat[a].ctypes.data for a in range(12)])
    ids = np.empty(n, dtype=np.uint16)
    table = np.empty((65536, 12), dtype=np.float32)
    nu = N.c_u32()
    N.check(N.lib().oems_compress_coefficients(ptrs, n, ids.ctypes.data, table.ctypes.data, 65536, ctypes.byref(nu)))
    return ids.reshape(c.shape[1:]), table[:nu.value].copy()


class Engine:
    """CUDA engine (EngineImpl, src/fdtd/engine_impl.rs:24-71) on one GPU."""

    def __init__(self, operator: Operator, engine_type: EngineType = EngineType.Cuda, *,
                 device: int = -1, compressed: bool = False, autotune: bool = True,
                 graphs: bool = True, kernels: str = "auto", storage: str = "f32"):
        """kernels: "auto" (tuner picks), "register", "staged" (bulk-async),
        "split" (staged between the x / y CPML slabs, register on them) or
        "zsplit" (plain register kernels on the CPML-free box, CPML register
        kernels on every slab cell) or "pipe" (pipelined register kernels:
        each thread's next x-planes copied into shared memory while it
        computes; float fields and full coefficients only).
        storage: field storage "f32", or "f16" / "bf16" (2 bytes per value,
        float arithmetic; register kernels, CPML, sources, probes, energies)."""
        if engine_type is not EngineType.Cuda:
            raise N.ConfigError("only the CUDA engine exists")
        if storage not in N.STORAGE_FLAGS:
            raise N.ConfigError(f"unknown field storage {storage!r}")
        flags = (N.ENGINE_COMPRESSED if compressed else 0) | (0 if autotune else N.ENGINE_NO_AUTOTUNE) \
            | (0 if graphs else N.ENGINE_NO_GRAPHS) \
            | {"auto": 0, "register": N.ENGINE_REGISTER_KERNELS, "staged": N.ENGINE_STAGED_KERNELS,
               "split": N.ENGINE_SPLIT_KERNELS, "zsplit": N.ENGINE_ZSPLIT_KERNELS,
               "pipe": N.ENGINE_PIPE_KERNELS}[kernels] \
            | N.STORAGE_FLAGS[storage]
        desc = N.OperatorDesc()
        N.check(N.lib().oems_operator_engine_desc(operator.handle, device, flags, ctypes.byref(desc)))
        h = ctypes.c_void_p()
        N.check(N.lib().oems_engine_create(ctypes.byref(desc), ctypes.byref(h)))
        self._h = h
        self.dims = operator.dimensions()
        self.dt = operator.timestep()
        self.num_probes = 0
        layers = operator.boundaries.cpml_layers() if operator.boundaries else (0,) * 6
        if any(layers):
            self.add_cpml(CpmlBoundaries(layers=layers))

    @classmethod
    def from_descriptor(cls, desc: N.OperatorDesc):
        self = cls.__new__(cls)
        h = ctypes.c_void_p()
        N.check(N.lib().oems_engine_create(ctypes.byref(desc), ctypes.byref(h)))
        self._h = h
        self.dims = (int(desc.nx), int(desc.ny), int(desc.nz))
        self.dt = float(desc.dt)
        self.num_probes = 0
        return self

    def close(self):
        h = getattr(self, "_h", None)
        if h:
            N.lib().oems_engine_destroy(h)
            self._h = None

    def __del__(self):
        # at interpreter exit the module globals (the library handle) may be
        # gone already; the process is ending and the driver frees the device
        try:
            self.close()
        except (TypeError, AttributeError):
            pass

    @property
    def handle(self):
        return self._h

    def add_cpml(self, cpml: CpmlBoundaries):
        d = cpml.to_c()
        N.check(N.lib().oems_engine_add_cpml(self._h, ctypes.byref(d)))

    def add_tfsf(self, cfg: TfsfConfig):
        """TF/SF plane source (TfsfBoundary)."""
        d = cfg.to_c()
        N.check(N.lib().oems_engine_add_tfsf(self._h, ctypes.byref(d)))

    def add_mur(self, mur: MurAbcConfig):
        d = mur.to_c()
        N.check(N.lib().oems_engine_add_mur(self._h, ctypes.byref(d)))

    def add_upml(self, pml: PmlBoundaries):
        d = pml.to_c()
        N.check(N.lib().oems_engine_add_upml(self._h, ctypes.byref(d)))

    def add_dispersive(self, material, cells):
        """Dispersive material (Drude / Lorentz / Debye) on cells (n, 3)."""
        c = np.ascontiguousarray(cells, dtype=np.uint64).reshape(-1, 3)
        d = material.to_c()
        N.check(N.lib().oems_engine_add_dispersive(self._h, ctypes.byref(d), c.ctypes.data, len(c)))

    def add_lumped_rlc(self, elements: Sequence[RlcElement]):
        arr = (N.LumpedRlcDescC * max(1, len(elements)))()
        for i, e in enumerate(elements):
            arr[i] = e.to_c()
        N.check(N.lib().oems_engine_add_lumped_rlc(self._h, arr, len(elements)))

    def add_point_probe(self, component: int, position) -> int:
        """FieldProbe-style value of one component at one cell."""
        p = (N.c_u64 * 3)(*[int(v) for v in position])
        pid = N.c_i32()
        N.check(N.lib().oems_engine_add_point_probe(self._h, component, p, ctypes.byref(pid)))
        self.num_probes += 1
        return pid.value

    def add_probe(self, terms: "ProbeTerms") -> int:
        """General probe from a term list (see probe_* builders)."""
        arr = (N.ProbeTermC * max(1, len(terms.terms)))()
        for i, (c, pos, w) in enumerate(terms.terms):
            arr[i].component = int(c)
            for a in range(3):
                arr[i].position[a] = int(pos[a])
            arr[i].weight = float(w)
        pid = N.c_i32()
        N.check(N.lib().oems_engine_add_probe(self._h, arr, len(terms.terms), terms.mode,
                                              ctypes.byref(pid)))
        self.num_probes += 1
        return pid.value

    def probe_traces(self) -> np.ndarray:
        """Traces of the most recent batch, shape (steps, probes), float64."""
        steps = N.c_u64()
        N.check(N.lib().oems_engine_read_probe_traces(self._h, None, 0, ctypes.byref(steps)))
        out = np.zeros((steps.value, self.num_probes), dtype=np.float64)
        if out.size:
            N.check(N.lib().oems_engine_read_probe_traces(
                self._h, out.ctypes.data_as(ctypes.POINTER(N.c_f64)), steps.value, None))
        return out

    def add_probe_dft(self, probe_id: int, freqs) -> int:
        f = np.ascontiguousarray(freqs, dtype=np.float64)
        did = N.c_i32()
        N.check(N.lib().oems_engine_add_probe_dft(self._h, probe_id,
                                                  f.ctypes.data_as(ctypes.POINTER(N.c_f64)), len(f),
                                                  ctypes.byref(did)))
        self._dft_sizes = getattr(self, "_dft_sizes", {})
        self._dft_sizes[did.value] = len(f)
        return did.value

    def probe_dft(self, dft_id: int) -> np.ndarray:
        n = self._dft_sizes[dft_id]
        out = np.zeros(2 * n, dtype=np.float64)
        N.check(N.lib().oems_engine_read_probe_dft(self._h, dft_id,
                                                   out.ctypes.data_as(ctypes.POINTER(N.c_f64))))
        return out[0::2] + 1j * out[1::2]

    def add_field_dft(self, region, freqs, components=0x3F, sub_sample=(1, 1, 1), interval=1) -> int:
        """Frequency-domain field dump (FrequencyDomainFieldDump) over the
        half-open region (i0, i1, j0, j1, k0, k1); components is a bit mask or
        "E" / "H" / "EH"."""
        if isinstance(components, str):
            components = {"E": 0x07, "H": 0x38, "EH": 0x3F, "HE": 0x3F}[components]
        d = N.FieldDftDescC()
        for a in range(6):
            d.region[a] = int(region[a])
        for a in range(3):
            d.sub_sample[a] = int(sub_sample[a])
        d.components = int(components)
        d.interval = int(interval)
        f = np.ascontiguousarray(freqs, dtype=np.float64)
        did = N.c_i32()
        N.check(N.lib().oems_engine_add_field_dft(self._h, ctypes.byref(d),
                                                  f.ctypes.data_as(ctypes.POINTER(N.c_f64)), len(f),
                                                  ctypes.byref(did)))
        ext = self.dims
        shape = []
        for a in range(3):
            lo, hi = min(int(region[2 * a]), ext[a]), min(int(region[2 * a + 1]), ext[a])
            ss = max(int(sub_sample[a]), 1)
            shape.append((max(hi - lo, 0) + ss - 1) // ss)
        self._fd_shapes = getattr(self, "_fd_shapes", {})
        self._fd_shapes[did.value] = tuple(shape)
        return did.value

    def field_dft(self, dump_id: int, freq_index: int, component: int) -> np.ndarray:
        """Complex accumulator of one component, shape of the sub-sampled region."""
        shape = self._fd_shapes[dump_id]
        n = int(np.prod(shape))
        out = np.zeros(2 * n, dtype=np.float64)
        N.check(N.lib().oems_engine_read_field_dft(self._h, dump_id, freq_index, component,
                                                   out.ctypes.data_as(ctypes.POINTER(N.c_f64)), n))
        return (out[0::2] + 1j * out[1::2]).reshape(shape)

    def run_batch(self, batch: EngineBatch) -> BatchResult:
        b, r, samples, cap, keep = _batch_c(batch)
        N.check(N.lib().oems_engine_run_batch(self._h, ctypes.byref(b), ctypes.byref(r)))
        return _batch_result(r, samples, cap)

    def current_timestep(self) -> int:
        t = N.c_u64()
        N.check(N.lib().oems_engine_current_timestep(self._h, ctypes.byref(t)))
        return int(t.value)

    timestep = current_timestep

    def read_fields(self) -> Tuple[np.ndarray, np.ndarray]:
        e = np.empty((3,) + tuple(self.dims), dtype=np.float32)
        h = np.empty_like(e)
        ep = (N.PF * 3)(*[N.fptr(e[c]) for c in range(3)])
        hp = (N.PF * 3)(*[N.fptr(h[c]) for c in range(3)])
        N.check(N.lib().oems_engine_read_fields(self._h, ep, hp))
        return e, h

    def write_fields(self, e: np.ndarray, h: np.ndarray) -> None:
        e = np.ascontiguousarray(e, dtype=np.float32)
        h = np.ascontiguousarray(h, dtype=np.float32)
        if e.shape != (3,) + tuple(self.dims) or h.shape != e.shape:
            raise N.InvalidArgumentError("fields must have shape (3, nx, ny, nz)")
        ep = (N.PF * 3)(*[N.fptr(e[c]) for c in range(3)])
        hp = (N.PF * 3)(*[N.fptr(h[c]) for c in range(3)])
        N.check(N.lib().oems_engine_write_fields(self._h, ep, hp))

    def reset(self) -> None:
        N.check(N.lib().oems_engine_reset(self._h))

    # -- checkpoint / resume (openems_b200.checkpoint) ----------------------

    def state_sections(self) -> List[Tuple[int, int, int]]:
        """(kind, bytes, variant) of every state section, in the engine's
        order; variant is the field storage type of the fields section (0
        float, 1 half, 2 bfloat16) and 0 for the others."""
        n = N.c_u64()
        N.check(N.lib().oems_engine_state_sections(self._h, None, 0, ctypes.byref(n)))
        arr = (N.StateSectionC * max(n.value, 1))()
        N.check(N.lib().oems_engine_state_sections(self._h, arr, n.value, ctypes.byref(n)))
        return [(int(arr[i].kind), int(arr[i].bytes), int(arr[i].variant)) for i in range(n.value)]

    def read_state(self, index: int, nbytes: int) -> bytearray:
        buf = bytearray(int(nbytes))
        ptr = (ctypes.c_char * len(buf)).from_buffer(buf) if buf else None  # no extra copy
        N.check(N.lib().oems_engine_read_state(self._h, int(index), ptr, int(nbytes)))
        return buf

    def write_state(self, index: int, data: bytes, variant: int = 0) -> None:
        """Writes section `index`; `variant` must be the section's (the field
        storage type for the fields section)."""
        data = bytes(data)
        N.check(N.lib().oems_engine_write_state(self._h, int(index), int(variant), data, len(data)))

    def state_counters(self) -> Tuple[int, int]:
        """(timestep, TF/SF step)."""
        t, f = N.c_u64(), N.c_u64()
        N.check(N.lib().oems_engine_get_state_counters(self._h, ctypes.byref(t), ctypes.byref(f)))
        return int(t.value), int(f.value)

    def set_state_counters(self, timestep: int, tfsf_step: int) -> None:
        N.check(N.lib().oems_engine_set_state_counters(self._h, int(timestep), int(tfsf_step)))

    def save_state(self) -> bytes:
        """The whole evolving state as a checkpoint blob."""
        from . import checkpoint
        return checkpoint.pack(self)

    def load_state(self, blob) -> None:
        """Continues from a checkpoint of an engine built the same way."""
        from . import checkpoint
        checkpoint.unpack(self, blob)

    def evaluate_probe(self, probe: "ProbeTerms") -> float:
        """A probe's value on the present fields, with the probe's arithmetic
        (VoltageProbe / CurrentProbe::sample, src/processing/probes.rs:98-239,
        called between steps)."""
        n = len(probe.terms)
        arr = (N.ProbeTermC * max(1, n))()
        for t, (c, pos, w) in enumerate(probe.terms):
            arr[t].component = c
            arr[t].position[:] = [int(v) for v in pos]
            arr[t].weight = w
        out = N.c_f64()
        N.check(N.lib().oems_engine_eval_terms(self._h, arr, n, probe.mode, ctypes.byref(out)))
        return out.value

    def energy(self) -> Tuple[float, float]:
        e, h = N.c_f64(), N.c_f64()
        N.check(N.lib().oems_engine_energy(self._h, ctypes.byref(e), ctypes.byref(h)))
        return e.value, h.value

    def set_kernel_profiling(self, enable: bool) -> None:
        N.check(N.lib().oems_engine_set_kernel_profiling(self._h, int(bool(enable))))

    def kernel_profile(self):
        """(H seconds, H launches, E seconds, E launches) since profiling was enabled."""
        hs, hn, es, en = N.c_f64(), N.c_u64(), N.c_f64(), N.c_u64()
        N.check(N.lib().oems_engine_kernel_profile(self._h, ctypes.byref(hs), ctypes.byref(hn),
                                                   ctypes.byref(es), ctypes.byref(en)))
        return hs.value, int(hn.value), es.value, int(en.value)

    def launch_info(self) -> dict:
        v = [N.c_i32() for _ in range(6)]
        N.check(N.lib().oems_engine_launch_info(self._h, *[ctypes.byref(x) for x in v]))
        keys = ("staged", "threads", "ichunk", "rows_per_tile", "stages", "grid")
        return {k: int(x.value) for k, x in zip(keys, v)}

    def tune_report(self) -> list:
        """Launch shapes the autotuner timed for this grid: dicts with kind (0
        register, 1 staged, 2 staged interior + register slabs, 3 register
        z-only interior + full-CPML slabs), threads, ichunk, extra (stages or
        prefetch distance), reps and ms (device time of the timed H + E pairs)."""
        n = N.c_u64()
        N.check(N.lib().oems_engine_tune_report(self._h, None, 0, ctypes.byref(n)))
        rec = np.zeros(int(n.value), dtype=[("kind", "<i4"), ("threads", "<i4"), ("ichunk", "<i4"),
                                            ("extra", "<i4"), ("reps", "<i4"), ("ms", "<f4")])
        if len(rec):
            N.check(N.lib().oems_engine_tune_report(self._h, rec.ctypes.data, len(rec), ctypes.byref(n)))
        return [{k: (float(r[k]) if k == "ms" else int(r[k])) for k in rec.dtype.names} for r in rec]

    def last_batch_stats(self) -> Tuple[int, float]:
        n, s = N.c_u64(), N.c_f64()
        N.check(N.lib().oems_engine_last_batch_stats(self._h, ctypes.byref(n), ctypes.byref(s)))
        return int(n.value), float(s.value)


def _batch_c(batch: "EngineBatch"):
    """The C form of an EngineBatch: (batch, result with its energy sample
    buffer, that buffer, its capacity, the arrays the batch borrows)."""
    num_steps = batch.num_steps
    if num_steps is None:
        num_steps = batch.termination.max_timesteps
    if num_steps is None:
        raise N.ConfigError("EngineBatch needs num_steps or termination.max_timesteps")
    keep = []
    arr = (N.ScheduledExcitationC * max(1, len(batch.excitations)))()
    for x, e in enumerate(batch.excitations):
        s = np.ascontiguousarray(e.samples, dtype=np.float32)
        keep.append(s)
        for a in range(3):
            arr[x].position[a] = int(e.position[a])
        arr[x].direction = int(e.direction)
        arr[x].soft_source = int(bool(e.soft_source))
        arr[x].samples = N.fptr(s)
        arr[x].num_samples = len(s)
    keep.append(arr)
    b = N.BatchC()
    b.num_steps = int(num_steps)
    b.excitations = arr
    b.num_excitations = len(batch.excitations)
    b.has_energy_decay_db = int(batch.termination.energy_decay_db is not None)
    b.energy_decay_db = float(batch.termination.energy_decay_db or 0.0)
    b.check_interval = int(batch.termination.check_interval)
    b.sample_interval = int(batch.energy_monitoring.sample_interval)
    b.track_peak = int(bool(batch.energy_monitoring.track_peak))
    b.initial_peak_energy = float(batch.initial_peak_energy)
    si = batch.energy_monitoring.sample_interval
    cap = (int(num_steps) // si + 2) if si > 0 else 1
    samples = (N.EnergySampleC * cap)()
    r = N.BatchResultC()
    r.energy_samples = samples
    r.energy_capacity = cap
    return b, r, samples, cap, keep


def _batch_result(r, samples, cap) -> "BatchResult":
    es = [EnergySample(int(s.timestep), s.e_energy, s.h_energy, s.total_energy)
          for s in samples[:min(cap, r.num_energy_samples)]]
    return BatchResult(int(r.timesteps_executed), TerminationReason(r.termination_reason),
                       float(r.final_decay_db), es, float(r.peak_energy), float(r.elapsed_seconds))


class Pack:
    """Several engines stepped by shared launches (oems_pack_*): one launch
    per half-step of the plain update kernels over the grids without CPML
    and one of the CPML kernels over the grids with it, a post-step launch
    with a CTA per engine and two energy launches for all.  Each engine ends
    a batch with the bits oems_engine_run_batch would give it.  The first
    batch tunes the launch shape (CTA size, x-planes per work item, CPML
    grids whole or split into box and slabs) unless set_shape chose one.  The engines need full coefficients and only CPML,
    sources, probes and probe DFTs; keep them alive while the pack exists."""

    def __init__(self, engines: Sequence["Engine"]):
        self.engines = list(engines)
        arr = (ctypes.c_void_p * len(self.engines))(*[e._h for e in self.engines])
        h = ctypes.c_void_p()
        N.check(N.lib().oems_pack_create(arr, len(self.engines), ctypes.byref(h)))
        self._h = h

    def close(self):
        h = getattr(self, "_h", None)
        if h:
            N.lib().oems_pack_destroy(h)
            self._h = None

    def __del__(self):
        # at interpreter exit the module globals (the library handle) may be
        # gone already; the process is ending and the driver frees the device
        try:
            self.close()
        except (TypeError, AttributeError):
            pass

    def set_shape(self, threads: int, ichunk: int, split: int = 0):
        """CTAs of `threads` over work items of `ichunk` x-planes; split: 0
        CPML grids whole, 1 as their CPML-free box plus their slab cells, 2 / 3
        as 1 with the slab launch on a second stream beside the box launch
        (3: the box launch's grid cut by one CTA per SM).  No tuning."""
        N.check(N.lib().oems_pack_set_shape(self._h, threads, ichunk, int(split)))

    def shape(self) -> tuple:
        """(threads, ichunk, split) of the update launches."""
        t, c, sp = N.c_i32(), N.c_i32(), N.c_i32()
        N.check(N.lib().oems_pack_shape(self._h, ctypes.byref(t), ctypes.byref(c), ctypes.byref(sp)))
        return t.value, c.value, sp.value

    def run_batch(self, batches: Sequence[Optional["EngineBatch"]]):
        """batches[i] for engine i (None: engine i sits this batch out); the
        batches share num_steps, the energy intervals and whether they carry
        a decay end condition, and the engines their timestep.  Returns a
        BatchResult per engine (None where skipped); raises NumericalError
        if an engine's energy stopped being finite (the others still ran)."""
        n = len(self.engines)
        if len(batches) != n:
            raise N.ConfigError("one batch (or None) per engine of the pack")
        conv = [(_batch_c(b) if b is not None else None) for b in batches]
        bp = (ctypes.c_void_p * n)(*[ctypes.addressof(c[0]) if c else None for c in conv])
        res = (N.BatchResultC * n)()
        for i, c in enumerate(conv):
            if c:
                res[i] = c[1]
        st = (N.c_i32 * n)()
        N.check(N.lib().oems_pack_run_batch(self._h, bp, res, st))
        out = [(_batch_result(res[i], c[2], c[3]) if c else None) for i, c in enumerate(conv)]
        bad = [i for i in range(n) if st[i] != N.OK]
        if bad:
            N.check(st[bad[0]])
        return out


# ---------------------------------------------------------------------------
# simulation
# ---------------------------------------------------------------------------


@dataclass
class EndCondition:
    """EndCondition (src/fdtd/simulation.rs:36-49): kind 0 Timesteps(n),
    1 EnergyDecay(dB), 2 SimulationTime(s)."""

    kind: int = 0
    value: float = 10000.0

    @classmethod
    def timesteps(cls, n: int):
        return cls(0, float(n))

    @classmethod
    def energy_decay(cls, db: float):
        return cls(1, float(db))

    @classmethod
    def simulation_time(cls, t: float):
        return cls(2, float(t))


@dataclass
class TimestepInfo:
    """TimestepInfo (src/fdtd/timestep.rs:7-75): dt = 0.99 of the 3D CFL
    limit of the grid's smallest spacings, the Nyquist frequency, the cell
    count and the reference's memory estimate (18 f32 arrays per cell)."""

    dt: float
    dt_max: float
    nyquist_freq: float
    num_cells: int
    memory_bytes: int

    @classmethod
    def calculate(cls, grid: Grid) -> "TimestepInfo":
        from .constants import C0
        dx, dy, dz = grid.cell_size()
        nx, ny, nz = grid.dimensions()
        dt_max = 1.0 / (C0 * math.sqrt(1.0 / (dx * dx) + 1.0 / (dy * dy) + 1.0 / (dz * dz)))
        dt = 0.99 * dt_max
        n = nx * ny * nz
        return cls(dt, dt_max, 1.0 / (2.0 * dt), n, n * 18 * 4)

    def timesteps_for_duration(self, duration: float) -> int:
        return int(math.ceil(duration / self.dt))

    def timesteps_per_period(self, frequency: float) -> float:
        return 1.0 / (frequency * self.dt)

    def memory_display(self) -> str:
        b = float(self.memory_bytes)
        if b < 1024.0:
            return f"{b:.0f} B"
        if b < 1024.0 ** 2:
            return f"{b / 1024.0:.2f} KB"
        if b < 1024.0 ** 3:
            return f"{b / 1024.0 ** 2:.2f} MB"
        return f"{b / 1024.0 ** 3:.2f} GB"


class SimulationState(enum.Enum):
    """SimulationState (src/fdtd/simulation.rs:21-32)."""

    Created = 0
    Ready = 1
    Running = 2
    Finished = 3
    Stopped = 4


@dataclass
class SimulationStats:
    timesteps: int
    sim_time: float
    wall_time: float
    peak_energy: float
    final_energy: float
    speed_mcells_per_sec: float


class Simulation:
    """Simulation (src/fdtd/simulation.rs:69-360) driving the CUDA engine.

    Unlike the reference, whose Simulation cannot carry materials, the
    operator is exposed as `sim.operator` for set_material / set_pec before
    the first run.
    """

    def __init__(self, grid: Grid, boundaries: Optional[BoundaryConditions] = None, *,
                 device: int = -1, compressed: bool = False):
        self.grid = grid
        self.boundaries = boundaries if boundaries is not None else BoundaryConditions()
        self.operator = Operator(grid, self.boundaries)
        self.excitations: List[Excitation] = []
        self.end_condition = EndCondition()
        self.batch_size: Optional[int] = None
        self.device = device
        self.flags = N.ENGINE_COMPRESSED if compressed else 0
        self.verbose = 1
        self.show_progress = True
        self._state = SimulationState.Created
        self._sim = None

    def __del__(self):
        # at interpreter exit the module globals (the library handle) may be
        # gone already; the process is ending and the driver frees the device
        try:
            s = getattr(self, "_sim", None)
            if s:
                N.lib().oems_simulation_destroy(s)
                self._sim = None
        except (TypeError, AttributeError):
            pass

    def set_boundaries(self, boundaries: BoundaryConditions):
        self.boundaries = boundaries
        self.operator.boundaries = boundaries
        return self

    def add_excitation(self, exc: Excitation):
        self.excitations.append(exc)
        return self

    def set_end_condition(self, cond: EndCondition):
        self.end_condition = cond
        return self

    def set_batch_size(self, n: Optional[int]):
        self.batch_size = n
        return self

    def set_engine_type(self, engine_type: "EngineType"):
        """Only EngineType.Cuda exists; the reference's CPU engine types are
        refused like in Engine()."""
        if engine_type is not EngineType.Cuda:
            raise N.ConfigError("only the CUDA engine exists")
        return self

    def set_verbose(self, level: int):
        """Kept for the reference's builder chain (its log level); this
        mirror logs nothing."""
        self.verbose = int(level)
        return self

    def set_show_progress(self, show: bool):
        """Kept for the reference's builder chain (its progress bar); this
        mirror draws none."""
        self.show_progress = bool(show)
        return self

    def timestep_info(self) -> TimestepInfo:
        return TimestepInfo.calculate(self.grid)

    def state(self) -> SimulationState:
        return self._state

    def timestep(self) -> float:
        return self.operator.timestep()

    def setup(self):
        if self._sim is not None:
            raise N.ConfigError("Simulation already set up")
        h = ctypes.c_void_p()
        N.check(N.lib().oems_simulation_create(self.operator.handle, self.device, self.flags,
                                               ctypes.byref(h)))
        self._sim = h
        for e in self.excitations:
            c = e.to_c()
            N.check(N.lib().oems_simulation_add_excitation(h, ctypes.byref(c)))
        N.check(N.lib().oems_simulation_set_end_condition(h, self.end_condition.kind,
                                                          self.end_condition.value))
        N.check(N.lib().oems_simulation_set_batch_size(h, int(self.batch_size or 0)))
        layers = self.boundaries.cpml_layers()
        if any(layers):
            d = CpmlBoundaries(layers=layers).to_c()
            N.check(N.lib().oems_simulation_set_cpml(h, ctypes.byref(d)))
        N.check(N.lib().oems_simulation_setup(h))
        self._state = SimulationState.Ready

    def run(self) -> SimulationStats:
        """Sets up if needed, then runs (Simulation::run, simulation.rs:200-360):
        the state goes Ready -> Running -> Finished; a second run is refused
        as in the reference."""
        if self._state == SimulationState.Created:
            self.setup()
        if self._state != SimulationState.Ready:
            raise N.ConfigError("Simulation not ready to run")
        self._state = SimulationState.Running
        st = N.SimulationStatsC()
        N.check(N.lib().oems_simulation_run(self._sim, ctypes.byref(st)))
        self._state = SimulationState.Finished
        return SimulationStats(int(st.timesteps), st.sim_time, st.wall_time, st.peak_energy,
                               st.final_energy, st.speed_mcells_per_sec)

    def engine_handle(self):
        return N.lib().oems_simulation_engine(self._sim) if self._sim else None
