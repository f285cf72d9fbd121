"""The engine interface over a CUDA engine's resident fields.

`EngineInterface` and `EngineInterfaceMut` (src/fdtd/engine_interface.rs:
10-595) give processing code and extensions field values at physical
positions, derived fields, line and surface integrals and energies.  The
reference holds references to host arrays; here the fields stay on the GPU
and every read is a launch over the queries (`oems_engine_sample`,
`oems_engine_integral`), so a batch of positions costs one launch.  Values
carry the bits of the reference's f64 arithmetic (same snap, same
interpolation order, each operation rounded on its own).

Method names, arguments and defaults follow the reference; the batched forms
(`e_fields`, `h_fields`, `sample`) take an (n, 3) array of positions.
"""
from __future__ import annotations

import ctypes
import enum
from typing import Optional, Sequence, Tuple

import numpy as np

from . import _native as N
from .constants import EPS0, MU0


class InterpolationType(enum.IntEnum):
    """InterpolationType (src/fdtd/engine_interface.rs:10-20)."""

    NoInterpolation = N.INTERP_NONE
    NodeInterpolate = N.INTERP_NODE
    CellInterpolate = N.INTERP_CELL


class _GridDesc:
    """The grid's mesh lines as an oems_sample_desc (kept alive with it)."""

    def __init__(self, grid, dims):
        self.lines = [np.ascontiguousarray(v, dtype=np.float64) for v in (grid.x_lines, grid.y_lines, grid.z_lines)]
        for ax, v in enumerate(self.lines):
            if max(len(v), 2) - 1 != dims[ax]:
                raise N.ConfigError("the grid's mesh lines do not match the engine's cells")
        self.desc = N.SampleDescC()
        for ax, v in enumerate(self.lines):
            self.desc.lines[ax] = v.ctypes.data_as(ctypes.POINTER(N.c_f64))
            self.desc.nlines[ax] = len(v)
        self.desc.unit = float(grid.unit)


def _positions(pos) -> np.ndarray:
    p = np.ascontiguousarray(pos, dtype=np.float64)
    if p.ndim == 1:
        p = p.reshape(1, 3)
    if p.ndim != 2 or p.shape[1] != 3:
        raise N.InvalidArgumentError("positions must have shape (n, 3)")
    return p


class EngineInterface:
    """EngineInterface::new(e, h, grid, dt) (:49-67), over `engine`'s fields."""

    def __init__(self, engine, grid, dt: Optional[float] = None):
        self._engine = engine
        self._grid = grid
        self._g = _GridDesc(grid, tuple(engine.dims))
        self._dt = float(engine.dt if dt is None else dt)
        self._timestep = 0
        self._time = 0.0
        self._interp = InterpolationType.NoInterpolation
        self._eps: Optional[np.ndarray] = None
        self._mu: Optional[np.ndarray] = None

    # ---- builder and accessors (:69-111) ----
    def _material(self, m) -> np.ndarray:
        a = np.ascontiguousarray(m, dtype=np.float32)
        if a.shape != (3,) + tuple(self._engine.dims):
            raise N.InvalidArgumentError("material must have shape (3, nx, ny, nz)")
        return a

    def with_epsilon(self, eps) -> "EngineInterface":
        """D = eps * E with these per-cell values (3, nx, ny, nz)."""
        self._eps = self._material(eps)
        return self

    def with_mu(self, mu) -> "EngineInterface":
        """B = mu * H with these per-cell values (3, nx, ny, nz)."""
        self._mu = self._material(mu)
        return self

    def with_interpolation(self, interp: InterpolationType) -> "EngineInterface":
        self._interp = InterpolationType(interp)
        return self

    @property
    def op_eps(self) -> Optional[np.ndarray]:
        return self._eps

    @property
    def op_mu(self) -> Optional[np.ndarray]:
        return self._mu

    def set_time(self, timestep: int, time: float) -> None:
        self._timestep = int(timestep)
        self._time = float(time)

    def timestep(self) -> int:
        return self._timestep

    def time(self) -> float:
        return self._time

    def dt(self) -> float:
        return self._dt

    def dims(self) -> Tuple[int, int, int]:
        return tuple(self._engine.dims)

    def grid(self):
        return self._grid

    # ---- batched reads ----
    def sample(self, quantity: int, positions, interpolation: Optional[int] = None,
               cells: bool = False) -> Tuple[np.ndarray, np.ndarray]:
        """(values (n, 3) f64, snapped cells (n, 3)) of E, H or curl H
        (N.SAMPLE_*) at n positions in metres, or at n cells when `cells`."""
        if cells:
            q = np.ascontiguousarray(positions, dtype=np.uint64).reshape(-1, 3)
        else:
            q = _positions(positions)
        n = q.shape[0]
        vals = np.empty((n, 3), dtype=np.float64)
        snapped = np.empty((n, 3), dtype=np.uint64)
        d = N.SampleDescC.from_buffer_copy(self._g.desc)  # per call: interfaces may be shared by threads
        d.quantity = int(quantity)
        d.interpolation = int(self._interp if interpolation is None else interpolation)
        qp = q.ctypes.data_as(ctypes.c_void_p)
        N.check(N.lib().oems_engine_sample(self._engine.handle, ctypes.byref(d), None if cells else qp,
                                           qp if cells else None, n, vals.ctypes.data_as(ctypes.c_void_p),
                                           snapped.ctypes.data_as(ctypes.c_void_p)))
        return vals, snapped

    def e_fields(self, positions) -> np.ndarray:
        return self.sample(N.SAMPLE_E, positions)[0]

    def h_fields(self, positions) -> np.ndarray:
        return self.sample(N.SAMPLE_H, positions)[0]

    def _scaled(self, quantity, mat, vac, positions) -> np.ndarray:
        v, c = self.sample(quantity, positions)
        if mat is None:
            return v * vac
        i, j, k = (c[:, a].astype(np.int64) for a in range(3))
        return v * np.stack([mat[a][i, j, k].astype(np.float64) for a in range(3)], axis=1)

    def d_fields(self, positions) -> np.ndarray:
        return self._scaled(N.SAMPLE_E, self._eps, EPS0, positions)

    def b_fields(self, positions) -> np.ndarray:
        return self._scaled(N.SAMPLE_H, self._mu, MU0, positions)

    def rot_h_fields(self, positions) -> np.ndarray:
        return self.sample(N.SAMPLE_CURL_H, positions)[0]

    # ---- the reference's single-point reads (:113-206) ----
    def get_e_field_raw(self, i: int, j: int, k: int) -> list:
        return self.sample(N.SAMPLE_E, [[i, j, k]], cells=True)[0][0].tolist()

    def get_h_field_raw(self, i: int, j: int, k: int) -> list:
        return self.sample(N.SAMPLE_H, [[i, j, k]], cells=True)[0][0].tolist()

    def get_e_field(self, pos: Sequence[float]) -> list:
        return self.e_fields(pos)[0].tolist()

    def get_h_field(self, pos: Sequence[float]) -> list:
        return self.h_fields(pos)[0].tolist()

    def get_j_field(self, pos: Sequence[float]) -> list:
        """curl H at the snapped cell (:157-163)."""
        return self.rot_h_fields(pos)[0].tolist()

    def get_d_field(self, pos: Sequence[float]) -> list:
        return self.d_fields(pos)[0].tolist()

    def get_b_field(self, pos: Sequence[float]) -> list:
        return self.b_fields(pos)[0].tolist()

    def get_rot_h_field(self, pos: Sequence[float]) -> list:
        return self.rot_h_fields(pos)[0].tolist()

    # ---- integrals and energies (:208-324) ----
    def _integral(self, kind, start, stop, normal) -> float:
        out = N.c_f64()
        N.check(N.lib().oems_engine_integral(self._engine.handle, ctypes.byref(self._g.desc), kind,
                                             (N.c_f64 * 3)(*map(float, start)), (N.c_f64 * 3)(*map(float, stop)),
                                             int(normal), ctypes.byref(out)))
        return out.value

    def calc_voltage_integral(self, start: Sequence[float], stop: Sequence[float]) -> float:
        """V = -sum E . dl along x, then y, then z (:208-247)."""
        return self._integral(0, start, stop, 0)

    def calc_current_integral(self, start: Sequence[float], stop: Sequence[float], normal_dir: int) -> float:
        """I over the face cells of the surface normal to `normal_dir` (:251-305)."""
        if normal_dir < 0:
            raise N.ConfigError("normal direction must be >= 0")
        return self._integral(1, start, stop, normal_dir)

    def calc_fast_energy(self) -> float:
        e, h = self._engine.energy()
        return 0.5 * (EPS0 * e + MU0 * h)

    def calc_e_energy(self) -> float:
        return 0.5 * EPS0 * self._engine.energy()[0]

    def calc_h_energy(self) -> float:
        return 0.5 * MU0 * self._engine.energy()[1]


class _FieldEdit:
    """Context of e_field_mut / h_field_mut: the host copy is written back on exit."""

    def __init__(self, engine, which: int):
        self._engine, self._which = engine, which

    def __enter__(self) -> np.ndarray:
        self._fields = self._engine.read_fields()
        return self._fields[self._which]

    def __exit__(self, exc_type, exc, tb) -> None:
        if exc_type is None:
            self._engine.write_fields(*self._fields)


class EngineInterfaceMut:
    """EngineInterfaceMut (:508-595): writes into `engine`'s fields."""

    def __init__(self, engine, grid, dt: Optional[float] = None):
        self._engine = engine
        self._grid = grid
        self._dt = float(engine.dt if dt is None else dt)
        self.timestep = 0
        self.time = 0.0

    def _set(self, field: int, cells, values, add: bool) -> None:
        c = np.ascontiguousarray(cells, dtype=np.uint64).reshape(-1, 3)
        v = np.ascontiguousarray(values, dtype=np.float32).reshape(-1, 3)
        if c.shape[0] != v.shape[0]:
            raise N.InvalidArgumentError("one value triple per cell")
        N.check(N.lib().oems_engine_set_cells(self._engine.handle, field, c.ctypes.data_as(ctypes.c_void_p),
                                              v.ctypes.data_as(ctypes.c_void_p), c.shape[0], int(add)))

    def set_e_field(self, i: int, j: int, k: int, value: Sequence[float]) -> None:
        self._set(0, [[i, j, k]], [value], False)

    def set_h_field(self, i: int, j: int, k: int, value: Sequence[float]) -> None:
        self._set(1, [[i, j, k]], [value], False)

    def add_e_field(self, i: int, j: int, k: int, value: Sequence[float]) -> None:
        self._set(0, [[i, j, k]], [value], True)

    def set_e_fields(self, cells, values) -> None:
        """Batched set_e_field, applied in list order."""
        self._set(0, cells, values, False)

    def set_h_fields(self, cells, values) -> None:
        self._set(1, cells, values, False)

    def add_e_fields(self, cells, values) -> None:
        self._set(0, cells, values, True)

    def e_field(self) -> np.ndarray:
        """A host copy of E, (3, nx, ny, nz)."""
        return self._engine.read_fields()[0]

    def h_field(self) -> np.ndarray:
        return self._engine.read_fields()[1]

    def e_field_mut(self) -> _FieldEdit:
        """`with iface.e_field_mut() as e:` edits E on the host, written back on exit."""
        return _FieldEdit(self._engine, 0)

    def h_field_mut(self) -> _FieldEdit:
        return _FieldEdit(self._engine, 1)

    def grid(self):
        return self._grid

    def dt(self) -> float:
        return self._dt

    def set_time(self, timestep: int, time: float) -> None:
        self.timestep = int(timestep)
        self.time = float(time)
