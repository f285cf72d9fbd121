"""ctypes binding of liboems_b200.so (include/oems.h, include/oems_host.h).

The library is required: there is no CPU fallback.  Importing this module
without the built library raises immediately with the build command.
"""
from __future__ import annotations

import ctypes
import os

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "liboems_b200.so")

c_u64, c_i64, c_i32, c_u32, c_f64, c_f32 = (ctypes.c_uint64, ctypes.c_int64, ctypes.c_int32,
                                              ctypes.c_uint32, ctypes.c_double, ctypes.c_float)
P = ctypes.c_void_p
PF = ctypes.POINTER(c_f32)

# status codes (include/oems.h)
OK, ERR_CONFIG, ERR_IO, ERR_GRID, ERR_MATERIAL, ERR_NUMERICAL, ERR_XML, ERR_CUDA, \
    ERR_NO_DEVICE, ERR_TIMEOUT, ERR_INVALID_ARGUMENT = range(11)

ENGINE_COMPRESSED = 0x1
ENGINE_NO_AUTOTUNE = 0x2
ENGINE_NO_GRAPHS = 0x4
ENGINE_REGISTER_KERNELS = 0x10
ENGINE_STAGED_KERNELS = 0x20
ENGINE_SPLIT_KERNELS = 0x40
ENGINE_FIELDS_F16 = 0x80
ENGINE_FIELDS_BF16 = 0x100
ENGINE_ZSPLIT_KERNELS = 0x200
ENGINE_PIPE_KERNELS = 0x400
H_STORAGE_SCALE = 512.0
STORAGE_FLAGS = {"f32": 0, "f16": ENGINE_FIELDS_F16, "bf16": ENGINE_FIELDS_BF16}


class OpenEMSError(Exception):
    """crate::Error (src/lib.rs:60-85); `status` is the C status code."""

    status = -1

    def __init__(self, msg, status=None):
        super().__init__(msg)
        if status is not None:
            self.status = status


class ConfigError(OpenEMSError):
    status = ERR_CONFIG


class IoError(OpenEMSError):
    status = ERR_IO


class GridError(OpenEMSError):
    status = ERR_GRID


class MaterialError(OpenEMSError):
    status = ERR_MATERIAL


class NumericalError(OpenEMSError):
    status = ERR_NUMERICAL


class XmlError(OpenEMSError):
    status = ERR_XML


class CudaError(OpenEMSError):
    status = ERR_CUDA


class NoDeviceError(OpenEMSError):
    status = ERR_NO_DEVICE


class DeviceTimeoutError(OpenEMSError):
    status = ERR_TIMEOUT


class InvalidArgumentError(OpenEMSError):
    status = ERR_INVALID_ARGUMENT


_ERRORS = {c.status: c for c in (ConfigError, IoError, GridError, MaterialError, NumericalError,
                                 XmlError, CudaError, NoDeviceError, DeviceTimeoutError,
                                 InvalidArgumentError)}


class OperatorDesc(ctypes.Structure):
    _fields_ = [("nx", c_u64), ("ny", c_u64), ("nz", c_u64), ("dt", c_f64), ("delta", c_f64 * 3),
                ("ca", PF * 3), ("cb", PF * 3), ("da", PF * 3), ("db", PF * 3),
                ("device", c_i32), ("flags", c_u32)]


class ScheduledExcitationC(ctypes.Structure):
    _fields_ = [("position", c_u64 * 3), ("direction", c_u32), ("soft_source", c_u32),
                ("samples", PF), ("num_samples", c_u64)]


class BatchC(ctypes.Structure):
    _fields_ = [("num_steps", c_u64), ("excitations", ctypes.POINTER(ScheduledExcitationC)),
                ("num_excitations", c_u32), ("has_energy_decay_db", c_i32),
                ("energy_decay_db", c_f64), ("check_interval", c_u64), ("sample_interval", c_u64),
                ("track_peak", c_i32), ("reserved0", c_i32), ("initial_peak_energy", c_f64)]


class EnergySampleC(ctypes.Structure):
    _fields_ = [("timestep", c_u64), ("e_energy", c_f64), ("h_energy", c_f64),
                ("total_energy", c_f64)]


class BatchResultC(ctypes.Structure):
    _fields_ = [("timesteps_executed", c_u64), ("termination_reason", c_i32),
                ("reserved0", c_i32), ("final_decay_db", c_f64),
                ("energy_samples", ctypes.POINTER(EnergySampleC)), ("energy_capacity", c_u64),
                ("num_energy_samples", c_u64), ("peak_energy", c_f64),
                ("elapsed_seconds", c_f64)]


class CpmlDescC(ctypes.Structure):
    _fields_ = [("layers", c_i32 * 6), ("grading_order", c_f64), ("reflection_coeff", c_f64),
                ("alpha_max", c_f64), ("kappa_max", c_f64)]


class ProbeTermC(ctypes.Structure):
    _fields_ = [("component", c_i32), ("reserved0", c_i32), ("position", c_u64 * 3),
                ("weight", c_f64)]


PROBE_SUM_F32 = 0
PROBE_SUM_F64 = 1

SAMPLE_E, SAMPLE_H, SAMPLE_CURL_H = 0, 1, 2
INTERP_NONE, INTERP_NODE, INTERP_CELL = 0, 1, 2


class SampleDescC(ctypes.Structure):
    _fields_ = [("quantity", c_i32), ("interpolation", c_i32), ("lines", ctypes.POINTER(c_f64) * 3),
                ("nlines", c_u64 * 3), ("unit", c_f64)]


class MurDescC(ctypes.Structure):
    _fields_ = [("enabled", c_i32 * 6), ("order", c_i32), ("reserved0", c_i32),
                ("phase_velocity", c_f64)]


class UpmlDescC(ctypes.Structure):
    _fields_ = [("layers", c_u32 * 6), ("grading_order", c_f64), ("reflection_coeff", c_f64), ("kind", c_i32),
                ("reserved0", c_i32)]


class DispersiveDescC(ctypes.Structure):
    _fields_ = [("kind", c_i32), ("reserved0", c_i32), ("params", c_f64 * 3), ("eps_inf", c_f64)]


class LumpedRlcDescC(ctypes.Structure):
    _fields_ = [("position", c_u64 * 3), ("direction", c_u32), ("type", c_i32),
                ("resistance", c_f64), ("inductance", c_f64), ("capacitance", c_f64)]


class FieldDftDescC(ctypes.Structure):
    _fields_ = [("region", c_u64 * 6), ("sub_sample", c_u32 * 3), ("components", c_u32),
                ("interval", c_u32), ("reserved0", c_u32)]


class Nf2ffBoxDescC(ctypes.Structure):
    _fields_ = [("start", c_u64 * 3), ("stop", c_u64 * 3), ("directions", c_i32 * 6),
                ("interval", c_u32), ("reserved0", c_u32)]


class Nf2ffRequestC(ctypes.Structure):
    _fields_ = [("theta", ctypes.POINTER(c_f64)), ("ntheta", c_u64),
                ("phi", ctypes.POINTER(c_f64)), ("nphi", c_u64), ("radius", c_f64),
                ("center", c_f64 * 3), ("lines", ctypes.POINTER(c_f64) * 3)]


class Nf2ffResultC(ctypes.Structure):
    _fields_ = [("e_theta", ctypes.POINTER(c_f64)), ("e_phi", ctypes.POINTER(c_f64)),
                ("p_rad", ctypes.POINTER(c_f64)), ("prad", c_f64), ("dmax", c_f64)]


class ExcitationC(ctypes.Structure):
    _fields_ = [("kind", c_i32), ("direction", c_u32), ("position", c_u64 * 3),
                ("params", c_f64 * 3), ("amplitude", c_f64), ("soft_source", c_i32),
                ("reserved0", c_i32)]


class SimulationStatsC(ctypes.Structure):
    _fields_ = [("timesteps", c_u64), ("sim_time", c_f64), ("wall_time", c_f64),
                ("peak_energy", c_f64), ("final_energy", c_f64),
                ("speed_mcells_per_sec", c_f64)]


class SweepInstanceC(ctypes.Structure):
    _fields_ = [("op", P), ("cpml", CpmlDescC), ("port_position", c_u64 * 3),
                ("port_direction", c_i32), ("reserved0", c_i32), ("port_resistance", c_f64),
                ("port_eps_r", c_f64), ("port_sigma", c_f64), ("waveform", ExcitationC),
                ("energy_decay_db", c_f64), ("max_timesteps", c_u64)]


class TfsfDescC(ctypes.Structure):
    _fields_ = [("direction", c_i32), ("polarization", c_i32), ("frequency", c_f64), ("amplitude", c_f64),
                ("boundary_layer", c_u64), ("phase_velocity", c_f64), ("kind", c_i32), ("reserved0", c_i32)]


class StateSectionC(ctypes.Structure):
    _fields_ = [("kind", c_u32), ("variant", c_u32), ("bytes", c_u64)]


class CylDescC(ctypes.Structure):
    _fields_ = [("n_rho", c_u64), ("n_alpha", c_u64), ("n_z", c_u64), ("closed_alpha", c_i32),
                ("r0_included", c_i32), ("dt", c_f64), ("vi", PF * 3), ("iv", PF * 3), ("device", c_i32),
                ("reserved0", c_i32)]


class SweepResultC(ctypes.Structure):
    _fields_ = [("timesteps", c_u64), ("termination_reason", c_i32), ("status", c_i32),
                ("final_decay_db", c_f64), ("device_seconds", c_f64), ("cells", c_f64),
                ("setup_seconds", c_f64), ("host_seconds", c_f64), ("paused", c_i32), ("reserved0", c_i32)]


# name -> (restype, argtypes); every symbol the headers declare
SIGNATURES = {
    # include/oems.h
    "oems_engine_create": (c_i32, [ctypes.POINTER(OperatorDesc), ctypes.POINTER(P)]),
    "oems_engine_destroy": (None, [P]),
    "oems_release_cached_memory": (c_i32, [c_i32]),
    "oems_engine_add_tfsf": (c_i32, [P, ctypes.POINTER(TfsfDescC)]),
    "oems_engine_state_sections": (c_i32, [P, ctypes.POINTER(StateSectionC), c_u64, ctypes.POINTER(c_u64)]),
    "oems_engine_read_state": (c_i32, [P, c_u64, ctypes.c_void_p, c_u64]),
    "oems_engine_write_state": (c_i32, [P, c_u64, c_u32, ctypes.c_char_p, c_u64]),
    "oems_engine_get_state_counters": (c_i32, [P, ctypes.POINTER(c_u64), ctypes.POINTER(c_u64)]),
    "oems_engine_set_state_counters": (c_i32, [P, c_u64, c_u64]),
    "oems_cyl_create": (c_i32, [ctypes.POINTER(CylDescC), ctypes.POINTER(P)]),
    "oems_cyl_destroy": (None, [P]),
    "oems_cyl_step": (c_i32, [P, c_u64]),
    "oems_cyl_read_fields": (c_i32, [P, PF * 3, PF * 3]),
    "oems_cyl_write_fields": (c_i32, [P, PF * 3, PF * 3]),
    "oems_cyl_reset": (c_i32, [P]),
    "oems_cyl_time": (c_i32, [P, ctypes.POINTER(c_u64), ctypes.POINTER(c_f64)]),
    "oems_cyl_last_step_ms": (c_i32, [P, ctypes.POINTER(c_f32)]),
    "oems_engine_run_batch": (c_i32, [P, ctypes.POINTER(BatchC), ctypes.POINTER(BatchResultC)]),
    "oems_engine_current_timestep": (c_i32, [P, ctypes.POINTER(c_u64)]),
    "oems_engine_read_fields": (c_i32, [P, PF * 3, PF * 3]),
    "oems_engine_write_fields": (c_i32, [P, PF * 3, PF * 3]),
    "oems_engine_reset": (c_i32, [P]),
    "oems_engine_add_cpml": (c_i32, [P, ctypes.POINTER(CpmlDescC)]),
    "oems_engine_add_mur": (c_i32, [P, ctypes.POINTER(MurDescC)]),
    "oems_engine_add_upml": (c_i32, [P, ctypes.POINTER(UpmlDescC)]),
    "oems_engine_add_dispersive": (c_i32, [P, ctypes.POINTER(DispersiveDescC), P, c_u64]),
    "oems_engine_add_lumped_rlc": (c_i32, [P, ctypes.POINTER(LumpedRlcDescC), c_u64]),
    "oems_engine_add_field_dft": (c_i32, [P, ctypes.POINTER(FieldDftDescC), ctypes.POINTER(c_f64), c_u32,
                                          ctypes.POINTER(c_i32)]),
    "oems_engine_read_field_dft": (c_i32, [P, c_i32, c_u32, c_u32, ctypes.POINTER(c_f64), c_u64]),
    "oems_engine_add_nf2ff_box": (c_i32, [P, ctypes.POINTER(Nf2ffBoxDescC), ctypes.POINTER(c_f64), c_u32,
                                          ctypes.POINTER(c_i32)]),
    "oems_engine_read_nf2ff_face": (c_i32, [P, c_i32, c_u32, c_u32, ctypes.POINTER(c_f64), c_u64,
                                            ctypes.POINTER(c_u64)]),
    "oems_engine_nf2ff": (c_i32, [P, c_i32, c_u32, ctypes.POINTER(Nf2ffRequestC),
                                  ctypes.POINTER(Nf2ffResultC)]),
    "oems_nf2ff_surface": (c_i32, [c_i32, ctypes.POINTER(c_f64), c_u64, c_f64, ctypes.POINTER(Nf2ffRequestC),
                                   ctypes.POINTER(Nf2ffResultC)]),
    "oems_engine_add_point_probe": (c_i32, [P, c_i32, c_u64 * 3, ctypes.POINTER(c_i32)]),
    "oems_engine_read_probe_traces": (c_i32, [P, ctypes.POINTER(c_f64), c_u64, ctypes.POINTER(c_u64)]),
    "oems_engine_add_probe": (c_i32, [P, ctypes.POINTER(ProbeTermC), c_u64, c_i32, ctypes.POINTER(c_i32)]),
    "oems_engine_add_probe_dft": (c_i32, [P, c_i32, ctypes.POINTER(c_f64), c_u64, ctypes.POINTER(c_i32)]),
    "oems_engine_read_probe_dft": (c_i32, [P, c_i32, ctypes.POINTER(c_f64)]),
    "oems_engine_energy": (c_i32, [P, ctypes.POINTER(c_f64), ctypes.POINTER(c_f64)]),
    "oems_engine_sample": (c_i32, [P, ctypes.POINTER(SampleDescC), P, P, c_u64, P, P]),
    "oems_engine_integral": (c_i32, [P, ctypes.POINTER(SampleDescC), c_i32, c_f64 * 3, c_f64 * 3, c_i32,
                                     ctypes.POINTER(c_f64)]),
    "oems_engine_eval_terms": (c_i32, [P, ctypes.POINTER(ProbeTermC), c_u64, c_i32, ctypes.POINTER(c_f64)]),
    "oems_engine_set_cells": (c_i32, [P, c_i32, P, P, c_u64, c_i32]),
    "oems_status_string": (ctypes.c_char_p, [c_i32]),
    "oems_last_error_message": (ctypes.c_char_p, []),
    "oems_abi_version": (c_i32, []),
    "oems_engine_last_batch_stats": (c_i32, [P, ctypes.POINTER(c_u64), ctypes.POINTER(c_f64)]),
    "oems_field_energy_noalloc": (c_i32, [ctypes.c_void_p * 6, c_u64, P, P]),
    "oems_engine_set_kernel_profiling": (c_i32, [P, c_i32]),
    "oems_engine_launch_info": (c_i32, [P] + [ctypes.POINTER(c_i32)] * 6),
    "oems_engine_tune_report": (c_i32, [P, P, c_u64, ctypes.POINTER(c_u64)]),
    "oems_engine_kernel_profile": (c_i32, [P, ctypes.POINTER(c_f64), ctypes.POINTER(c_u64),
                                           ctypes.POINTER(c_f64), ctypes.POINTER(c_u64)]),
    # include/oems_host.h
    "oems_operator_create": (c_i32, [P, c_u64, P, c_u64, P, c_u64, c_f64, ctypes.POINTER(P)]),
    "oems_compress_coefficients": (c_i32, [ctypes.POINTER(ctypes.c_void_p), c_u64, P, P, c_u32, ctypes.POINTER(c_u32)]),
    "oems_operator_create_uniform": (c_i32, [c_u64, c_u64, c_u64, c_f64, ctypes.POINTER(P)]),
    "oems_operator_destroy": (None, [P]),
    "oems_operator_set_material": (c_i32, [P, c_f64, c_f64, c_f64, c_f64, c_u64 * 6]),
    "oems_operator_set_pec": (c_i32, [P, c_u64 * 6]),
    "oems_operator_info": (c_i32, [P, c_u64 * 3, ctypes.POINTER(c_f64), c_f64 * 3]),
    "oems_operator_coefficients": (c_i32, [P, PF * 12]),
    "oems_operator_clone": (c_i32, [P, ctypes.POINTER(P)]),
    "oems_operator_set_material_cells": (c_i32, [P, c_f64, c_f64, c_f64, c_f64, P, c_u64]),
    "oems_sweep_create": (c_i32, [c_i32, c_u32, c_u32, ctypes.POINTER(c_f64), c_u64, ctypes.POINTER(P)]),
    "oems_sweep_destroy": (None, [P]),
    "oems_sweep_add": (c_i32, [P, ctypes.POINTER(SweepInstanceC), ctypes.POINTER(c_i32)]),
    "oems_sweep_run": (c_i32, [P, c_u64]),
    "oems_sweep_get_result": (c_i32, [P, c_i32, ctypes.POINTER(SweepResultC), ctypes.POINTER(c_f64),
                                      ctypes.POINTER(c_f64), ctypes.POINTER(c_f64)]),
    "oems_sweep_stats": (c_i32, [P, ctypes.POINTER(c_f64), ctypes.POINTER(c_f64)]),
    "oems_sweep_set_trace_steps": (c_i32, [P, c_u64]),
    "oems_sweep_set_packed": (c_i32, [P, c_i32]),
    "oems_pack_create": (c_i32, [ctypes.POINTER(P), c_u64, ctypes.POINTER(P)]),
    "oems_pack_destroy": (None, [P]),
    "oems_pack_run_batch": (c_i32, [P, ctypes.POINTER(ctypes.c_void_p), P, ctypes.POINTER(c_i32)]),
    "oems_pack_set_shape": (c_i32, [P, c_i32, c_i32, c_i32]),
    "oems_pack_shape": (c_i32, [P, ctypes.POINTER(c_i32), ctypes.POINTER(c_i32), ctypes.POINTER(c_i32)]),
    "oems_sweep_run_until": (c_i32, [P, c_u64, c_u64]),
    "oems_sweep_finish": (c_i32, [P, c_i32]),
    "oems_sweep_advance": (c_i32, [P, c_i32, c_u64, c_u64]),
    "oems_tc_gemm_bf16": (c_i32, [P, c_i32, P, c_i32, P, c_i32, c_i32, c_i32, c_i32, ctypes.c_float, P, P]),
    "oems_tc_check": (c_i32, [P]),
    "oems_tc_wait_probe": (c_i32, [P]),
    "oems_pk_f32_to_bf16": (c_i32, [P, P, c_i64, P]),
    "oems_pk_transpose_bf16": (c_i32, [P, c_i32, P, c_i32, c_i32, c_i32, P]),
    "oems_pk_im2col": (c_i32, [P, P, c_i32, c_i32, c_i32, c_i32, c_i32, c_i32, P]),
    "oems_pk_col2im": (c_i32, [P, c_i32, P, c_i32, c_i32, c_i32, c_i32, c_i32, P]),
    "oems_pk_im2col_causal": (c_i32, [P, P, c_i32, c_i32, c_i32, c_i32, c_i32, c_i32, P]),
    "oems_pk_col2im_causal": (c_i32, [P, c_i32, P, c_i32, c_i32, c_i32, c_i32, c_i32, P]),
    "oems_pk_relu": (c_i32, [P, P, c_i64, c_i32, c_i32, P]),
    "oems_pk_relu_bwd": (c_i32, [P, P, c_i64, P]),
    "oems_pk_colsum": (c_i32, [P, c_i64, c_i32, P, P]),
    "oems_pk_mse": (c_i32, [P, P, P, P, c_i64, c_i32, P, c_i32, P]),
    "oems_pk_adam": (c_i32, [P, P, P, P, P, c_i64, ctypes.c_float, ctypes.c_float, ctypes.c_float,
                             ctypes.c_float, ctypes.c_float, c_i32, P]),
    "oems_sweep_get_trace": (c_i32, [P, c_i32, ctypes.POINTER(c_f64), c_u64, ctypes.POINTER(c_u64)]),
    "oems_operator_set_lumped": (c_i32, [P, c_u64 * 3, c_i32, c_f64, c_f64, c_f64, c_f64,
                                         ctypes.POINTER(c_f64)]),
    "oems_operator_engine_desc": (c_i32, [P, c_i32, c_u32, ctypes.POINTER(OperatorDesc)]),
    "oems_excitation_gaussian": (c_i32, [c_f64, c_f64, c_u32, c_u64 * 3, ctypes.POINTER(ExcitationC)]),
    "oems_excitation_gaussian_modulated": (c_i32, [c_f64, c_f64, c_u32, c_u64 * 3,
                                                   ctypes.POINTER(ExcitationC)]),
    "oems_excitation_sinusoidal": (c_i32, [c_f64, c_u32, c_u64 * 3, ctypes.POINTER(ExcitationC)]),
    "oems_excitation_dirac": (c_i32, [c_f64, c_u32, c_u64 * 3, ctypes.POINTER(ExcitationC)]),
    "oems_excitation_evaluate": (c_f64, [ctypes.POINTER(ExcitationC), c_f64]),
    "oems_excitation_sample": (c_i32, [ctypes.POINTER(ExcitationC), c_u64, c_u64, c_f64, PF]),
    "oems_probe_voltage_terms": (c_i32, [c_u64 * 3, c_u64 * 3, c_i32, ctypes.POINTER(ProbeTermC), c_u64,
                                         ctypes.POINTER(c_u64)]),
    "oems_probe_current_terms": (c_i32, [c_u64 * 3, c_u64 * 3, c_i32, ctypes.POINTER(ProbeTermC), c_u64,
                                         ctypes.POINTER(c_u64)]),
    "oems_probe_voltage_integral_terms": (c_i32, [P, c_u64 * 3, c_u64 * 3, ctypes.POINTER(ProbeTermC), c_u64,
                                                  ctypes.POINTER(c_u64)]),
    "oems_probe_current_integral_terms": (c_i32, [P, c_u64 * 3, c_u64 * 3, c_i32, ctypes.POINTER(ProbeTermC),
                                                  c_u64, ctypes.POINTER(c_u64)]),
    "oems_probe_port_terms": (c_i32, [P, c_u64 * 3, c_i32, c_i32, ctypes.POINTER(ProbeTermC), c_u64,
                                      ctypes.POINTER(c_u64)]),
    "oems_simulation_create": (c_i32, [P, c_i32, c_u32, ctypes.POINTER(P)]),
    "oems_simulation_destroy": (None, [P]),
    "oems_simulation_add_excitation": (c_i32, [P, ctypes.POINTER(ExcitationC)]),
    "oems_simulation_set_end_condition": (c_i32, [P, c_i32, c_f64]),
    "oems_simulation_set_batch_size": (c_i32, [P, c_u64]),
    "oems_simulation_set_cpml": (c_i32, [P, ctypes.POINTER(CpmlDescC)]),
    "oems_simulation_setup": (c_i32, [P]),
    "oems_simulation_run": (c_i32, [P, ctypes.POINTER(SimulationStatsC)]),
    "oems_simulation_engine": (P, [P]),
}

_lib = None


def lib() -> ctypes.CDLL:
    """The loaded native library (raises if it has not been built)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(
                f"{LIB_PATH} is missing: build it with `python openems_b200/build.py` "
                "(the engine has no CPU fallback)")
        L = ctypes.CDLL(LIB_PATH)
        for name, (res, args) in SIGNATURES.items():
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        _lib = L
    return _lib


def check(status: int) -> None:
    """Raise the OpenEMSError subclass matching a non-zero status."""
    if status == OK:
        return
    msg = lib().oems_last_error_message().decode(errors="replace")
    name = lib().oems_status_string(status).decode(errors="replace")
    cls = _ERRORS.get(status, OpenEMSError)
    raise cls(f"{name}: {msg}" if msg else name, status)


def fptr(a) -> "ctypes._Pointer":
    """float* to the data of a C-contiguous float32 numpy array."""
    return a.ctypes.data_as(PF)
