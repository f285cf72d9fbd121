"""openems_b200 -- B200-native Yee FDTD engine with the engine surface of the
Rust openEMS rewrite (Simulation / Operator / EngineImpl).

The compute path is hand-written sm_100a CUDA in liboems_b200.so, reached
through the C ABI in include/oems.h; this package is a thin Python mirror of
the reference's API over that library.  There is no CPU fallback.
"""
from ._native import (OpenEMSError, ConfigError, IoError, GridError, MaterialError,  # noqa: F401
                      NumericalError, XmlError, CudaError, NoDeviceError, DeviceTimeoutError,
                      InvalidArgumentError, LIB_PATH)
from .constants import C0, EPS0, MU0, Z0  # noqa: F401
from .fdtd import (Grid, BoundaryCondition, BoundaryConditions, CpmlBoundaries, MurAbcConfig, Operator,  # noqa: F401
                   Excitation, ExcitationType, ScheduledExcitation, TerminationConfig,
                   EnergyMonitorConfig, EngineBatch, TerminationReason, EnergySample, BatchResult,
                   EngineType, Engine, EndCondition, SimulationStats, Simulation, SimulationState, TimestepInfo,
                   ProbeTerms, voltage_probe, current_probe, voltage_integral, current_integral,
                   port_probe, LumpedPort, DrudeMaterial, LorentzMaterial, DebyeMaterial,
                   RlcType, RlcElement, Nf2ffBox, Nf2ffResults, nf2ff_surface, PmlBoundaries,
                   PropagationDirection, Polarization, TfsfConfig, Pack, compress_coefficients,
                   waveguide_te10)
from .engine_interface import EngineInterface, EngineInterfaceMut, InterpolationType  # noqa: F401
from .processing import (Processing, VoltageProbe, CurrentProbe, FieldProbe,  # noqa: F401
                         FrequencyDomainFieldDump, TimeDomainFieldDump, FdDumpType)

__all__ = [n for n in dir() if not n.startswith("_")]
