/*
 * oems.h -- C ABI of the B200 FDTD engine (liboems_b200.so).
 *
 * This is the drop-in boundary for the Rust openEMS rewrite's engine
 * interface.  Each entry point names the reference item it replaces
 * (paths relative to the reference project):
 *
 *   EngineImpl::new(&Operator)          src/fdtd/engine_impl.rs:32   -> oems_engine_create
 *   EngineImpl::run_batch(EngineBatch)  src/fdtd/engine_impl.rs:48   -> oems_engine_run_batch
 *   EngineImpl::current_timestep()      src/fdtd/engine_impl.rs:53   -> oems_engine_current_timestep
 *   EngineImpl::read_fields()           src/fdtd/engine_impl.rs:59   -> oems_engine_read_fields
 *   EngineImpl::write_fields()          src/fdtd/engine_impl.rs:65   -> oems_engine_write_fields
 *   EngineImpl::reset()                 src/fdtd/engine_impl.rs:70   -> oems_engine_reset
 *   drop(Engine)                        src/fdtd/new_engine.rs:20    -> oems_engine_destroy
 *   crate::Error variants               src/lib.rs:60-85             -> oems_status
 *
 * Extensions are attached to the engine once and stay resident on the GPU
 * (the reference passes them per batch as `EngineBatch::extensions`,
 * src/fdtd/batch.rs:25, and calls per-cell hooks; here they are fused into the
 * update kernels):
 *
 *   Cpml::new           src/extensions/cpml.rs:235     -> oems_engine_add_cpml
 *   MurAbc::new         src/extensions/mur_abc.rs:175  -> oems_engine_add_mur
 *   FieldProbe::sample  src/processing/probes.rs:289   -> oems_engine_add_point_probe
 *
 * Conventions
 *   - Arrays are float32, one array per component, z fastest:
 *     idx = (i*ny + j)*nz + k  (src/arrays/mod.rs:61-64).
 *   - Host pointers passed in are borrowed for the duration of the call only.
 *   - No call throws or aborts.  Every failure returns a status;
 *     oems_last_error_message() gives the detail for the calling thread.
 *   - A handle is thread-compatible, not thread-safe (the reference trait is
 *     Send but not Sync): one thread drives a handle at a time.  Each handle
 *     owns one CUDA stream on its device.
 */
#ifndef OEMS_H
#define OEMS_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define OEMS_ABI_VERSION 1

#if defined(__GNUC__)
#define OEMS_API __attribute__((visibility("default")))
#else
#define OEMS_API
#endif

/* Status codes.  1..6 map one to one onto crate::Error (src/lib.rs:60-85). */
typedef enum oems_status {
  OEMS_OK = 0,
  OEMS_ERR_CONFIG = 1,    /* Error::Config    */
  OEMS_ERR_IO = 2,        /* Error::Io        */
  OEMS_ERR_GRID = 3,      /* Error::Grid      */
  OEMS_ERR_MATERIAL = 4,  /* Error::Material  */
  OEMS_ERR_NUMERICAL = 5, /* Error::Numerical: a field became NaN or infinite */
  OEMS_ERR_XML = 6,       /* Error::Xml       */
  OEMS_ERR_CUDA = 7,      /* CUDA runtime failure (maps to Error::Numerical on the Rust side) */
  OEMS_ERR_NO_DEVICE = 8, /* no usable CUDA device */
  OEMS_ERR_TIMEOUT = 9,   /* a bounded device-side wait gave up */
  OEMS_ERR_INVALID_ARGUMENT = 10
} oems_status;

typedef struct oems_engine oems_engine;

/* Engine creation flags. */
#define OEMS_ENGINE_COMPRESSED 0x1u /* store a per-cell material id + table of unique
                                       coefficient sets instead of 12 arrays
                                       (replaces CompressedCoefficients,
                                       src/fdtd/compressed.rs:125-192) */
#define OEMS_ENGINE_NO_AUTOTUNE 0x2u /* keep the default launch shape */
#define OEMS_ENGINE_NO_GRAPHS 0x4u   /* launch kernels one by one instead of
                                        replaying captured CUDA graphs */
#define OEMS_ENGINE_REGISTER_KERNELS 0x10u /* only the register-blocked update kernels */
#define OEMS_ENGINE_STAGED_KERNELS 0x20u   /* only the bulk-async (TMA) staged update
                                              kernels, where their stages fit */
#define OEMS_ENGINE_SPLIT_KERNELS 0x40u    /* with CPML: staged kernels on the box
                                              between the x / y slabs, register
                                              kernels on those slabs */
#define OEMS_ENGINE_ZSPLIT_KERNELS 0x200u  /* with CPML: plain register kernels on
                                              the CPML-free box (between the x / y
                                              slabs, float4 chunks clear of the z
                                              slabs), CPML register kernels on
                                              every slab cell */
#define OEMS_ENGINE_PIPE_KERNELS 0x400u    /* only the pipelined register kernels
                                              (each thread's next x-planes copied
                                              into shared memory by cp.async while
                                              it computes), where they apply:
                                              float fields, full coefficients,
                                              nz <= 1024 */
/* Field storage in 2 bytes per value, arithmetic still in float (no
 * counterpart in the reference, whose fields are f32): IEEE half or
 * bfloat16, rounded to nearest on every store.  H is kept multiplied by
 * OEMS_H_STORAGE_SCALE (folded into the coefficients, a power of two, so the
 * float arithmetic is exactly the scaled one) to keep it in half's range;
 * probes, energies and read / write_fields see unscaled values.  Register
 * kernels only; CPML, excitations, probes and their DFTs, energies and the
 * energy-decay end condition are supported, the other extensions are
 * refused with OEMS_ERR_CONFIG. */
#define OEMS_ENGINE_FIELDS_F16 0x80u
#define OEMS_ENGINE_FIELDS_BF16 0x100u
#define OEMS_H_STORAGE_SCALE 512.0f

/* What Operator hands to EngineImpl::new: dimensions, dt, cell sizes and the
 * 12 per-cell coefficient arrays (src/fdtd/operator.rs:21-38, :145-185). */
typedef struct oems_operator_desc {
  uint64_t nx, ny, nz;
  double dt;
  double delta[3];    /* cell size per axis (Grid::cell_size), used by extensions */
  const float* ca[3]; /* E: E = ca*E + cb*curl(H) */
  const float* cb[3];
  const float* da[3]; /* H: H = da*H + db*curl(E) (db carries the minus sign) */
  const float* db[3];
  int32_t device;     /* CUDA device ordinal, -1 = the calling thread's current device */
  uint32_t flags;     /* OEMS_ENGINE_* */
} oems_operator_desc;

/* ScheduledExcitation with a Sampled waveform (src/fdtd/batch.rs:71-100).
 * samples[s] is applied after the E update of batch step s; steps beyond
 * num_samples inject nothing (src/fdtd/basic_engine.rs:319-325). */
typedef struct oems_scheduled_excitation {
  uint64_t position[3];
  uint32_t direction;   /* 0 = x, 1 = y, 2 = z */
  uint32_t soft_source; /* 1: E += v, 0: E = v */
  const float* samples;
  uint64_t num_samples;
} oems_scheduled_excitation;

/* EngineBatch without the extension list (src/fdtd/batch.rs:17-32), with
 * TerminationConfig (:150-170) and EnergyMonitorConfig (:173-193) inlined. */
typedef struct oems_batch {
  uint64_t num_steps;
  const oems_scheduled_excitation* excitations;
  uint32_t num_excitations;
  int32_t has_energy_decay_db;
  double energy_decay_db;
  uint64_t check_interval;   /* 0 disables the termination check */
  uint64_t sample_interval;  /* 0 disables energy sampling */
  int32_t track_peak;
  int32_t reserved0;
  double initial_peak_energy; /* peak carried in from earlier batches; 0 reproduces the
                                 reference, whose peak restarts at 0 every batch
                                 (src/fdtd/basic_engine.rs:62) */
} oems_batch;

/* EnergySample (src/fdtd/batch.rs:197-220): unweighted sums of squares. */
typedef struct oems_energy_sample {
  uint64_t timestep;
  double e_energy;
  double h_energy;
  double total_energy;
} oems_energy_sample;

/* TerminationReason (src/fdtd/batch.rs:52-67). */
#define OEMS_TERMINATION_STEPS_COMPLETED 0
#define OEMS_TERMINATION_ENERGY_DECAY 1
#define OEMS_TERMINATION_EXTENSION_STOP 2

/* BatchResult (src/fdtd/batch.rs:36-48). energy_samples is caller-owned and
 * may be NULL; num_energy_samples reports how many were produced even when
 * that exceeds energy_capacity. */
typedef struct oems_batch_result {
  uint64_t timesteps_executed;
  int32_t termination_reason;
  int32_t reserved0;
  double final_decay_db;
  oems_energy_sample* energy_samples;
  uint64_t energy_capacity;
  uint64_t num_energy_samples;
  double peak_energy;
  double elapsed_seconds;
} oems_batch_result;

/* CpmlBoundaries (src/extensions/cpml.rs:27-51).  layers: xmin xmax ymin ymax
 * zmin zmax, 0 disables a face.  The profile follows cpml.rs:68-177; the field
 * correction is the standard Roden-Gedney recursive convolution (the
 * reference computes psi but never applies it, cpml.rs:344-350). */
typedef struct oems_cpml_desc {
  int32_t layers[6];
  double grading_order;    /* default 3    */
  double reflection_coeff; /* default 1e-6 */
  double alpha_max;        /* default 0    */
  double kappa_max;        /* default 1    */
} oems_cpml_desc;

/* MurAbcConfig (src/extensions/mur_abc.rs:13-28).  enabled: xmin xmax ymin
 * ymax zmin zmax.  order 1 restates the reference (mur_abc.rs:88-324): pre
 * before the E update, post and apply after it, faces applied in order.
 * order 2 is the second-order Mur condition (no counterpart in the
 * reference) on face interiors, first order on the two outermost rows and
 * columns of a face; at a min face its boundary is line 1, the first line the
 * E update writes. */
typedef struct oems_mur_desc {
  int32_t enabled[6];
  int32_t order;
  int32_t reserved0;
  double phase_velocity; /* <= 0: c0 */
} oems_mur_desc;

/* PmlBoundaries (src/extensions/pml.rs:85-101): layers per face (-x +x -y
 * +y -z +z; a face is active when 0 < layers < n), polynomial grading order
 * and target reflection.  kind 0: the reference's coefficients (they grow
 * without bound); kind 1: the uniaxial PML of Taflove & Hagness 7.8 in the
 * reference's flux form -- per-axis conductivities at each component's Yee
 * position (edges and corners graded along every axis whose slab holds
 * them), consistent flux coefficients, and the next axis' conductivity
 * folded into the region cells' main update coefficients (Ca, Cb, Da, Db;
 * PEC cells stay as they are).  Kind 1 needs full coefficient arrays. */
typedef struct oems_upml_desc {
  uint32_t layers[6];
  double grading_order;
  double reflection_coeff;
  int32_t kind;
  int32_t reserved0;
} oems_upml_desc;

/* Dispersive material on a list of cells (src/extensions/dispersive.rs),
 * applied after the E update to all three components of every cell:
 *   kind 0 Drude    params (omega_p, gamma)            :476-535
 *   kind 1 Lorentz  params (omega_0, gamma, delta_eps) :134-196, as the
 *          reference (first order in J; unstable for usual parameters)
 *   kind 2 Debye    params (tau, delta_eps)             :570-630
 *   kind 3 Lorentz, second order: P' = a P + b P_prev + c E_n,
 *          E -= (P' - P) / (eps0 eps_inf), E_n the field before the E
 *          update (no counterpart in the reference)
 *   kind 4 Drude as the same recursion with omega_0 = 0, params (omega_p,
 *          gamma): stable where kind 0 grows (gamma << omega_p)
 * Angular frequencies in rad/s.  eps_inf divides the E correction; 1 gives
 * the reference's coefficients. */
typedef struct oems_dispersive_desc {
  int32_t kind;
  int32_t reserved0;
  double params[3];
  double eps_inf;
} oems_dispersive_desc;

/* RlcElement (src/extensions/lumped_rlc.rs:20-112); type 0 parallel, 1
 * series; resistance / inductance / capacitance <= 0 mean absent.  Applied
 * after the E update as LumpedRlc::post_update_e (:263-286). */
typedef struct oems_lumped_rlc_desc {
  uint64_t position[3];
  uint32_t direction;
  int32_t type;
  double resistance, inductance, capacitance;
} oems_lumped_rlc_desc;

/* Frequency-domain field dump (FrequencyDomainFieldDump,
 * src/processing/fields_fd.rs:31-217) over a half-open cell region with
 * per-axis sub-sampling.  X(f) += x(t) exp(-j 2 pi f t) 2 dt interval at every
 * timestep count that is a multiple of `interval` (>= 1; the reference
 * accumulates every call with 2 dt), E at t = n dt and H at (n - 1/2) dt,
 * in f64.  components: bit c records component c (0..2 Ex Ey Ez, 3..5 Hx Hy
 * Hz); FdDumpType EField / HField / Both are 0x07 / 0x38 / 0x3F. */
typedef struct oems_field_dft_desc {
  uint64_t region[6];
  uint32_t sub_sample[3];
  uint32_t components;
  uint32_t interval;
  uint32_t reserved0;
} oems_field_dft_desc;

/* Near-field to far-field recording box on the node planes start..stop
 * (1 <= start < stop <= n - 1 per axis), faces -x +x -y +y -z +z enabled by
 * `directions` (the nf2ff box of python/openEMS/nf2ff.py:38-97 with
 * frequency-domain recording).  Per face it records tangential E on the
 * face plane and tangential H averaged over the two half-cells around it, in
 * f64 at the sampled timesteps as above. */
typedef struct oems_nf2ff_box_desc {
  uint64_t start[3], stop[3];
  int32_t directions[6];
  uint32_t interval;
  uint32_t reserved0;
} oems_nf2ff_box_desc;

/* Far-field request (nf2ff.CalcNF2FF, python/openEMS/nf2ff.py:98-165):
 * angles in radians, observation radius in metres, phase centre, and the
 * mesh lines in metres per axis (n + 1 values; NULL = uniform delta). */
typedef struct oems_nf2ff_request {
  const double* theta;
  uint64_t ntheta;
  const double* phi;
  uint64_t nphi;
  double radius;
  double center[3];
  const double* lines[3];
} oems_nf2ff_request;

/* Far-field result (nf2ff_results, python/openEMS/nf2ff.py:167-220), caller
 * owned, theta-major: e_theta / e_phi 2 x ntheta x nphi doubles (re, im) in
 * V/m at the radius, p_rad ntheta x nphi in W/m^2 (= |E|^2 / (2 Z0)); any
 * pointer may be NULL.  prad = the integral of p_rad r^2 sin(theta) over the
 * requested grid (trapezoid rule), dmax = 4 pi r^2 max(p_rad) / prad: both
 * need a grid covering the whole sphere. */
typedef struct oems_nf2ff_result {
  double* e_theta;
  double* e_phi;
  double* p_rad;
  double prad;
  double dmax;
} oems_nf2ff_result;

/* Field components for probes: 0..2 = Ex Ey Ez, 3..5 = Hx Hy Hz. */
#define OEMS_COMPONENT_EX 0
#define OEMS_COMPONENT_HX 3

/* ---- lifetime ---------------------------------------------------------- */

OEMS_API oems_status oems_engine_create(const oems_operator_desc* desc, oems_engine** out);
OEMS_API void oems_engine_destroy(oems_engine* engine);
/* Engine device memory comes from a stream-ordered pool per device that keeps
 * freed blocks for the next engine (no device-wide synchronisation when an
 * engine is destroyed); this returns the device's unused pooled memory and
 * the cached pinned host buffers to the driver.  device < 0: the current
 * device. */
OEMS_API oems_status oems_release_cached_memory(int32_t device);

/* ---- TF/SF plane source (src/extensions/tfsf.rs:54-355) ---------------- */

/* TfsfConfig: direction 0 XPlus 1 XMinus 2 YPlus 3 YMinus 4 ZPlus 5 ZMinus
 * (as in the reference only the axis is used), polarization 0 Transverse1
 * (E along axis+1, H along axis+2) or 1 Transverse2, frequency (Hz) and
 * amplitude (V/m) of the sinusoid driving the 1D auxiliary grid,
 * boundary_layer the plane index along the axis, phase_velocity <= 0: c0. */
typedef struct oems_tfsf_desc {
  int32_t direction;
  int32_t polarization;
  double frequency;
  double amplitude;
  uint64_t boundary_layer;
  double phase_velocity;
  int32_t kind;      /* 0: the reference's update, whose 1D grid has the wrong
                        sign in its E update and grows exponentially; 1: the
                        corrected source (positive directions, boundary_layer
                        >= 1): stable 1D grid, scattered-side H plane at
                        boundary_layer - 1, total-side E plane at boundary_layer */
  int32_t reserved0;
} oems_tfsf_desc;

/* ---- EngineImpl --------------------------------------------------------- */

OEMS_API oems_status oems_engine_run_batch(oems_engine* engine, const oems_batch* batch,
                                  oems_batch_result* result);
OEMS_API oems_status oems_engine_current_timestep(const oems_engine* engine, uint64_t* timestep);
/* e[c], h[c]: host buffers of nx*ny*nz floats each. */
OEMS_API oems_status oems_engine_read_fields(oems_engine* engine, float* const e[3], float* const h[3]);
OEMS_API oems_status oems_engine_write_fields(oems_engine* engine, const float* const e[3],
                                     const float* const h[3]);
/* Clears fields, extension state and the timestep counter. */
OEMS_API oems_status oems_engine_reset(oems_engine* engine);

/* ---- packs: several engines stepped together ------------------------------
 * No counterpart in the reference (its EngineBatch batches timesteps of one
 * grid, src/fdtd/batch.rs:12-32).  A pack holds engines of one device and
 * one field storage, with full coefficient arrays and only CPML, sources,
 * probes and probe DFTs attached.  oems_pack_run_batch runs batches[i] on
 * engine i for every i with batches[i] != NULL, with the results and state
 * oems_engine_run_batch would give each engine on its own (bit for bit),
 * but every half-step of all of them is one launch of the plain update
 * kernels over the grids without CPML and one of the CPML kernels over the
 * grids with it, replayed from CUDA graphs, with one post-step launch and
 * one energy launch pair for all.  The first batch times the update
 * kernels' CTA size, x-planes per work item and whether CPML grids enter
 * whole or split (below) on saved copies of the engines' state (restored
 * afterwards) and keeps the fastest; a batch whose engines hold under half
 * the cells of the tuned set tunes again.  oems_pack_set_shape fixes the
 * shape instead.  The batches must share num_steps,
 * sample_interval, check_interval and whether they carry an energy-decay end
 * condition, and their engines must be at the same timestep; each engine
 * keeps its own decay threshold, peak and termination step.  statuses[i] is
 * OEMS_ERR_NUMERICAL for an engine whose energy stopped being finite (it
 * stops at that check), OEMS_OK otherwise.  The engines must not be used
 * elsewhere while a pack call runs; destroy the pack before its engines. */
typedef struct oems_pack oems_pack;
OEMS_API oems_status oems_pack_create(oems_engine* const* engines, uint64_t count, oems_pack** out);
OEMS_API void oems_pack_destroy(oems_pack* pack);
OEMS_API oems_status oems_pack_run_batch(oems_pack* pack, const oems_batch* const* batches,
                                         oems_batch_result* results, oems_status* statuses);
/* The update kernels' launch shape: CTAs of `threads` (a multiple of 32, at
 * most 512) over work items of `ichunk` x-planes, and `split`: 0 gives each
 * CPML grid to the CPML launch whole; 1 as two parts, its CPML-free box
 * (plain kernels) and its slab cells (CPML kernels); 2 and 3 as 1 with the
 * CPML launch on a second stream beside the plain one (3: the plain
 * launch's grid cut by one CTA per SM to leave room for it).  Setting it
 * skips the tuning of the first batch. */
OEMS_API oems_status oems_pack_set_shape(oems_pack* pack, int32_t threads, int32_t ichunk,
                                         int32_t split);
OEMS_API oems_status oems_pack_shape(const oems_pack* pack, int32_t* threads, int32_t* ichunk,
                                     int32_t* split);

/* ---- checkpoint / resume --------------------------------------------------
 * The engine's evolving state as sections: the buffers oems_engine_reset
 * clears (fields in their storage type, CPML psi, Mur, probe DFTs, each
 * dispersive material, lumped RLC, UPML flux, each field DFT dump, each NF2FF
 * box, the TF/SF 1D grid), in a fixed order that depends only on the
 * extensions attached.  A snapshot is every section plus the two counters;
 * loading it into an engine built the same way continues the run bit for bit.
 * The reference has only read_fields / write_fields (src/fdtd/engine_impl.rs:59-70). */
enum {
  OEMS_STATE_FIELDS = 1,
  OEMS_STATE_CPML = 2,
  OEMS_STATE_MUR = 3,
  OEMS_STATE_PROBE_DFT = 4,
  OEMS_STATE_DISPERSIVE = 5,
  OEMS_STATE_LUMPED_RLC = 6,
  OEMS_STATE_UPML = 7,
  OEMS_STATE_FIELD_DFT = 8,
  OEMS_STATE_NF2FF = 9,
  OEMS_STATE_TFSF_E = 10,
  OEMS_STATE_TFSF_H = 11
};
typedef struct oems_state_section {
  uint32_t kind;    /* OEMS_STATE_* */
  uint32_t variant; /* how the bytes are encoded beyond their kind: for
                       OEMS_STATE_FIELDS the field storage (0 float, 1 IEEE
                       half, 2 bfloat16 -- half and bfloat16 sections have the
                       same size, so only this tells them apart); 0 otherwise */
  uint64_t bytes;
} oems_state_section;
/* Writes up to `capacity` section descriptors; *count = the number of sections. */
OEMS_API oems_status oems_engine_state_sections(oems_engine* engine, oems_state_section* out,
                                                uint64_t capacity, uint64_t* count);
/* Copies section `index` to / from host memory; `bytes` must equal its size,
 * and for a write `variant` must equal the section's (a snapshot of half
 * fields is refused by a bfloat16 engine and the reverse). */
OEMS_API oems_status oems_engine_read_state(oems_engine* engine, uint64_t index, void* host, uint64_t bytes);
OEMS_API oems_status oems_engine_write_state(oems_engine* engine, uint64_t index, uint32_t variant,
                                             const void* host, uint64_t bytes);
/* The step counter and the TF/SF 1D grid's step; setting them also empties
 * the probe-trace buffer, as oems_engine_reset does. */
OEMS_API oems_status oems_engine_get_state_counters(const oems_engine* engine, uint64_t* timestep,
                                                    uint64_t* tfsf_step);
OEMS_API oems_status oems_engine_set_state_counters(oems_engine* engine, uint64_t timestep, uint64_t tfsf_step);

/* ---- extensions ---------------------------------------------------------- */

OEMS_API oems_status oems_engine_add_cpml(oems_engine* engine, const oems_cpml_desc* desc);
/* MurAbc::new (src/extensions/mur_abc.rs:175). */
OEMS_API oems_status oems_engine_add_mur(oems_engine* engine, const oems_mur_desc* desc);
/* TfsfBoundary::new (src/extensions/tfsf.rs:142-190): before every H update
 * plane boundary_layer of the H component gets h - db e_inc, before every E
 * update that of the E component gets e + cb h_inc, the 1D grid's values
 * there.  Float field storage only. */
OEMS_API oems_status oems_engine_add_tfsf(oems_engine* engine, const oems_tfsf_desc* desc);
/* Upml::new (src/extensions/pml.rs:209-219) with the flux hooks of
 * pml.rs:505-655 around the H and E updates.  Kind 0 reproduces the
 * reference's coefficients, under which the scheme grows without bound (the
 * reference disables its PML tests, src/fdtd/engine_testing.rs:2322-2330);
 * kind 1 is the corrected uniaxial PML (see oems_upml_desc). */
OEMS_API oems_status oems_engine_add_upml(oems_engine* engine, const oems_upml_desc* desc);
/* LorentzMaterial / DrudeMaterial / DebyeMaterial::new (src/extensions/
 * dispersive.rs:134, 476, 570); cells: ncells x (i, j, k). Materials apply in
 * the order they are added. */
OEMS_API oems_status oems_engine_add_dispersive(oems_engine* engine, const oems_dispersive_desc* desc,
                                                const uint64_t* cells, uint64_t ncells);
/* FrequencyDomainFieldDump::new (src/processing/fields_fd.rs:73-123) with
 * set_sub_sample (:126-128); recording starts with the next batch. */
OEMS_API oems_status oems_engine_add_field_dft(oems_engine* engine, const oems_field_dft_desc* desc,
                                               const double* freqs, uint32_t nfreq, int32_t* dump_id);
/* get_e_field / get_h_field (src/processing/fields_fd.rs:222-238) for one
 * component: npoints (re, im) pairs in region order (k fastest) of the
 * sub-sampled region. */
OEMS_API oems_status oems_engine_read_field_dft(oems_engine* engine, int32_t dump_id, uint32_t freq_index,
                                                uint32_t component, double* out, uint64_t npoints);
/* NF2FF recording box (no counterpart in the reference engine). */
OEMS_API oems_status oems_engine_add_nf2ff_box(oems_engine* engine, const oems_nf2ff_box_desc* desc,
                                               const double* freqs, uint32_t nfreq, int32_t* box_id);
/* Raw accumulators of one face (0..5 = -x +x -y +y -z +z) at one frequency:
 * 4 arrays Eb, Ec, Hb, Hc (b = a+1, c = a+2 mod 3 for normal axis a) of
 * nb x nc points (b-major) as (re, im); *npoints receives nb nc; out NULL
 * only queries the size. */
OEMS_API oems_status oems_engine_read_nf2ff_face(oems_engine* engine, int32_t box_id, uint32_t face,
                                                 uint32_t freq_index, double* out, uint64_t cap_doubles,
                                                 uint64_t* npoints);
/* Far field of a recorded box at one of its frequencies (Nf2ff::calculate,
 * src/nf2ff/mod.rs:117-170, with the radiation vectors its
 * integrate_surfaces leaves at zero computed on the GPU in f64). */
OEMS_API oems_status oems_engine_nf2ff(oems_engine* engine, int32_t box_id, uint32_t freq_index,
                                       const oems_nf2ff_request* request, oems_nf2ff_result* result);
/* The same transform from a host point list: npoints x 16 doubles
 * (x y z weight, J (re, im) x 3, M (re, im) x 3; J = n x H, M = -n x E,
 * weight = area).  device -1 = current. */
OEMS_API oems_status oems_nf2ff_surface(int32_t device, const double* points, uint64_t npoints, double frequency,
                                        const oems_nf2ff_request* request, oems_nf2ff_result* result);
/* LumpedRlc::new (src/extensions/lumped_rlc.rs:145-160).  Elements apply in
 * list order; adding elements restarts every element's integrator at 0. */
OEMS_API oems_status oems_engine_add_lumped_rlc(oems_engine* engine, const oems_lumped_rlc_desc* elements,
                                                uint64_t n);

/* ---- probes ---------------------------------------------------------------- */

/* One term of a probe: the value of `component` at `position`, with weight. */
typedef struct oems_probe_term {
  int32_t component; /* 0..2 = Ex Ey Ez, 3..5 = Hx Hy Hz */
  int32_t reserved0;
  uint64_t position[3];
  double weight;
} oems_probe_term;

/* Probe modes.  F32: the term values summed in order in f32, weight +1 adds
 * and weight -1 subtracts (VoltageProbe::sample / CurrentProbe::sample,
 * src/processing/probes.rs:98-239).  F64: sum of weight * value in f64, one
 * rounding per term (the integrals of EngineInterface::calc_voltage_integral /
 * calc_current_integral, src/fdtd/engine_interface.rs:208-305, recorded per
 * step, and the port loop integrals; for a current integral the reference
 * subtracts each cell's two products before adding them, which
 * oems_engine_integral follows). */
#define OEMS_PROBE_SUM_F32 0
#define OEMS_PROBE_SUM_F64 1

/* A probe records one value per executed step, after the excitation: E
 * values belong to t = (n+1) dt, H values to (n+1/2) dt. */
OEMS_API oems_status oems_engine_add_probe(oems_engine* engine, const oems_probe_term* terms,
                                           uint64_t nterms, int32_t mode, int32_t* probe_id);
/* FieldProbe-style single value (src/processing/probes.rs:289-303). */
OEMS_API oems_status oems_engine_add_point_probe(oems_engine* engine, int32_t component,
                                        const uint64_t position[3], int32_t* probe_id);
/* Traces of the most recent batch, layout [step][probe], f64; *steps_out
 * receives the number of steps recorded (at most max_steps are copied). */
OEMS_API oems_status oems_engine_read_probe_traces(oems_engine* engine, double* out, uint64_t max_steps,
                                          uint64_t* steps_out);
/* Running DFT of a probe's trace (FrequencyDomainFieldDump::accumulate,
 * src/processing/fields_fd.rs:149-217, applied to the probe value):
 * X(f) += x(t) exp(-j 2 pi f t) 2 dt in f64, t = (timestep after the step -
 * h) dt with h = 1/2 for a probe of H components only, 0 otherwise.
 * Accumulates over every step run after the call, until reset. */
OEMS_API oems_status oems_engine_add_probe_dft(oems_engine* engine, int32_t probe_id,
                                               const double* freqs, uint64_t nfreq, int32_t* dft_id);
/* out: 2 * nfreq doubles (re, im per frequency). */
OEMS_API oems_status oems_engine_read_probe_dft(oems_engine* engine, int32_t dft_id, double* out);

/* ---- engine interface (EngineInterface / EngineInterfaceMut,
 * src/fdtd/engine_interface.rs:27-595): field reads at positions, on the
 * resident fields ---- */

/* Sampled quantity: E, H (get_e_field / get_h_field, :131-154) or curl H at
 * the snapped cell (get_rot_h_field and get_j_field, :157-206, :336-377;
 * interpolation is ignored for it). */
#define OEMS_SAMPLE_E 0
#define OEMS_SAMPLE_H 1
#define OEMS_SAMPLE_CURL_H 2
/* InterpolationType (:12-20). */
#define OEMS_INTERP_NONE 0
#define OEMS_INTERP_NODE 1
#define OEMS_INTERP_CELL 2

typedef struct oems_sample_desc {
  int32_t quantity;        /* OEMS_SAMPLE_* */
  int32_t interpolation;   /* OEMS_INTERP_*; used with positions only */
  const double* lines[3];  /* the grid's mesh lines per axis, in grid units */
  uint64_t nlines[3];      /* lines per axis: the engine's cells + 1 */
  double unit;             /* metres per grid unit (Grid::unit) */
} oems_sample_desc;

/* count queries, each either a position in metres (positions: [count][3];
 * snapped like EngineInterface::snap_to_grid, :327-333, then read as the
 * interpolation says) or a cell (cells: [count][3]; get_e_field_raw /
 * get_h_field_raw, :113-128, or curl H there).  Give exactly one of the two.
 * values: [count][3] f64, the bits of the reference's f64 arithmetic;
 * snapped (optional): [count][3], the cell each query read at (for
 * get_d_field / get_b_field, :165-199, which scale by the material there).
 * Synchronous: returns after the values are in host memory. */
OEMS_API oems_status oems_engine_sample(oems_engine* engine, const oems_sample_desc* desc, const double* positions,
                                        const uint64_t* cells, uint64_t count, double* values, uint64_t* snapped);
/* calc_voltage_integral (kind 0, :208-247) or calc_current_integral (kind 1,
 * :251-305; normal_dir 0 = x, 1 = y, anything larger = z) between two
 * positions in metres, snapped like the samples, on the current fields: the
 * reference's loop order and f64 arithmetic (a current term's two products
 * are subtracted before the sum takes them).  desc gives the grid; its
 * quantity and interpolation are ignored.  Synchronous. */
OEMS_API oems_status oems_engine_integral(oems_engine* engine, const oems_sample_desc* desc, int32_t kind,
                                          const double start[3], const double stop[3], int32_t normal_dir,
                                          double* value);
/* A probe term list evaluated once on the current fields, in list order with
 * the probes' arithmetic: with OEMS_PROBE_SUM_F32 the VoltageProbe /
 * CurrentProbe::sample of the present step (src/processing/probes.rs:98-239).
 * Synchronous. */
OEMS_API oems_status oems_engine_eval_terms(oems_engine* engine, const oems_probe_term* terms, uint64_t nterms,
                                            int32_t mode, double* value);
/* EngineInterfaceMut::set_e_field / set_h_field / add_e_field (:542-561):
 * field 0 = E, 1 = H; values [count][3] f32 replace (add = 0) or are added
 * to (add != 0) the cell's three components, applied in list order.
 * Synchronous. */
OEMS_API oems_status oems_engine_set_cells(oems_engine* engine, int32_t field, const uint64_t* cells,
                                           const float* values, uint64_t count, int32_t add);

/* Unweighted field energies sum(E^2), sum(H^2) in f64 over the whole grid
 * (VectorField3D::energy, src/arrays/field.rs:314-316), computed on the GPU. */
OEMS_API oems_status oems_engine_energy(oems_engine* engine, double* e_energy, double* h_energy);

/* Energies without allocation.  No counterpart in the reference.  For callers
 * that cannot let the library call cudaMalloc (a host that owns all device
 * memory, a loop that must not stall on an allocation's implicit device
 * synchronisation): the same sums as oems_engine_energy, computed from six
 * caller-owned device arrays (Ex Ey Ez Hx Hy Hz, `count` floats each, 16-byte
 * aligned, count <= 67108864), written to the device pointer `energies`
 * (energies[0] = sum E^2, energies[1] = sum H^2), on `stream` (a
 * cudaStream_t; NULL = the legacy default stream), asynchronously.  Partial
 * sums live in a fixed 192 KB device array inside the library that every call
 * on a device shares (calls that overlap on the GPU race on it).  Each call
 * looks up that array's address in the current context (so a device reset
 * leaves no stale address behind); the first call on a device also loads the
 * library's device code there, so make it before any stream capture. */
OEMS_API oems_status oems_field_energy_noalloc(const float* const fields[6], uint64_t count,
                                               double* energies, void* stream);

/* ---- diagnostics ---------------------------------------------------------- */

/* Per-kernel timing: while enabled, run_batch launches the update kernels one
 * by one (no graphs) with CUDA events around every H and E launch on the
 * engine's stream, and accumulates their device time.  Enabling resets the
 * totals. */
OEMS_API oems_status oems_engine_set_kernel_profiling(oems_engine* engine, int32_t enable);
/* Launch shape chosen for the update kernels (valid after the first batch):
 * staged = 0 for the register kernels, 1 for the bulk-async staged kernels
 * (2: staged on the box between the x / y CPML slabs, register kernels on
 * the slabs; 3: the z-split, plain register kernels on the CPML-free box and
 * CPML register kernels on every slab cell; 4: the pipelined register
 * kernels), threads per CTA, x-planes per work item, rows per tile (staged),
 * pipeline stages (staged, pipelined) or the L2 prefetch distance in
 * x-planes (register kernels, 0 = none), CTAs. */
OEMS_API oems_status oems_engine_launch_info(const oems_engine* engine, int32_t* staged,
                                             int32_t* threads, int32_t* ichunk,
                                             int32_t* rows_per_tile, int32_t* stages,
                                             int32_t* grid);
/* One launch shape the autotuner timed: kind as `staged` above, threads per
 * CTA, x-planes per work item, pipeline stages (staged, pipelined) or, for
 * the register kernels, the L2 prefetch distance + 10 x the register budget
 * variant + 100 x that of the CPML slab kernels of a z-split (0: up to 128
 * registers with 512-thread CTAs, 1 / 2: 256-thread CTAs capped at 85 / 64
 * registers) + 1000 for a forked z-split slab launch (2000 with the interior
 * grid cut by one CTA per SM), the number of H + E pairs timed and their
 * device time in milliseconds. */
typedef struct oems_tune_entry {
  int32_t kind;
  int32_t threads;
  int32_t ichunk;
  int32_t extra;
  int32_t reps;
  float ms;
} oems_tune_entry;
/* The candidates of the tuning that chose this engine's shape (the process
 * caches tunings per grid and variant, so a later engine of the same grid
 * reports the same list).  Writes min(capacity, count) entries; out may be
 * NULL to ask for the count.  No reference counterpart: a diagnostic of the
 * project's autotuner. */
OEMS_API oems_status oems_engine_tune_report(const oems_engine* engine, oems_tune_entry* out,
                                             uint64_t capacity, uint64_t* count);
OEMS_API oems_status oems_engine_kernel_profile(const oems_engine* engine, double* h_seconds,
                                                uint64_t* h_launches, double* e_seconds,
                                                uint64_t* e_launches);

/* ---- cylindrical engine (src/fdtd/cylindrical.rs:394-638) ------------- */

/* CylindricalOperator's per-cell coefficients (rho-major, z fastest, n_rho x
 * n_alpha x n_z floats each): vi[c] = dt / (eps0 area), iv[c] = dt / (mu0
 * length) of component c (rho, alpha, z); vv = ii = 1. */
typedef struct oems_cyl_engine oems_cyl_engine;
typedef struct oems_cyl_desc {
  uint64_t n_rho, n_alpha, n_z;
  int32_t closed_alpha; /* alpha spans 2 pi: neighbours wrap around */
  int32_t r0_included;  /* the first rho line is R = 0 (needs n_rho >= 2) */
  double dt;
  const float* vi[3];
  const float* iv[3];
  int32_t device;       /* < 0: current */
  int32_t reserved0;
} oems_cyl_desc;
/* CylindricalEngine::new; fields start at zero. */
OEMS_API oems_status oems_cyl_create(const oems_cyl_desc* desc, oems_cyl_engine** out);
OEMS_API void oems_cyl_destroy(oems_cyl_engine* engine);
/* `steps` x step(): voltage pass, the R = 0 fix-up, current pass. */
OEMS_API oems_status oems_cyl_step(oems_cyl_engine* engine, uint64_t steps);
/* e[c], h[c]: host buffers of n_rho * n_alpha * n_z floats. */
OEMS_API oems_status oems_cyl_read_fields(oems_cyl_engine* engine, float* const e[3], float* const h[3]);
OEMS_API oems_status oems_cyl_write_fields(oems_cyl_engine* engine, const float* const e[3],
                                           const float* const h[3]);
OEMS_API oems_status oems_cyl_reset(oems_cyl_engine* engine);
/* Device time (CUDA events on the engine's stream) of the last oems_cyl_step. */
OEMS_API oems_status oems_cyl_last_step_ms(const oems_cyl_engine* engine, float* ms);
/* timestep() and time() (the sum of dt over the steps, as the reference). */
OEMS_API oems_status oems_cyl_time(const oems_cyl_engine* engine, uint64_t* timestep, double* time);

OEMS_API const char* oems_status_string(oems_status status);
/* Detail of the last failure on the calling thread ("" if none). */
OEMS_API const char* oems_last_error_message(void);
OEMS_API int32_t oems_abi_version(void);
/* Launch statistics of the most recent batch: kernels launched on the GPU
 * (each graph node counts) and the device time of the batch in seconds. */
OEMS_API oems_status oems_engine_last_batch_stats(const oems_engine* engine, uint64_t* kernel_launches,
                                         double* device_seconds);

#ifdef __cplusplus
}
#endif
#endif /* OEMS_H */
