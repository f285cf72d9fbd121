/*
 * oems_host.h -- C ABI of the host-side mirror of the reference's
 * Operator / Excitation / Simulation surface (liboems_b200.so).
 *
 * The Rust openEMS rewrite keeps these types in Rust (its FFI would bind only
 * include/oems.h).  Without a Rust toolchain, the same surface is provided in
 * C++ so that C, C++ and Python callers can build an operator, sample
 * excitations and run a simulation exactly as the reference does:
 *
 *   Grid::uniform / Grid::cartesian   src/geometry/mod.rs:60-71     -> oems_operator_create*
 *   Operator::new                     src/fdtd/operator.rs:59-77    -> oems_operator_create*
 *   Operator::set_material            src/fdtd/operator.rs:187-244  -> oems_operator_set_material
 *   Operator::set_pec                 src/fdtd/operator.rs:249-263  -> oems_operator_set_pec
 *   Operator::timestep/dimensions     src/fdtd/operator.rs:145-159  -> oems_operator_info
 *   Operator::e/h_coefficients        src/fdtd/operator.rs:163-171  -> oems_operator_coefficients
 *   Excitation::gaussian & co.        src/fdtd/excitation.rs:67-147 -> oems_excitation_*
 *   Excitation::evaluate              src/fdtd/excitation.rs:150-200 -> oems_excitation_evaluate
 *   ScheduledExcitation::from_excitation src/fdtd/batch.rs:110-129  -> oems_excitation_sample
 *   Simulation::new/setup/run         src/fdtd/simulation.rs:96-360 -> oems_simulation_*
 */
#ifndef OEMS_HOST_H
#define OEMS_HOST_H

#include <stdint.h>

#include "oems.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct oems_operator oems_operator;
typedef struct oems_simulation oems_simulation;

/* ---- Operator ----------------------------------------------------------- */

/* Compressed coefficients (replaces CompressedCoefficients::from_fields,
 * src/fdtd/compressed.rs:125-192): deduplicates the 12 coefficients of each
 * of ncells cells (coef = ca0..2, cb0..2, da0..2, db0..2, one float per cell
 * each) into a table of unique sets, compared bit for bit, with ids in cell
 * order -- the engine's OEMS_ENGINE_COMPRESSED storage.  ids (ncells,
 * may be NULL) receives each cell's set; table (may be NULL) the first
 * table_cap sets, 12 floats each; *nunique the number of sets.
 * OEMS_ERR_MATERIAL above 65536 sets. */
OEMS_API oems_status oems_compress_coefficients(const float* const coef[12], uint64_t ncells, uint16_t* ids,
                                                float* table, uint32_t table_cap, uint32_t* nunique);

/* Cartesian grid from mesh lines (cells = lines - 1 per axis), scaled by unit. */
OEMS_API oems_status oems_operator_create(const double* x_lines, uint64_t nxl, const double* y_lines,
                                 uint64_t nyl, const double* z_lines, uint64_t nzl, double unit,
                                 oems_operator** out);
/* Grid::uniform(nx, ny, nz, delta). */
OEMS_API oems_status oems_operator_create_uniform(uint64_t nx, uint64_t ny, uint64_t nz, double delta,
                                         oems_operator** out);
OEMS_API void oems_operator_destroy(oems_operator* op);
/* Independent copy (grid, dt and all coefficients). */
OEMS_API oems_status oems_operator_clone(const oems_operator* op, oems_operator** out);
/* region = i0, i1, j0, j1, k0, k1 (half-open, clipped to the grid). */
OEMS_API oems_status oems_operator_set_material(oems_operator* op, double eps_r, double mu_r,
                                       double sigma_e, double sigma_m, const uint64_t region[6]);
OEMS_API oems_status oems_operator_set_pec(oems_operator* op, const uint64_t region[6]);
/* set_material's coefficients on a list of cells (ncells x (i, j, k)), for
 * shapes other than boxes (spheres, shells); later calls overwrite. */
OEMS_API oems_status oems_operator_set_material_cells(oems_operator* op, double eps_r, double mu_r,
                                                      double sigma_e, double sigma_m, const uint64_t* cells,
                                                      uint64_t ncells);
OEMS_API oems_status oems_operator_info(const oems_operator* op, uint64_t dims[3], double* dt,
                               double delta[3]);
/* Borrowed pointers to the 12 coefficient arrays (ca0 ca1 ca2 cb0 cb1 cb2 da0
 * da1 da2 db0 db1 db2), valid until the operator is modified or destroyed. */
OEMS_API oems_status oems_operator_coefficients(const oems_operator* op, const float* out[12]);
/* Lumped resistor R and/or capacitor C across the E edge (position,
 * direction), folded into that edge's Ca/Cb (no counterpart in the
 * reference, whose LumpedRlc leaves a series resistor without effect):
 * eps = eps_r eps0 + C dl / A, sigma = sigma + dl / (R A) with dl the edge
 * length and A the cell face normal to it; R or C <= 0 means absent.
 * *source_scale (may be NULL) receives the factor that turns a voltage
 * source in series with R into the soft-source sample added to that E
 * component: dt / (eps (1 + sigma dt / 2 eps) R A). */
OEMS_API oems_status oems_operator_set_lumped(oems_operator* op, const uint64_t position[3],
                                              int32_t direction, double resistance,
                                              double capacitance, double eps_r, double sigma,
                                              double* source_scale);
/* Fills an engine descriptor that borrows the operator's arrays. */
OEMS_API oems_status oems_operator_engine_desc(const oems_operator* op, int32_t device, uint32_t flags,
                                      oems_operator_desc* out);

/* ---- Excitation ---------------------------------------------------------- */

/* ExcitationType (src/fdtd/excitation.rs:9-42). */
#define OEMS_EXC_GAUSSIAN 0           /* params: t0, tau            */
#define OEMS_EXC_SINUSOIDAL 1         /* params: frequency          */
#define OEMS_EXC_GAUSSIAN_MODULATED 2 /* params: frequency, t0, tau */
#define OEMS_EXC_DIRAC 3
#define OEMS_EXC_STEP 4

typedef struct oems_excitation {
  int32_t kind;
  uint32_t direction;
  uint64_t position[3];
  double params[3];
  double amplitude;
  int32_t soft_source;
  int32_t reserved0;
} oems_excitation;

OEMS_API oems_status oems_excitation_gaussian(double center_freq, double bandwidth, uint32_t direction,
                                     const uint64_t position[3], oems_excitation* out);
OEMS_API oems_status oems_excitation_gaussian_modulated(double center_freq, double bandwidth,
                                               uint32_t direction, const uint64_t position[3],
                                               oems_excitation* out);
OEMS_API oems_status oems_excitation_sinusoidal(double frequency, uint32_t direction,
                                       const uint64_t position[3], oems_excitation* out);
OEMS_API oems_status oems_excitation_dirac(double amplitude, uint32_t direction, const uint64_t position[3],
                                  oems_excitation* out);
OEMS_API double oems_excitation_evaluate(const oems_excitation* exc, double t);
/* out[s] = (float) evaluate((start_timestep + s) * dt), s < n. */
OEMS_API oems_status oems_excitation_sample(const oems_excitation* exc, uint64_t start_timestep, uint64_t n,
                                   double dt, float* out);

/* ---- probe term builders --------------------------------------------------
 * Each fills up to `cap` terms into `out` and the required count into *n
 * (call with cap = 0 to size the buffer); the terms go to
 * oems_engine_add_probe with the mode named below. */

/* VoltageProbe::sample (src/processing/probes.rs:98-131): E[direction] summed
 * over the inclusive line start..end along `direction`; mode F32.  An
 * invalid direction gives no term (value 0). */
OEMS_API oems_status oems_probe_voltage_terms(const uint64_t start[3], const uint64_t end[3],
                                              int32_t direction, oems_probe_term* out, uint64_t cap,
                                              uint64_t* n);
/* CurrentProbe::sample (src/processing/probes.rs:193-239): +H and -H of the
 * two tangential components over the inclusive surface; mode F32. */
OEMS_API oems_status oems_probe_current_terms(const uint64_t start[3], const uint64_t end[3],
                                              int32_t normal, oems_probe_term* out, uint64_t cap,
                                              uint64_t* n);
/* EngineInterface::calc_voltage_integral (src/fdtd/engine_interface.rs:208-
 * 247) between cell indices: V = -sum E . dl along x, then y, then z; mode F64. */
OEMS_API oems_status oems_probe_voltage_integral_terms(const oems_operator* op, const uint64_t start[3],
                                                       const uint64_t stop[3], oems_probe_term* out,
                                                       uint64_t cap, uint64_t* n);
/* EngineInterface::calc_current_integral (src/fdtd/engine_interface.rs:251-
 * 305) between cell indices; mode F64. */
OEMS_API oems_status oems_probe_current_integral_terms(const oems_operator* op, const uint64_t start[3],
                                                       const uint64_t stop[3], int32_t normal,
                                                       oems_probe_term* out, uint64_t cap, uint64_t* n);
/* Lumped-port probes on the E edge (position, direction): kind 0 voltage
 * V = -E . dl over the edge; kind 1 current I = loop integral of H around the
 * edge (the curl of H that drives that E component, times the cell sides);
 * mode F64. */
OEMS_API oems_status oems_probe_port_terms(const oems_operator* op, const uint64_t position[3],
                                           int32_t direction, int32_t kind, oems_probe_term* out,
                                           uint64_t cap, uint64_t* n);

/* ---- Simulation ---------------------------------------------------------- */

/* EndCondition (src/fdtd/simulation.rs:36-43). */
#define OEMS_END_TIMESTEPS 0
#define OEMS_END_ENERGY_DECAY 1
#define OEMS_END_SIMULATION_TIME 2

/* SimulationStats (src/fdtd/simulation.rs:53-66). */
typedef struct oems_simulation_stats {
  uint64_t timesteps;
  double sim_time;
  double wall_time;
  double peak_energy;
  double final_energy;
  double speed_mcells_per_sec;
} oems_simulation_stats;

/* Simulation over a copy of `op` (materials included).  The engine is
 * created in setup (first run), on `device` (-1 = current) with `flags`. */
OEMS_API oems_status oems_simulation_create(const oems_operator* op, int32_t device, uint32_t flags,
                                   oems_simulation** out);
OEMS_API void oems_simulation_destroy(oems_simulation* sim);
OEMS_API oems_status oems_simulation_add_excitation(oems_simulation* sim, const oems_excitation* exc);
OEMS_API oems_status oems_simulation_set_end_condition(oems_simulation* sim, int32_t kind, double value);
/* 0 = automatic (1000 steps per batch, the reference's GPU batch size). */
OEMS_API oems_status oems_simulation_set_batch_size(oems_simulation* sim, uint64_t batch_size);
OEMS_API oems_status oems_simulation_set_cpml(oems_simulation* sim, const oems_cpml_desc* cpml);
OEMS_API oems_status oems_simulation_setup(oems_simulation* sim);
OEMS_API oems_status oems_simulation_run(oems_simulation* sim, oems_simulation_stats* stats);
/* Borrowed engine handle (NULL before setup). */
OEMS_API oems_engine* oems_simulation_engine(oems_simulation* sim);

/* ---- batched port sweep --------------------------------------------------
 * Many independent lumped-port simulations (no counterpart in the reference)
 * run to energy decay, each in its own engine and CUDA stream on one device,
 * `concurrency` of them at a time from host worker threads, so that small
 * grids together fill the GPU.  Every instance records the port voltage u =
 * E . dl and current i (into the structure) as f64 running DFTs at the
 * sweep's frequencies and returns S11 = (u - u_inc) / u_inc with u_inc =
 * (u + i R) / 2 (Port.CalcPort, python/openEMS/ports.py:136-138). */

typedef struct oems_sweep oems_sweep;

typedef struct oems_sweep_instance {
  const oems_operator* op;   /* copied by oems_sweep_add */
  oems_cpml_desc cpml;       /* all layers 0 = no CPML */
  uint64_t port_position[3]; /* E edge of the port */
  int32_t port_direction;
  int32_t reserved0;
  double port_resistance;    /* > 0 */
  double port_eps_r;         /* background of the port edge */
  double port_sigma;
  oems_excitation waveform;  /* source voltage signal; position / direction ignored */
  double energy_decay_db;    /* stop below -|value| dB of the peak; 0 = run max_timesteps */
  uint64_t max_timesteps;
} oems_sweep_instance;

typedef struct oems_sweep_result {
  uint64_t timesteps;
  int32_t termination_reason; /* OEMS_TERMINATION_* */
  int32_t status;             /* OEMS_OK or the instance's error */
  double final_decay_db;      /* energy of the last sample (every 100 steps) below the peak so far, dB
                                 (<= 0); for a decayed instance the level that ended it */
  double device_seconds;      /* sum over the instance's batches */
  double cells;
  double setup_seconds;       /* host time from the start of the instance to its first batch */
  double host_seconds;        /* host time of the instance over every run call, teardown included */
  int32_t paused;             /* 1: stopped at a run_until cap, engine kept for the next call */
  int32_t reserved0;
} oems_sweep_result;

/* freqs: the DFT frequencies of every instance (Hz).  engine_flags as for
 * oems_engine_create; concurrency >= 1. */
OEMS_API oems_status oems_sweep_create(int32_t device, uint32_t concurrency, uint32_t engine_flags,
                                       const double* freqs, uint64_t nfreq, oems_sweep** out);
OEMS_API void oems_sweep_destroy(oems_sweep* sweep);
OEMS_API oems_status oems_sweep_add(oems_sweep* sweep, const oems_sweep_instance* inst, int32_t* instance_id);
/* Runs every instance that has not ended to its end (energy decay or
 * max_timesteps); batch_steps 0 = 2000.  Returns the first instance error
 * (the others still run; see oems_sweep_get_result). */
OEMS_API oems_status oems_sweep_run(oems_sweep* sweep, uint64_t batch_steps);
/* As oems_sweep_run, but an instance stops once it has run step_cap steps in
 * total and keeps its engine (paused): a later run / run_until continues it
 * bit-for-bit as if uninterrupted.  Results of a paused instance hold the
 * DFTs and S11 of the steps run so far. */
OEMS_API oems_status oems_sweep_run_until(oems_sweep* sweep, uint64_t batch_steps, uint64_t step_cap);
/* One instance only, on the calling thread: starts or continues it until it
 * ends or has run step_cap steps in total.  Different instances may be
 * advanced from different threads at the same time (one thread per instance
 * at a time); no call may run concurrently with oems_sweep_run(_until). */
OEMS_API oems_status oems_sweep_advance(oems_sweep* sweep, int32_t instance_id, uint64_t batch_steps,
                                        uint64_t step_cap);
/* Ends a paused instance (its engine is released); its result stays the
 * partial one.  No-op for an instance that has ended. */
OEMS_API oems_status oems_sweep_finish(oems_sweep* sweep, int32_t instance_id);
/* uf, if_ and s11: 2 x nfreq doubles (re, im) each; any may be NULL. */
OEMS_API oems_status oems_sweep_get_result(const oems_sweep* sweep, int32_t instance_id, oems_sweep_result* info,
                                           double* uf, double* if_, double* s11);
/* Keep the port voltage / current time traces (f64, u then i per step) of
 * the first `steps` timesteps of every instance run afterwards; 0 = none. */
OEMS_API oems_status oems_sweep_set_trace_steps(oems_sweep* sweep, uint64_t steps);
/* out: cap_steps x 2 doubles; *nsteps receives the recorded step count. */
OEMS_API oems_status oems_sweep_get_trace(const oems_sweep* sweep, int32_t instance_id, double* out,
                                          uint64_t cap_steps, uint64_t* nsteps);
/* on != 0: oems_sweep_run / run_until step the instances that have run the
 * same number of steps together through one pack (oems_pack_run_batch in
 * oems.h): shared launches over all their grids instead of one engine and
 * stream per instance, each instance ending with the same bits.  Needs full
 * coefficient arrays (no OEMS_ENGINE_COMPRESSED).  host_seconds of a packed
 * instance is the wall time of the packed runs it took part in.
 * oems_sweep_advance always runs one instance on its own. */
OEMS_API oems_status oems_sweep_set_packed(oems_sweep* sweep, int32_t on);
/* Wall time of the last run / run_until call and the cell x timestep count
 * it executed. */
OEMS_API oems_status oems_sweep_stats(const oems_sweep* sweep, double* wall_seconds, double* cell_steps);

#ifdef __cplusplus
}
#endif
#endif /* OEMS_HOST_H */
