/*
 * oems_oracle.h -- CPU oracle for the Yee FDTD hot path (TEST INFRASTRUCTURE).
 *
 * This library is the checker, never the product: only tests/, the smoke
 * check in __graft_entry__.py and the CPU-baseline leg of bench.py load it.
 * It restates, in plain C++, the semantics of the Rust openEMS rewrite's
 * scalar reference engine and its operator:
 *
 *   - src/fdtd/basic_engine.rs:56-163   run_batch step order, energy sampling,
 *                                       energy-decay termination
 *   - src/fdtd/basic_engine.rs:191-306  H / E update loops, loop bounds and the
 *                                       zero-derivative rule at the max faces
 *   - src/fdtd/basic_engine.rs:313-395  soft / hard excitation injection
 *   - src/fdtd/operator.rs:82-263       dt and the Ca/Cb/Da/Db coefficients
 *   - src/fdtd/excitation.rs:67-200     waveforms (evaluated in f64)
 *   - src/fdtd/batch.rs:110-129         pre-sampling f64 -> f32
 *   - src/arrays/field.rs:219-221       energy = sum of squares in f64
 *   - src/extensions/cpml.rs:68-177     CPML profile coefficients (the update
 *                                       itself is the standard Roden-Gedney
 *                                       recursive convolution; the reference
 *                                       leaves its correction disabled)
 *
 * Parity status: pinned to the reference's known-answer unit tests (operator
 * coefficients, excitation waveforms, probe sums, CPML coefficient ranges,
 * energy arithmetic) and to the physics checks of its scenario tests.  The
 * reference stores no golden field arrays and cannot be compiled here (no Rust
 * toolchain), so field-level parity rests on this restatement plus a second,
 * independent numpy restatement that must agree with it bit for bit.
 *
 * Arithmetic: compiled with -ffp-contract=off and no fast-math, so every
 * `a*b + c*d` rounds each product and the sum separately, like the Rust code.
 * The oracle exists in two precisions: FP32 (bit-faithful to the reference)
 * and FP64 (the accuracy oracle: same formulas, coefficients never rounded to
 * f32).
 */
#ifndef OEMS_ORACLE_H
#define OEMS_ORACLE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct orc_sim orc_sim;

/* Excitation kinds, same order as ExcitationType (src/fdtd/excitation.rs:9-42). */
enum {
  ORC_EXC_GAUSSIAN = 0,          /* params: t0, tau            */
  ORC_EXC_SINUSOIDAL = 1,        /* params: frequency          */
  ORC_EXC_GAUSSIAN_MODULATED = 2,/* params: frequency, t0, tau */
  ORC_EXC_DIRAC = 3,
  ORC_EXC_STEP = 4
};

typedef struct {
  uint64_t timestep;
  double e_energy;
  double h_energy;
  double total_energy;
} orc_energy_sample;

typedef struct {
  uint64_t timesteps_executed;
  int32_t termination_reason; /* 0 steps completed, 1 energy decay */
  int32_t pad_;
  double final_decay_db;
  uint64_t num_energy_samples;
  double peak_energy;
} orc_batch_result;

/* dt = 0.99 * CFL limit from the minimum line spacing per axis
 * (src/fdtd/operator.rs:82-89, src/geometry/mod.rs:113-119,242-255). */
void orc_grid_timestep(const double* xl, int64_t nxl, const double* yl, int64_t nyl,
                       const double* zl, int64_t nzl, double unit, double* dt_out,
                       double* delta_out3);

/* Reference evaluate(t) in f64 (src/fdtd/excitation.rs:150-200). */
double orc_excitation_eval(int32_t kind, const double* params, double amplitude, double t);

/* precision: 32 or 64. Coefficients start as vacuum (operator.rs:92-141). */
orc_sim* orc_new(int32_t precision, int64_t nx, int64_t ny, int64_t nz, double dt,
                 double dx, double dy, double dz);
void orc_free(orc_sim* s);
void orc_set_threads(orc_sim* s, int32_t threads);
/* Loop form of the H / E updates: 0 the parallel engine's cell loop
 * (src/fdtd/parallel_engine.rs:108-172), 1 the SIMD engine's z-lines
 * (src/fdtd/simd_engine.rs:252-391) with OpenMP over x-planes.  Both give
 * identical bits. */
void orc_set_zline(orc_sim* s, int32_t on);

/* Operator::set_material / set_pec (src/fdtd/operator.rs:187-263). region =
 * i0,i1,j0,j1,k0,k1 (half-open). */
void orc_set_material(orc_sim* s, double eps_r, double mu_r, double sigma_e, double sigma_m,
                      const int64_t* region6);
void orc_set_pec(orc_sim* s, const int64_t* region6);
/* 12 arrays of n values each in the order ca0 ca1 ca2 cb0 cb1 cb2 da0 da1 da2
 * db0 db1 db2; element type float (precision 32) or double (64). */
void orc_get_coefficients(const orc_sim* s, void* out12);
void orc_set_coefficients(orc_sim* s, const void* in12);

/* Fields: 6 arrays Ex Ey Ez Hx Hy Hz, z fastest, element type per precision. */
void orc_get_fields(const orc_sim* s, void* out6);
void orc_set_fields(orc_sim* s, const void* in6);
void orc_reset(orc_sim* s);
uint64_t orc_timestep(const orc_sim* s);

/* Sampled excitation: samples[step] is applied after the E update of batch
 * step `step` (basic_engine.rs:313-395). Samples are f32 for precision 32 and
 * f64 for precision 64. */
void orc_clear_excitations(orc_sim* s);
void orc_add_excitation_sampled(orc_sim* s, const int64_t* pos3, int32_t dir, int32_t soft,
                                const void* samples, int64_t n);
/* Analytic excitation sampled by the oracle itself in its own precision. */
void orc_add_excitation_analytic(orc_sim* s, const int64_t* pos3, int32_t dir, int32_t soft,
                                 int32_t kind, const double* params, double amplitude,
                                 uint64_t start_timestep, int64_t n);

/* Probes: one value per executed step, taken after the excitation, recorded
 * as double.  A point probe (comp 0..5 = Ex Ey Ez Hx Hy Hz) is a one-term
 * probe.  General probes are term lists (comp, i, j, k, weight):
 * mode 0 sums the values in order in f32 with weights +-1 (acc = acc + v or
 * acc = acc - v), as VoltageProbe/CurrentProbe::sample do
 * (src/processing/probes.rs:98-239); mode 1 sums weight*value in f64, as
 * EngineInterface::calc_voltage/current_integral do
 * (src/fdtd/engine_interface.rs:208-305). */
void orc_add_point_probe(orc_sim* s, int32_t comp, const int64_t* pos3);
int32_t orc_add_probe(orc_sim* s, const int32_t* comps, const int64_t* pos, const double* weights,
                      int64_t nterms, int32_t mode);
void orc_get_probe_traces(const orc_sim* s, double* out, int64_t max_steps);
/* Evaluates every probe on the current fields (no step); out[probe]. */
void orc_eval_probes(orc_sim* s, double* out);
/* Running DFT of a probe trace (src/processing/fields_fd.rs:149-217):
 * X(f) += x(t) exp(-j 2 pi f t) 2 dt with t = (timestep after the step
 * - half) dt, half = 0.5 for probes of H components, 0 otherwise.
 * Accumulates over every step run after the call.  out: re, im per frequency. */
int32_t orc_add_probe_dft(orc_sim* s, int32_t probe, const double* freqs, int64_t nfreq);
void orc_get_probe_dft(const orc_sim* s, int32_t dft, double* out);

/* CPML on the faces with layers[f] > 0 (f = xmin,xmax,ymin,ymax,zmin,zmax).
 * Profile: src/extensions/cpml.rs:68-177; update: Roden-Gedney. */
int32_t orc_enable_cpml(orc_sim* s, const int32_t* layers6, double grading_order,
                        double reflection_coeff, double alpha_max, double kappa_max);
/* Per-face profile arrays for tests: out has 6 rows (b_e, c_e, ik_e, b_h, c_h,
 * ik_h) of `layers` doubles for face f (values after rounding to the sim's
 * precision). Returns the layer count, 0 if the face is disabled. */
int32_t orc_cpml_profile(const orc_sim* s, int32_t face, double* out);

/* Mur absorbing boundary on the faces with enabled[f] != 0.  order 1 restates
 * src/extensions/mur_abc.rs:88-324 (pre before the E update, post and apply
 * after it, faces applied in order); order 2 is the second-order Mur
 * condition (Mur 1981) on face interiors, first order on face edges.
 * phase_velocity <= 0 means c0.  Returns 0 or a negative error. */
/* Frequency-domain field dump (src/processing/fields_fd.rs:31-217): region
 * i0 i1 j0 j1 k0 k1 half-open, sub-sampling per axis, components by bit mask
 * (0..2 E, 3..5 H), accumulated at timesteps that are multiples of interval
 * with factor exp(-j 2 pi f t) 2 dt interval; E at t = n dt, H at
 * (n - 1/2) dt.  Returns the dump id. */
int32_t orc_add_field_dft(orc_sim* s, const int64_t* region6, const int64_t* sub3, uint32_t comp_mask,
                          const double* freqs, int64_t nfreq, uint64_t interval);
int64_t orc_field_dft_points(const orc_sim* s, int32_t id);
/* out: npoints (re, im) of frequency f, component slot (ascending order of
 * the mask), points in region order (k fastest). */
void orc_get_field_dft(const orc_sim* s, int32_t id, int64_t f, int64_t comp_slot, double* out);
/* NF2FF recording box on node planes lo..hi (1 <= lo < hi <= n - 1) with
 * faces -x +x -y +y -z +z enabled by dirs6: tangential E on the face plane and
 * tangential H averaged over the two half-planes around it. */
int32_t orc_add_nf2ff_box(orc_sim* s, const int64_t* lo3, const int64_t* hi3, const int32_t* dirs6,
                          const double* freqs, int64_t nfreq, uint64_t interval);
int64_t orc_get_nf2ff_face(const orc_sim* s, int32_t id, int32_t face, int64_t f, double* out);
/* Uniaxial PML as the reference (src/extensions/pml.rs:194-655), hooks
 * around the H and E updates (innermost); returns the number of regions. */
/* kind 0: the reference's UPML coefficients; kind 1: the corrected uniaxial
 * PML (main update coefficients of the region cells changed as well). */
int32_t orc_enable_upml(orc_sim* s, const int64_t* layers6, double grading_order, double reflection_coeff,
                        int32_t kind);
/* Upml::calculate_kappa (pml.rs:370-420) for known-answer checks. */
void orc_upml_kappa(const orc_sim* s, int32_t comp, int32_t dir, const int64_t* pos3, int32_t is_min,
                    int64_t layers, double width, double smax, double m, double* kv, double* ki);
int32_t orc_enable_mur(orc_sim* s, const int32_t* enabled6, int32_t order, double phase_velocity);
/* TF/SF plane source (src/extensions/tfsf.rs:115-355): direction 0 +x 1 -x
 * 2 +y 3 -y 4 +z 5 -z (kind 0: only the axis matters, as in the
 * reference), polarization 0 / 1 (Transverse1 / 2), phase_velocity <= 0:
 * c0; kind 0 the reference's update (its 1D grid grows exponentially), 1 the
 * corrected one (positive directions, boundary_layer >= 1).  -1 bad enum,
 * -2 boundary_layer outside the grid, -3 kind 1 limits. */
int32_t orc_enable_tfsf(orc_sim* s, int32_t direction, int32_t polarization, double frequency, double amplitude,
                        int64_t boundary_layer, double phase_velocity, int32_t kind);

/* Dispersive material on a list of cells (src/extensions/dispersive.rs),
 * applied after the E update, all three components per cell:
 *   kind 0 Drude  (:476-535)  j = a j + b e;  e = e - c j
 *   kind 1 Lorentz as the reference (:134-196) j = a j + c e; e = e - b j
 *   kind 2 Debye  (:570-630)  p' = a p + b e; e = e - c (p' - p) / dt
 *   kind 3 Lorentz, second order: p' = a p + b p_prev + c e_n;
 *          e = e - (p' - p) / (eps0 eps_inf), e_n = E before the E update
 *   kind 4 Drude as the same recursion with omega_0 = 0 (params omega_p, gamma)
 * params: Drude (omega_p, gamma) rad/s; Lorentz (omega_0, gamma, delta_eps);
 * Debye (tau, delta_eps).  eps_inf divides the E correction (1 = reference). */
int32_t orc_add_dispersive(orc_sim* s, int32_t kind, const double* params, double eps_inf,
                           const int64_t* cells, int64_t ncells);
/* LumpedRlc (src/extensions/lumped_rlc.rs:155-286) after the E update:
 * e' = v_vv e + v_il int; int += e dt.  type 0 parallel, 1 series; r, l, c
 * <= 0 mean absent. */
int32_t orc_add_lumped_rlc(orc_sim* s, const int64_t* pos3, int32_t dir, int32_t type, double r,
                           double l, double c);
/* Lumped resistor / capacitor across the E edge (pos, dir) folded into Ca/Cb
 * (eps = eps_r eps0 + C dl / A, sigma = sigma + dl / (R A)); returns the
 * factor that turns a series source voltage into the soft-source sample. */
double orc_set_lumped(orc_sim* s, const int64_t* pos3, int32_t dir, double r, double c, double eps_r,
                      double sigma);

int32_t orc_run_batch(orc_sim* s, uint64_t num_steps, uint64_t sample_interval,
                      int32_t track_peak, uint64_t check_interval, int32_t has_decay,
                      double decay_db, double initial_peak, orc_batch_result* res);
void orc_get_energy_samples(const orc_sim* s, orc_energy_sample* out, uint64_t cap);
void orc_energy(const orc_sim* s, double* e_energy, double* h_energy);

#ifdef __cplusplus
}
#endif
#endif
