// oems_oracle.cpp -- CPU oracle for the Yee FDTD hot path (TEST INFRASTRUCTURE).
//
// Only tests/, the smoke check and bench.py's CPU-baseline leg use this file;
// the product path never links it.  See oems_oracle.h for the reference
// files each part restates.  Build: oracle/Makefile (-O2 -ffp-contract=off).
#include "oems_oracle.h"

#include <algorithm>
#include <cmath>
#include <cstring>
#include <limits>
#include <vector>

#ifdef _OPENMP
#include <omp.h>
#endif

namespace {

// src/constants.rs:8-18
constexpr double kC0 = 299792458.0;
constexpr double kEps0 = 8.854187817e-12;
constexpr double kMu0 = 1.256637062e-6;
constexpr double kZ0 = 376.730313668;
constexpr double kPi = 3.14159265358979323846;

// src/geometry/mod.rs:242-255 (min positive spacing; 1.0 if fewer than 2 lines)
double min_delta(const double* l, int64_t n) {
  if (n < 2) return 1.0;
  double m = std::numeric_limits<double>::max();
  for (int64_t i = 0; i + 1 < n; ++i) {
    double d = l[i + 1] - l[i];
    if (d > 0.0 && d < m) m = d;
  }
  return m;
}

// src/fdtd/excitation.rs:150-200
double eval_excitation(int kind, const double* p, double amplitude, double t) {
  double v = 0.0;
  switch (kind) {
    case ORC_EXC_GAUSSIAN: {
      double arg = (t - p[0]) / p[1];
      v = std::exp(-arg * arg);
      break;
    }
    case ORC_EXC_SINUSOIDAL:
      v = std::sin(2.0 * kPi * p[0] * t);
      break;
    case ORC_EXC_GAUSSIAN_MODULATED: {
      double arg = (t - p[1]) / p[2];
      double env = std::exp(-arg * arg);
      double car = std::sin(2.0 * kPi * p[0] * t);
      v = env * car;
      break;
    }
    case ORC_EXC_DIRAC:
      v = std::fabs(t) < 1e-15 ? 1.0 : 0.0;
      break;
    case ORC_EXC_STEP:
      v = t >= 0.0 ? 1.0 : 0.0;
      break;
    default:
      v = 0.0;
  }
  return amplitude * v;
}

struct CpmlFace {
  int layers = 0;
  // per layer: b, c (standard Roden-Gedney a), 1/kappa for E and H positions
  std::vector<double> b_e, c_e, ik_e, b_h, c_h, ik_h;
};

template <typename T>
struct Sim {
  int64_t nx, ny, nz, n;
  double dt;
  double delta[3];
  int threads = 1;
  bool zline = false;  // z-line (SimdEngine) loop form of the H / E updates
  uint64_t timestep = 0;
  std::vector<T> E[3], H[3], ca[3], cb[3], da[3], db[3];

  struct Exc {
    int64_t i, j, k;
    int dir;
    bool soft;
    std::vector<T> samples;
  };
  std::vector<Exc> excs;

  struct Probe {
    std::vector<int> comp;
    std::vector<int64_t> q;   // linear index per term
    std::vector<double> w;    // weight per term
    int mode;                 // 0: f32 sum with +-1, 1: f64 weighted sum
    double half;              // time offset (0.5 for H-only probes)
  };
  std::vector<Probe> probes;
  std::vector<double> traces;  // [step][probe]

  struct ProbeDft {
    int probe;
    std::vector<double> freqs;
    std::vector<double> re, im;
  };
  std::vector<ProbeDft> dfts;

  // Frequency-domain field dump (src/processing/fields_fd.rs:31-217) over a
  // half-open region with sub-sampling; components in ascending order.
  // Accumulated when the timestep count is a multiple of `interval`, with
  // scale 2 dt interval.  acc: [freq][component][point] (re, im).
  struct FieldDft {
    int64_t r[6], ss[3], n[3], npts;
    std::vector<int> comps;
    uint64_t interval;
    std::vector<double> freqs, acc;
  };
  std::vector<FieldDft> fdumps;

  // NF2FF box: per enabled face (-x +x -y +y -z +z) at node plane p of axis
  // a, with b = a+1, c = a+2 (mod 3): Eb, Ec at plane p and Hb, Hc averaged
  // over planes p-1 and p, on the face's node grid (nb x nc, b-major).
  // acc: [face slot][freq][4][nb * nc] (re, im).
  struct Nf2ffBox {
    int64_t lo[3], hi[3];
    int dirs[6];
    uint64_t interval;
    std::vector<double> freqs;
    std::vector<int> faces;                 // enabled faces in order
    std::vector<std::vector<double>> acc;   // per enabled face
  };
  std::vector<Nf2ffBox> boxes;

  // Uniaxial PML as the reference (src/extensions/pml.rs:130-655): regions
  // with per-cell coefficients (vv vvfo vvfn for E, ii iifo iifn for H) and
  // flux arrays, applied before and after each field update.
  struct UpmlRegion {
    int64_t start[3], size[3];
    std::vector<T> cv[3][3], ci[3][3];  // [vv|vvfo|vvfn][component]
    std::vector<T> vflux[3], iflux[3];
  };
  std::vector<UpmlRegion> upml;

  void upml_hook(bool h, bool pre) {
    for (UpmlRegion& R : upml) {
      int64_t m = 0;
      for (int64_t li = 0; li < R.size[0]; ++li)
        for (int64_t lj = 0; lj < R.size[1]; ++lj)
          for (int64_t lk = 0; lk < R.size[2]; ++lk, ++m) {
            const int64_t q = idx(R.start[0] + li, R.start[1] + lj, R.start[2] + lk);
            for (int c = 0; c < 3; ++c) {
              std::vector<T>& F = h ? H[c] : E[c];
              std::vector<T>& fl = h ? R.iflux[c] : R.vflux[c];
              auto& co = h ? R.ci : R.cv;
              if (pre) {  // pml.rs:505-549 / 586-620
                const T f_help = co[0][c][m] * F[q] - co[1][c][m] * fl[m];
                F[q] = fl[m];
                fl[m] = f_help;
              } else {    // pml.rs:554-581 / 625-655
                const T f_help = fl[m];
                const T flux_new = F[q];
                fl[m] = flux_new;
                F[q] = f_help + co[2][c][m] * flux_new;
              }
            }
          }
    }
  }

  // Upml::calculate_kappa (pml.rs:370-420)
  void upml_kappa(int comp, int dir, const int64_t pos[3], bool is_min, int64_t layers, double width,
                  double smax, double m, double* kv, double* ki) const {
    const int64_t ext[3] = {nx, ny, nz};
    const double d = delta[dir];
    double depth = 0.0;
    if (is_min) {
      if (pos[dir] <= layers) depth = (double)(layers - pos[dir]) * d;
    } else {
      const int64_t bs = ext[dir] - layers - 1;
      if (pos[dir] >= bs) depth = (double)(pos[dir] - bs) * d;
    }
    if (depth <= 0.0) {
      *kv = 0.0;
      *ki = 0.0;
      return;
    }
    *kv = smax * std::pow(depth / width, m);
    const double di = depth + (comp == dir ? -0.5 : 0.5) * d;
    *ki = smax * std::pow(std::clamp(di / width, 0.0, 1.0), m);
  }

  // Conductivity of the corrected UPML (kind 1) along `dir` at cell index
  // i, at the node (half = false) or half a cell above it: the graded
  // sigma_max (depth / width)^m with the depth measured from the region's
  // inner node (L at a min face, n - L - 1 at a max face), as the reference
  // grades, but at the Yee position of the component.
  double upml_sigma(int dir, bool is_min, int64_t L, int64_t i, bool half, double smax, double m) const {
    const int64_t ext[3] = {nx, ny, nz};
    const double x = (double)i + (half ? 0.5 : 0.0);
    double depth = is_min ? (double)L - x : x - (double)(ext[dir] - L - 1);
    depth = std::clamp(depth, 0.0, (double)L);
    return smax * std::pow(depth / (double)L, m);
  }
  // Conductivity along `dir` at index i of every active face of that axis
  // (a cell lies in at most one of them): corners and edges of the PML are
  // graded along each axis whose slab they are in.
  double upml_sigma_axis(const int64_t* L, int dir, int64_t i, bool half, double m, double R0) const {
    const int64_t ext[3] = {nx, ny, nz};
    double sg = 0.0;
    for (int side = 0; side < 2; ++side) {
      const int64_t l = L[2 * dir + side];
      if (l <= 0 || l >= ext[dir]) continue;
      const double smax = -(m + 1.0) * std::log(R0) / (2.0 * kZ0 * (double)l * delta[dir]);
      sg = std::max(sg, upml_sigma(dir, side == 0, l, i, half, smax, m));
    }
    return sg;
  }

  // Upml::build_regions + init_region_coefficients (pml.rs:222-367).
  // kind 0: the reference's coefficients.  kind 1: the uniaxial PML of
  // Taflove & Hagness 7.8 in the same flux form: for component n (nP, nPP
  // the next two axes) the main update advances D with sigma_nP
  // (Ca = (2 eps0 - s_nP dt) / (2 eps0 + s_nP dt), Cb scaled by
  // 2 eps0 / (2 eps0 + s_nP dt)), and the hooks take E from D with
  // vv = (2 eps0 - s_nPP dt) / den, vvfo / vvfn = (2 eps0 -/+ s_n dt) / den,
  // den = 2 eps0 + s_nPP dt.  Every cell of the regions is graded along
  // each axis whose slab holds it (so edges and corners absorb along all
  // of them), at the Yee position of each component; a zero conductivity
  // gives vv = vvfo = vvfn = 1 (E follows D).  The reference instead grades
  // only the region's own axis and puts that value in every axis slot,
  // writes vvfo = 0 where nothing is graded and leaves the main update
  // unchanged, which grows without bound.
  int enable_upml(const int64_t* L, double m, double R0, int kind = 0) {
    const int64_t ext[3] = {nx, ny, nz};
    struct Box {
      int64_t s[3], z[3];
      int dir;
      bool mn;
    };
    std::vector<Box> bx;
    if (L[0] > 0 && L[0] < nx) bx.push_back({{0, 0, 0}, {L[0] + 1, ny, nz}, 0, true});
    if (L[1] > 0 && L[1] < nx) bx.push_back({{nx - L[1] - 1, 0, 0}, {L[1] + 1, ny, nz}, 0, false});
    const int64_t xs = L[0] > 0 ? L[0] + 1 : 0, xe = L[1] > 0 ? nx - L[1] - 1 : nx;
    if (L[2] > 0 && L[2] < ny && xs < xe) bx.push_back({{xs, 0, 0}, {xe - xs, L[2] + 1, nz}, 1, true});
    if (L[3] > 0 && L[3] < ny && xs < xe) bx.push_back({{xs, ny - L[3] - 1, 0}, {xe - xs, L[3] + 1, nz}, 1, false});
    const int64_t ys = L[2] > 0 ? L[2] + 1 : 0, ye = L[3] > 0 ? ny - L[3] - 1 : ny;
    if (L[4] > 0 && L[4] < nz && xs < xe && ys < ye)
      bx.push_back({{xs, ys, 0}, {xe - xs, ye - ys, L[4] + 1}, 2, true});
    if (L[5] > 0 && L[5] < nz && xs < xe && ys < ye)
      bx.push_back({{xs, ys, nz - L[5] - 1}, {xe - xs, ye - ys, L[5] + 1}, 2, false});
    (void)ext;
    upml.clear();
    for (const Box& b : bx) {
      UpmlRegion Rg;
      const int64_t layers = L[2 * b.dir + (b.mn ? 0 : 1)];
      const double width = (double)layers * delta[b.dir];
      const double smax = -(m + 1.0) * std::log(R0) / (2.0 * kZ0 * width);
      const int64_t cnt = b.z[0] * b.z[1] * b.z[2];
      for (int a = 0; a < 3; ++a) {
        Rg.start[a] = b.s[a];
        Rg.size[a] = b.z[a];
        Rg.vflux[a].assign(cnt, T(0));
        Rg.iflux[a].assign(cnt, T(0));
        for (int k = 0; k < 3; ++k) {
          Rg.cv[k][a].assign(cnt, T(0));
          Rg.ci[k][a].assign(cnt, T(0));
        }
      }
      int64_t t = 0;
      for (int64_t li = 0; li < b.z[0]; ++li)
        for (int64_t lj = 0; lj < b.z[1]; ++lj)
          for (int64_t lk = 0; lk < b.z[2]; ++lk, ++t) {
            const int64_t pos[3] = {b.s[0] + li, b.s[1] + lj, b.s[2] + lk};
            if (kind == 1) {
              const int64_t q = idx(pos[0], pos[1], pos[2]);
              for (int c = 0; c < 3; ++c) {
                // E_c sits half a cell up its own axis, H_c along the others
                double sv[3], si[3];
                for (int d = 0; d < 3; ++d) {
                  sv[d] = upml_sigma_axis(L, d, pos[d], c == d, m, R0);
                  si[d] = upml_sigma_axis(L, d, pos[d], c != d, m, R0);
                }
                const int np = (c + 1) % 3, npp = (c + 2) % 3;
                const double dv = 2.0 * kEps0 + sv[npp] * dt, di = 2.0 * kEps0 + si[npp] * dt;
                Rg.cv[0][c][t] = T((2.0 * kEps0 - sv[npp] * dt) / dv);
                Rg.cv[1][c][t] = T((2.0 * kEps0 - sv[c] * dt) / dv);
                Rg.cv[2][c][t] = T((2.0 * kEps0 + sv[c] * dt) / dv);
                Rg.ci[0][c][t] = T((2.0 * kEps0 - si[npp] * dt) / di);
                Rg.ci[1][c][t] = T((2.0 * kEps0 - si[c] * dt) / di);
                Rg.ci[2][c][t] = T((2.0 * kEps0 + si[c] * dt) / di);
                if (ca[c][q] != T(0) || cb[c][q] != T(0)) {
                  ca[c][q] = T((2.0 * kEps0 - sv[np] * dt) / (2.0 * kEps0 + sv[np] * dt));
                  cb[c][q] = T((double)cb[c][q] * (2.0 * kEps0 / (2.0 * kEps0 + sv[np] * dt)));
                }
                if (da[c][q] != T(0) || db[c][q] != T(0)) {
                  da[c][q] = T((2.0 * kEps0 - si[np] * dt) / (2.0 * kEps0 + si[np] * dt));
                  db[c][q] = T((double)db[c][q] * (2.0 * kEps0 / (2.0 * kEps0 + si[np] * dt)));
                }
              }
              continue;
            }
            double kv[3], ki[3];
            for (int c = 0; c < 3; ++c) upml_kappa(c, b.dir, pos, b.mn, layers, width, smax, m, &kv[c], &ki[c]);
            for (int c = 0; c < 3; ++c) {
              const int npp = (c + 2) % 3;
              if (kv[0] + kv[1] + kv[2] > 0.0) {
                const double den = 2.0 * kEps0 + kv[npp] * dt;
                Rg.cv[0][c][t] = T((2.0 * kEps0 - kv[npp] * dt) / den);
                Rg.cv[1][c][t] = T((2.0 * kEps0 - kv[c] * dt) / den);
                Rg.cv[2][c][t] = T((2.0 * kEps0 + kv[c] * dt) / den);
              } else {
                Rg.cv[0][c][t] = T(1);
                Rg.cv[1][c][t] = T(0);
                Rg.cv[2][c][t] = T(1);
              }
              if (ki[0] + ki[1] + ki[2] > 0.0) {
                const double den = 2.0 * kEps0 + ki[npp] * dt;
                Rg.ci[0][c][t] = T((2.0 * kEps0 - ki[npp] * dt) / den);
                Rg.ci[1][c][t] = T((2.0 * kEps0 - ki[c] * dt) / den);
                Rg.ci[2][c][t] = T((2.0 * kEps0 + ki[c] * dt) / den);
              } else {
                Rg.ci[0][c][t] = T(1);
                Rg.ci[1][c][t] = T(0);
                Rg.ci[2][c][t] = T(1);
              }
            }
          }
      upml.push_back(std::move(Rg));
    }
    return (int)upml.size();
  }

  std::vector<orc_energy_sample> energy;

  // CPML state
  bool cpml = false;
  CpmlFace face[6];
  // per axis, per index: side (-1 none, 0 min, 1 max) and layer
  std::vector<int> side[3], layer[3];
  // psi arrays, full size (only slab cells used): H: hx_y hx_z hy_z hy_x hz_x hz_y
  // E: ex_y ex_z ey_z ey_x ez_x ez_y
  std::vector<T> psi_h[6], psi_e[6];

  // Mur state (src/extensions/mur_abc.rs:60-131): per face the normal axis,
  // its two tangential axes, boundary and shift lines, face size and the
  // pending boundary values; second order also keeps the time-n-1 values of
  // both lines.
  struct MurFace {
    int ny, nyp, nypp;
    int64_t line, shift;
    int64_t size0, size1;
    int64_t lo0, lo1;               // second order: first live row / column of the face
    T coeff;                        // (c dt - d) / (c dt + d)
    T c2, c3p, c3q;                 // second order
    std::vector<T> v[2];            // pending values for nyp, nypp
    std::vector<T> ob[2], os[2];    // boundary / shift line at n-1 (second order)
  };
  std::vector<MurFace> mur;
  int mur_order = 0;

  // dispersive materials (src/extensions/dispersive.rs:75-96: coefficients
  // a, b, c per material, state per cell and component)
  struct Dispersive {
    int kind;
    float a, b, c, c2;          // as computed by the reference constructors, f32
    std::vector<int64_t> q;     // cells
    std::vector<T> j[3], pp[3]; // state (J or P) and P at n-1 (second-order kinds)
    std::vector<T> ep[3];       // E^n, taken before the E update (second-order kinds)
  };
  std::vector<Dispersive> disp;

  // LumpedRlc elements (src/extensions/lumped_rlc.rs:118-139)
  struct Rlc {
    int64_t q;
    int dir;
    float v_vv, v_il;
    T i_int;
  };
  std::vector<Rlc> rlc;

  // src/extensions/dispersive.rs:171-196, 510-535, 604-630 (+ second-order Lorentz)
  // E^n of the second-order kinds, before the E update
  void capture_dispersive() {
    for (Dispersive& D : disp) {
      if (D.kind < 3) continue;
      for (size_t m = 0; m < D.q.size(); ++m)
        for (int c = 0; c < 3; ++c) D.ep[c][m] = E[c][D.q[m]];
    }
  }

  void apply_dispersive() {
    const float dtf = (float)dt;
    for (Dispersive& D : disp) {
      for (size_t m = 0; m < D.q.size(); ++m)
        for (int c = 0; c < 3; ++c) {
          T& ef = E[c][D.q[m]];
          const T e = ef;
          const T old = D.j[c][m];
          if (D.kind == 0) {  // Drude: j = a j + b e; e -= c j
            const T jn = T(D.a) * old + T(D.b) * e;
            D.j[c][m] = jn;
            ef = e - T(D.c) * jn;
          } else if (D.kind == 1) {  // Lorentz as the reference: j = a j + c e; e -= b j
            const T jn = T(D.a) * old + T(D.c) * e;
            D.j[c][m] = jn;
            ef = e - T(D.b) * jn;
          } else if (D.kind == 2) {  // Debye: p' = a p + b e; e -= c (p' - p) / dt
            const T pn = T(D.a) * old + T(D.b) * e;
            D.j[c][m] = pn;
            const T dpdt = (pn - old) / T(dtf);
            ef = e - T(D.c) * dpdt;
          } else {  // second-order P recursion (Lorentz, kind 3; Drude, kind 4) driven by E^n
            const T t1 = T(D.a) * old;
            const T t2 = T(D.b) * D.pp[c][m];
            const T t3 = T(D.c) * D.ep[c][m];
            const T pn = (t1 + t2) + t3;
            D.pp[c][m] = old;
            D.j[c][m] = pn;
            ef = e - T(D.c2) * (pn - old);
          }
        }
    }
  }

  // src/extensions/lumped_rlc.rs:263-286
  void apply_rlc() {
    const T dtf = T((float)dt);
    for (Rlc& r : rlc) {
      T& ef = E[r.dir][r.q];
      const T e = ef;
      const T en = T(r.v_vv) * e + T(r.v_il) * r.i_int;
      r.i_int = r.i_int + e * dtf;
      ef = en;
    }
  }

  Sim(int64_t nx_, int64_t ny_, int64_t nz_, double dt_, double dx, double dy, double dz)
      : nx(nx_), ny(ny_), nz(nz_), n(nx_ * ny_ * nz_), dt(dt_) {
    delta[0] = dx;
    delta[1] = dy;
    delta[2] = dz;
    for (int c = 0; c < 3; ++c) {
      E[c].assign(n, T(0));
      H[c].assign(n, T(0));
    }
    init_vacuum();
  }

  int64_t idx(int64_t i, int64_t j, int64_t k) const { return (i * ny + j) * nz + k; }

  // src/fdtd/operator.rs:92-141
  void init_vacuum() {
    for (int c = 0; c < 3; ++c) {
      ca[c].assign(n, T(1));
      da[c].assign(n, T(1));
    }
    T cbv[3] = {T(dt / (kEps0 * delta[0])), T(dt / (kEps0 * delta[1])), T(dt / (kEps0 * delta[2]))};
    T dbv[3] = {T(-(dt / (kMu0 * delta[0]))), T(-(dt / (kMu0 * delta[1]))),
                T(-(dt / (kMu0 * delta[2])))};
    for (int c = 0; c < 3; ++c) {
      cb[c].assign(n, cbv[c]);
      db[c].assign(n, dbv[c]);
    }
  }

  // src/fdtd/operator.rs:187-244
  void set_material(double eps_r, double mu_r, double sigma_e, double sigma_m, const int64_t* r) {
    double eps = eps_r * kEps0;
    double loss_e = sigma_e * dt / (2.0 * eps);
    T ca_mat = T((1.0 - loss_e) / (1.0 + loss_e));
    double cb_factor = (dt / eps) / (1.0 + loss_e);
    T cbv[3] = {T(cb_factor / delta[0]), T(cb_factor / delta[1]), T(cb_factor / delta[2])};
    double mu = mu_r * kMu0;
    double loss_m = sigma_m * dt / (2.0 * mu);
    T da_mat = T((1.0 - loss_m) / (1.0 + loss_m));
    double db_factor = -(dt / mu) / (1.0 + loss_m);
    T dbv[3] = {T(db_factor / delta[0]), T(db_factor / delta[1]), T(db_factor / delta[2])};
    for (int64_t i = r[0]; i < r[1]; ++i)
      for (int64_t j = r[2]; j < r[3]; ++j)
        for (int64_t k = r[4]; k < r[5]; ++k) {
          int64_t q = idx(i, j, k);
          for (int c = 0; c < 3; ++c) {
            ca[c][q] = ca_mat;
            cb[c][q] = cbv[c];
            da[c][q] = da_mat;
            db[c][q] = dbv[c];
          }
        }
  }

  // src/fdtd/operator.rs:249-263
  void set_pec(const int64_t* r) {
    for (int64_t i = r[0]; i < r[1]; ++i)
      for (int64_t j = r[2]; j < r[3]; ++j)
        for (int64_t k = r[4]; k < r[5]; ++k) {
          int64_t q = idx(i, j, k);
          for (int c = 0; c < 3; ++c) {
            ca[c][q] = T(0);
            cb[c][q] = T(0);
          }
        }
  }

  // Profile: src/extensions/cpml.rs:68-72 (sigma_max from the largest layer
  // count and the smallest cell size) and :98-177 (per-layer b and a).
  int enable_cpml(const int32_t* layers6, double m, double R, double alpha_max, double kappa_max) {
    int lmax = 0;
    for (int f = 0; f < 6; ++f) lmax = std::max(lmax, (int)layers6[f]);
    if (lmax <= 0) return -1;
    double dmin = std::min(delta[0], std::min(delta[1], delta[2]));
    double d = (double)lmax * dmin;
    double sigma_max = -(m + 1.0) * std::log(R) / (2.0 * kZ0 * d);
    int64_t ext[3] = {nx, ny, nz};
    for (int a = 0; a < 3; ++a) {
      side[a].assign(ext[a], -1);
      layer[a].assign(ext[a], 0);
      int lmin_ = layers6[2 * a], lmax_ = layers6[2 * a + 1];
      bool use_min = lmin_ > 0 && lmin_ < ext[a];
      bool use_max = lmax_ > 0 && lmax_ < ext[a];
      if ((use_min ? lmin_ : 0) + (use_max ? lmax_ : 0) > ext[a]) return -2;
      for (int s = 0; s < 2; ++s) {
        int L = s == 0 ? lmin_ : lmax_;
        bool use = s == 0 ? use_min : use_max;
        CpmlFace& F = face[2 * a + s];
        F.layers = use ? L : 0;
        if (!use) continue;
        double width = (double)L * delta[a];
        F.b_e.resize(L);
        F.c_e.resize(L);
        F.ik_e.resize(L);
        F.b_h.resize(L);
        F.c_h.resize(L);
        F.ik_h.resize(L);
        for (int l = 0; l < L; ++l) {
          // grading of src/extensions/cpml.rs:114-155 at the positions of
          // the differences (min face: E (L - l) d, H half a cell shallower;
          // max face: E l d, H half a cell deeper); the reference's max-face
          // depths ((l + 1) d and (l + 1/2) d) mismatch E and H by a cell
          double depth_e = s == 0 ? (double)(L - l) * delta[a] : (double)l * delta[a];
          double depth_h = s == 0 ? depth_e - 0.5 * delta[a] : depth_e + 0.5 * delta[a];
          for (int w = 0; w < 2; ++w) {
            double depth = w == 0 ? depth_e : depth_h;
            double rho = std::min(1.0, std::max(0.0, depth / width));
            double sigma = sigma_max * std::pow(rho, m);
            double alpha = alpha_max * (1.0 - rho);
            double kappa = 1.0 + (kappa_max - 1.0) * std::pow(rho, m);
            double b = std::exp(-(sigma / kappa / kEps0 + alpha / kEps0) * dt);
            double sn = sigma / (kEps0 * kappa);
            double an = alpha / kEps0;
            double den = sn + an;
            double a_ref = std::fabs(den) > 1e-20 ? sn / den * (1.0 - b) : 0.0;
            // Standard Roden-Gedney a = sigma/(sigma*kappa + kappa^2*alpha)*(b-1),
            // which equals -a_ref/kappa.
            double c = -a_ref / kappa;
            double ik = 1.0 / kappa;
            // round to the sim precision so the profile matches the kernels
            if (w == 0) {
              F.b_e[l] = (double)T(b);
              F.c_e[l] = (double)T(c);
              F.ik_e[l] = (double)T(ik);
            } else {
              F.b_h[l] = (double)T(b);
              F.c_h[l] = (double)T(c);
              F.ik_h[l] = (double)T(ik);
            }
          }
        }
        for (int l = 0; l < L; ++l) {
          int64_t g = s == 0 ? l : ext[a] - L + l;
          side[a][g] = s;
          layer[a][g] = l;
        }
      }
    }
    for (int q = 0; q < 6; ++q) {
      psi_h[q].assign(n, T(0));
      psi_e[q].assign(n, T(0));
    }
    cpml = true;
    return 0;
  }

  // psi <- b*psi + c*d ; d <- d*ik + psi   (each product and sum rounded)
  static inline T stretch(T d, T& psi, T b, T c, T ik) {
    T t1 = b * psi;
    T t2 = c * d;
    psi = t1 + t2;
    T t3 = d * ik;
    return t3 + psi;
  }

  inline void cpml_h(int axis, int64_t g, int64_t q, T& d, int which) {
    int s = side[axis][g];
    if (s < 0) return;
    const CpmlFace& F = face[2 * axis + s];
    int l = layer[axis][g];
    d = stretch(d, psi_h[which][q], T(F.b_h[l]), T(F.c_h[l]), T(F.ik_h[l]));
  }
  inline void cpml_e(int axis, int64_t g, int64_t q, T& d, int which) {
    int s = side[axis][g];
    if (s < 0) return;
    const CpmlFace& F = face[2 * axis + s];
    int l = layer[axis][g];
    d = stretch(d, psi_e[which][q], T(F.b_e[l]), T(F.c_e[l]), T(F.ik_e[l]));
  }

  // CPML stretch of one z-line of differences d[k0, k1) with the profile of
  // one layer (x / y slabs: the whole line shares the layer).
  static void stretch_line(T* d, T* psi, int64_t k0, int64_t k1, T b, T c, T ik) {
    for (int64_t k = k0; k < k1; ++k) d[k] = stretch(d[k], psi[k], b, c, ik);
  }
  // z slabs of one line: each k has its own layer.
  void stretch_zslabs(T* d, T* psi, bool is_h) const {
    for (int s = 0; s < 2; ++s) {
      const CpmlFace& F = face[4 + s];
      if (F.layers <= 0) continue;
      const int64_t k0 = s == 0 ? 0 : nz - F.layers, k1 = s == 0 ? F.layers : nz;
      for (int64_t k = k0; k < k1; ++k) {
        const int l = layer[2][k];
        d[k] = is_h ? stretch(d[k], psi[k], T(F.b_h[l]), T(F.c_h[l]), T(F.ik_h[l]))
                    : stretch(d[k], psi[k], T(F.b_e[l]), T(F.c_e[l]), T(F.ik_e[l]));
      }
    }
  }
  void stretch_row(int axis, int64_t g, T* d, T* psi, bool is_h) const {
    const int s = side[axis][g];
    if (s < 0) return;
    const CpmlFace& F = face[2 * axis + s];
    const int l = layer[axis][g];
    if (is_h)
      stretch_line(d, psi, 0, nz, T(F.b_h[l]), T(F.c_h[l]), T(F.ik_h[l]));
    else
      stretch_line(d, psi, 0, nz, T(F.b_e[l]), T(F.c_e[l]), T(F.ik_e[l]));
  }

  // The same H update in the loop form of the reference's SimdEngine
  // (src/fdtd/simd_engine.rs:252-331): per (i, j) z-line, the differences are
  // formed in contiguous row buffers (a missing neighbour line gives 0, the
  // last k of a z difference is 0), CPML stretches the slab parts of those
  // rows, then one loop per component updates the line.  Every value goes
  // through the same rounded operations as update_h, so the results are
  // bit-identical; only the loop order differs, which lets the compiler
  // vectorise the k loops.  OpenMP over x-planes as the parallel engine.
  void update_h_zline() {
    const T* ex = E[0].data();
    const T* ey = E[1].data();
    const T* ez = E[2].data();
#pragma omp parallel num_threads(threads) if (threads > 1)
    {
      std::vector<T> buf(6 * nz);
      T* dzy = buf.data();
      T* dyz = dzy + nz;
      T* dxz = dyz + nz;
      T* dzx = dxz + nz;
      T* dyx = dzx + nz;
      T* dxy = dyx + nz;
#pragma omp for schedule(static)
      for (int64_t i = 0; i < nx; ++i)
        for (int64_t j = 0; j < ny; ++j) {
          const int64_t q = idx(i, j, 0);
          const T* exl = ex + q;
          const T* eyl = ey + q;
          const T* ezl = ez + q;
          if (j + 1 < ny) {
            for (int64_t k = 0; k < nz; ++k) dzy[k] = ezl[k + nz] - ezl[k];
            for (int64_t k = 0; k < nz; ++k) dxy[k] = exl[k + nz] - exl[k];
          } else {
            for (int64_t k = 0; k < nz; ++k) dzy[k] = dxy[k] = T(0);
          }
          for (int64_t k = 0; k + 1 < nz; ++k) dyz[k] = eyl[k + 1] - eyl[k];
          for (int64_t k = 0; k + 1 < nz; ++k) dxz[k] = exl[k + 1] - exl[k];
          dyz[nz - 1] = dxz[nz - 1] = T(0);
          if (i + 1 < nx) {
            const int64_t P = ny * nz;
            for (int64_t k = 0; k < nz; ++k) dzx[k] = ezl[k + P] - ezl[k];
            for (int64_t k = 0; k < nz; ++k) dyx[k] = eyl[k + P] - eyl[k];
          } else {
            for (int64_t k = 0; k < nz; ++k) dzx[k] = dyx[k] = T(0);
          }
          if (cpml) {
            stretch_row(1, j, dzy, psi_h[0].data() + q, true);
            stretch_zslabs(dyz, psi_h[1].data() + q, true);
            stretch_zslabs(dxz, psi_h[2].data() + q, true);
            stretch_row(0, i, dzx, psi_h[3].data() + q, true);
            stretch_row(0, i, dyx, psi_h[4].data() + q, true);
            stretch_row(1, j, dxy, psi_h[5].data() + q, true);
          }
          line_update(H[0].data() + q, da[0].data() + q, db[0].data() + q, dzy, dyz, 0);
          line_update(H[1].data() + q, da[1].data() + q, db[1].data() + q, dxz, dzx, 0);
          line_update(H[2].data() + q, da[2].data() + q, db[2].data() + q, dyx, dxy, 0);
        }
    }
  }

  // f[k] = a[k] * f[k] + b[k] * (d1[k] - d2[k]) for k in [k0, nz), each
  // product and sum rounded.
  void line_update(T* __restrict f, const T* __restrict a, const T* __restrict b, const T* __restrict d1,
                   const T* __restrict d2, int64_t k0) const {
    for (int64_t k = k0; k < nz; ++k) {
      const T curl = d1[k] - d2[k];
      const T t0 = a[k] * f[k];
      const T t1 = b[k] * curl;
      f[k] = t0 + t1;
    }
  }

  // E update in the SimdEngine loop form (src/fdtd/simd_engine.rs:339-391):
  // lines with i, j >= 1, elements k >= 1; bit-identical to update_e.
  void update_e_zline() {
    const T* hx = H[0].data();
    const T* hy = H[1].data();
    const T* hz = H[2].data();
#pragma omp parallel num_threads(threads) if (threads > 1)
    {
      std::vector<T> buf(6 * nz);
      T* dzy = buf.data();
      T* dyz = dzy + nz;
      T* dxz = dyz + nz;
      T* dzx = dxz + nz;
      T* dyx = dzx + nz;
      T* dxy = dyx + nz;
      const int64_t P = ny * nz;
#pragma omp for schedule(static)
      for (int64_t i = 1; i < nx; ++i)
        for (int64_t j = 1; j < ny; ++j) {
          const int64_t q = idx(i, j, 0);
          const T* hxl = hx + q;
          const T* hyl = hy + q;
          const T* hzl = hz + q;
          for (int64_t k = 1; k < nz; ++k) dzy[k] = hzl[k] - hzl[k - nz];
          for (int64_t k = 1; k < nz; ++k) dyz[k] = hyl[k] - hyl[k - 1];
          for (int64_t k = 1; k < nz; ++k) dxz[k] = hxl[k] - hxl[k - 1];
          for (int64_t k = 1; k < nz; ++k) dzx[k] = hzl[k] - hzl[k - P];
          for (int64_t k = 1; k < nz; ++k) dyx[k] = hyl[k] - hyl[k - P];
          for (int64_t k = 1; k < nz; ++k) dxy[k] = hxl[k] - hxl[k - nz];
          dzy[0] = dyz[0] = dxz[0] = dzx[0] = dyx[0] = dxy[0] = T(0);
          if (cpml) {
            // element k = 0 is never written, so stretching it (with its
            // psi, which stays untouched at 0 -> b*0 + c*0) is harmless only
            // if it does not change psi: skip it by starting at k = 1.
            stretch_row_from1(1, j, dzy, psi_e[0].data() + q, false);
            stretch_zslabs_from1(dyz, psi_e[1].data() + q);
            stretch_zslabs_from1(dxz, psi_e[2].data() + q);
            stretch_row_from1(0, i, dzx, psi_e[3].data() + q, false);
            stretch_row_from1(0, i, dyx, psi_e[4].data() + q, false);
            stretch_row_from1(1, j, dxy, psi_e[5].data() + q, false);
          }
          line_update(E[0].data() + q, ca[0].data() + q, cb[0].data() + q, dzy, dyz, 1);
          line_update(E[1].data() + q, ca[1].data() + q, cb[1].data() + q, dxz, dzx, 1);
          line_update(E[2].data() + q, ca[2].data() + q, cb[2].data() + q, dyx, dxy, 1);
        }
    }
  }
  void stretch_row_from1(int axis, int64_t g, T* d, T* psi, bool is_h) const {
    const int s = side[axis][g];
    if (s < 0) return;
    const CpmlFace& F = face[2 * axis + s];
    const int l = layer[axis][g];
    if (is_h)
      stretch_line(d, psi, 1, nz, T(F.b_h[l]), T(F.c_h[l]), T(F.ik_h[l]));
    else
      stretch_line(d, psi, 1, nz, T(F.b_e[l]), T(F.c_e[l]), T(F.ik_e[l]));
  }
  void stretch_zslabs_from1(T* d, T* psi) const {
    for (int s = 0; s < 2; ++s) {
      const CpmlFace& F = face[4 + s];
      if (F.layers <= 0) continue;
      const int64_t k0 = s == 0 ? 1 : nz - F.layers, k1 = s == 0 ? F.layers : nz;
      for (int64_t k = std::max<int64_t>(k0, 1); k < k1; ++k) {
        const int l = layer[2][k];
        d[k] = stretch(d[k], psi[k], T(F.b_e[l]), T(F.c_e[l]), T(F.ik_e[l]));
      }
    }
  }

  // src/fdtd/basic_engine.rs:191-254
  void update_h() {
    if (zline) {
      update_h_zline();
      return;
    }
    const T* ex = E[0].data();
    const T* ey = E[1].data();
    const T* ez = E[2].data();
#pragma omp parallel for num_threads(threads) if (threads > 1) schedule(static)
    for (int64_t i = 0; i < nx; ++i)
      for (int64_t j = 0; j < ny; ++j)
        for (int64_t k = 0; k < nz; ++k) {
          int64_t q = idx(i, j, k);
          T dez_dy = j + 1 < ny ? ez[q + nz] - ez[q] : T(0);
          T dey_dz = k + 1 < nz ? ey[q + 1] - ey[q] : T(0);
          T dex_dz = k + 1 < nz ? ex[q + 1] - ex[q] : T(0);
          T dez_dx = i + 1 < nx ? ez[q + ny * nz] - ez[q] : T(0);
          T dey_dx = i + 1 < nx ? ey[q + ny * nz] - ey[q] : T(0);
          T dex_dy = j + 1 < ny ? ex[q + nz] - ex[q] : T(0);
          if (cpml) {
            cpml_h(1, j, q, dez_dy, 0);  // Hx, y-slab
            cpml_h(2, k, q, dey_dz, 1);  // Hx, z-slab
            cpml_h(2, k, q, dex_dz, 2);  // Hy, z-slab
            cpml_h(0, i, q, dez_dx, 3);  // Hy, x-slab
            cpml_h(0, i, q, dey_dx, 4);  // Hz, x-slab
            cpml_h(1, j, q, dex_dy, 5);  // Hz, y-slab
          }
          T curl_x = dez_dy - dey_dz;
          T curl_y = dex_dz - dez_dx;
          T curl_z = dey_dx - dex_dy;
          T a0 = da[0][q] * H[0][q];
          T b0 = db[0][q] * curl_x;
          H[0][q] = a0 + b0;
          T a1 = da[1][q] * H[1][q];
          T b1 = db[1][q] * curl_y;
          H[1][q] = a1 + b1;
          T a2 = da[2][q] * H[2][q];
          T b2 = db[2][q] * curl_z;
          H[2][q] = a2 + b2;
        }
  }

  // src/fdtd/basic_engine.rs:262-306 (only i, j, k >= 1 are updated)
  void update_e() {
    if (zline) {
      update_e_zline();
      return;
    }
    const T* hx = H[0].data();
    const T* hy = H[1].data();
    const T* hz = H[2].data();
#pragma omp parallel for num_threads(threads) if (threads > 1) schedule(static)
    for (int64_t i = 1; i < nx; ++i)
      for (int64_t j = 1; j < ny; ++j)
        for (int64_t k = 1; k < nz; ++k) {
          int64_t q = idx(i, j, k);
          T dhz_dy = hz[q] - hz[q - nz];
          T dhy_dz = hy[q] - hy[q - 1];
          T dhx_dz = hx[q] - hx[q - 1];
          T dhz_dx = hz[q] - hz[q - ny * nz];
          T dhy_dx = hy[q] - hy[q - ny * nz];
          T dhx_dy = hx[q] - hx[q - nz];
          if (cpml) {
            cpml_e(1, j, q, dhz_dy, 0);  // Ex, y-slab
            cpml_e(2, k, q, dhy_dz, 1);  // Ex, z-slab
            cpml_e(2, k, q, dhx_dz, 2);  // Ey, z-slab
            cpml_e(0, i, q, dhz_dx, 3);  // Ey, x-slab
            cpml_e(0, i, q, dhy_dx, 4);  // Ez, x-slab
            cpml_e(1, j, q, dhx_dy, 5);  // Ez, y-slab
          }
          T curl_x = dhz_dy - dhy_dz;
          T curl_y = dhx_dz - dhz_dx;
          T curl_z = dhy_dx - dhx_dy;
          T a0 = ca[0][q] * E[0][q];
          T b0 = cb[0][q] * curl_x;
          E[0][q] = a0 + b0;
          T a1 = ca[1][q] * E[1][q];
          T b1 = cb[1][q] * curl_y;
          E[1][q] = a1 + b1;
          T a2 = ca[2][q] * E[2][q];
          T b2 = cb[2][q] * curl_z;
          E[2][q] = a2 + b2;
        }
  }

  // src/fdtd/basic_engine.rs:313-395 (samples beyond the vector are skipped)
  void apply_excitations(uint64_t step) {
    for (const Exc& x : excs) {
      if (step >= x.samples.size()) continue;
      T v = x.samples[step];
      int64_t q = idx(x.i, x.j, x.k);
      if (x.soft)
        E[x.dir][q] += v;
      else
        E[x.dir][q] = v;
    }
  }

  T field_value(int comp, int64_t q) const { return comp < 3 ? E[comp][q] : H[comp - 3][q]; }

  // probe values after the step; DFT accumulation at t = (timestep - half) dt
  // where `timestep` already counts this step (src/processing/fields_fd.rs:149-217)
  void record_probes(uint64_t t_after) {
    const size_t base = traces.size();
    for (const Probe& p : probes) {
      double val;
      if (p.mode == 0) {
        float acc = 0.0f;
        for (size_t t = 0; t < p.q.size(); ++t) {
          const float v = (float)field_value(p.comp[t], p.q[t]);
          acc = p.w[t] >= 0.0 ? acc + v : acc - v;
        }
        val = (double)acc;
      } else {
        double acc = 0.0;
        for (size_t t = 0; t < p.q.size(); ++t) acc += p.w[t] * (double)field_value(p.comp[t], p.q[t]);
        val = acc;
      }
      traces.push_back(val);
    }
    for (ProbeDft& d : dfts) {
      const double x = traces[base + d.probe];
      const double t = ((double)t_after - probes[d.probe].half) * dt;
      const double scale = 2.0 * dt;
      for (size_t f = 0; f < d.freqs.size(); ++f) {
        // factor = exp(-j 2 pi f t) * 2 dt, then acc += x * factor
        const double ph = -2.0 * kPi * d.freqs[f] * t;
        const double fr = std::cos(ph) * scale, fi = std::sin(ph) * scale;
        d.re[f] += x * fr;
        d.im[f] += x * fi;
      }
    }
  }

  // twiddle of one sample: exp(-j 2 pi f t) * scale (fields_fd.rs:163-167)
  static void twiddle(double f, double t, double scale, double* re, double* im) {
    const double ph = -2.0 * kPi * f * t;
    *re = std::cos(ph) * scale;
    *im = std::sin(ph) * scale;
  }

  void record_fd(uint64_t t_after) {
    for (FieldDft& d : fdumps) {
      if (t_after % d.interval != 0) continue;
      const double scale = 2.0 * dt * (double)d.interval;
      const size_t nc = d.comps.size();
      for (size_t f = 0; f < d.freqs.size(); ++f) {
        double tw[2][2];
        twiddle(d.freqs[f], (double)t_after * dt, scale, &tw[0][0], &tw[0][1]);
        twiddle(d.freqs[f], ((double)t_after - 0.5) * dt, scale, &tw[1][0], &tw[1][1]);
        for (size_t ci = 0; ci < nc; ++ci) {
          const int comp = d.comps[ci];
          const double* w = tw[comp >= 3 ? 1 : 0];
          double* acc = d.acc.data() + 2 * (f * nc + ci) * (size_t)d.npts;
          int64_t p = 0;
          for (int64_t a = 0; a < d.n[0]; ++a)
            for (int64_t b = 0; b < d.n[1]; ++b)
              for (int64_t c = 0; c < d.n[2]; ++c, ++p) {
                const double x = (double)field_value(
                    comp, idx(d.r[0] + a * d.ss[0], d.r[2] + b * d.ss[1], d.r[4] + c * d.ss[2]));
                acc[2 * p] = acc[2 * p] + x * w[0];
                acc[2 * p + 1] = acc[2 * p + 1] + x * w[1];
              }
        }
      }
    }
    for (Nf2ffBox& B : boxes) {
      if (t_after % B.interval != 0) continue;
      const double scale = 2.0 * dt * (double)B.interval;
      for (size_t fs = 0; fs < B.faces.size(); ++fs) {
        const int face = B.faces[fs], a = face / 2, b = (a + 1) % 3, c = (a + 2) % 3;
        const int64_t p = (face & 1) ? B.hi[a] : B.lo[a];
        const int64_t nb = B.hi[b] - B.lo[b] + 1, ncc = B.hi[c] - B.lo[c] + 1, np = nb * ncc;
        for (size_t f = 0; f < B.freqs.size(); ++f) {
          double te[2], th[2];
          twiddle(B.freqs[f], (double)t_after * dt, scale, &te[0], &te[1]);
          twiddle(B.freqs[f], ((double)t_after - 0.5) * dt, scale, &th[0], &th[1]);
          double* acc = B.acc[fs].data() + f * 8 * (size_t)np;
          for (int64_t jb = 0; jb < nb; ++jb)
            for (int64_t kc = 0; kc < ncc; ++kc) {
              int64_t pos[3];
              pos[a] = p;
              pos[b] = B.lo[b] + jb;
              pos[c] = B.lo[c] + kc;
              const int64_t q = idx(pos[0], pos[1], pos[2]);
              pos[a] = p - 1;
              const int64_t qm = idx(pos[0], pos[1], pos[2]);
              const double v[4] = {(double)E[b][q], (double)E[c][q],
                                   0.5 * ((double)H[b][qm] + (double)H[b][q]),
                                   0.5 * ((double)H[c][qm] + (double)H[c][q])};
              const int64_t m = jb * ncc + kc;
              for (int k = 0; k < 4; ++k) {
                const double* w = k < 2 ? te : th;
                double* z = acc + 2 * (k * np + m);
                z[0] = z[0] + v[k] * w[0];
                z[1] = z[1] + v[k] * w[1];
              }
            }
        }
      }
    }
  }

  int enable_mur(const int32_t* en, int order, double vphase) {
    const int64_t ext[3] = {nx, ny, nz};
    const double c = vphase > 0.0 ? vphase : kC0;
    mur.clear();
    for (int f = 0; f < 6; ++f) {
      if (!en[f]) continue;
      MurFace F;
      F.ny = f / 2;
      F.nyp = (F.ny + 1) % 3;
      F.nypp = (F.ny + 2) % 3;
      const int64_t n = ext[F.ny];
      if (n < 2) return -1;
      const bool is_max = f % 2 == 1;
      // first order: the reference's lines (mur_abc.rs:93-103).  Second order:
      // at a min face the plane 0 is never updated by the E loop (not even its
      // normal component), so the boundary sits on the first updated line.
      const int64_t off = (order == 2 && !is_max) ? 1 : 0;
      if (n < 2 + off) return -1;
      F.line = is_max ? n - 1 : off;
      F.shift = is_max ? n - 2 : off + 1;
      F.size0 = ext[F.nyp];
      F.size1 = ext[F.nypp];
      // second order: the plane 0 of a tangential axis whose min face is a
      // second-order Mur face is dead (never updated) and not part of this face
      F.lo0 = (order == 2 && en[2 * F.nyp]) ? 1 : 0;
      F.lo1 = (order == 2 && en[2 * F.nypp]) ? 1 : 0;
      // src/extensions/mur_abc.rs:138-151
      const double cdt = c * dt, d = delta[F.ny];
      F.coeff = T((cdt - d) / (cdt + d));
      F.c2 = T(2.0 * d / (cdt + d));
      F.c3p = T(cdt * cdt * d / (2.0 * delta[F.nyp] * delta[F.nyp] * (cdt + d)));
      F.c3q = T(cdt * cdt * d / (2.0 * delta[F.nypp] * delta[F.nypp] * (cdt + d)));
      const size_t m = (size_t)(F.size0 * F.size1);
      for (int t = 0; t < 2; ++t) {
        F.v[t].assign(m, T(0));
        F.ob[t].assign(m, T(0));
        F.os[t].assign(m, T(0));
      }
      mur.push_back(F);
    }
    mur_order = order;
    return 0;
  }

  int64_t mur_idx(const MurFace& F, int64_t line, int64_t p, int64_t q) const {
    int64_t pos[3];
    pos[F.ny] = line;
    pos[F.nyp] = p;
    pos[F.nypp] = q;
    return idx(pos[0], pos[1], pos[2]);
  }

  // (W(+1) + W(-1)) - 2 W along one face axis of line `line`
  T lap(const std::vector<T>& W, const MurFace& F, int64_t line, int64_t p, int64_t q, bool along_p) const {
    const int64_t a = along_p ? mur_idx(F, line, p + 1, q) : mur_idx(F, line, p, q + 1);
    const int64_t b = along_p ? mur_idx(F, line, p - 1, q) : mur_idx(F, line, p, q - 1);
    const T s1 = W[a] + W[b];
    const T s2 = T(2) * W[mur_idx(F, line, p, q)];
    return s1 - s2;
  }

  // Before the E update: src/extensions/mur_abc.rs:213-254 (first order).
  void mur_pre() {
    for (MurFace& F : mur) {
      const int comp[2] = {F.nyp, F.nypp};
      for (int64_t p = 0; p < F.size0; ++p)
        for (int64_t q = 0; q < F.size1; ++q) {
          const size_t m = (size_t)(p * F.size1 + q);
          if (p < F.lo0 || q < F.lo1) continue;
          const bool interior =
              mur_order == 2 && p > F.lo0 + 1 && p + 2 < F.size0 && q > F.lo1 + 1 && q + 2 < F.size1;
          for (int t = 0; t < 2; ++t) {
            const std::vector<T>& W = E[comp[t]];
            const T wb = W[mur_idx(F, F.line, p, q)];
            const T ws = W[mur_idx(F, F.shift, p, q)];
            if (!interior) {
              const T a = F.coeff * wb;
              F.v[t][m] = ws - a;
            } else {
              const T a1 = F.coeff * F.ob[t][m];
              T acc = a1 - F.os[t][m];
              const T s = wb + ws;
              acc = acc + F.c2 * s;
              const T lp = lap(W, F, F.line, p, q, true) + lap(W, F, F.shift, p, q, true);
              acc = acc + F.c3p * lp;
              const T lq = lap(W, F, F.line, p, q, false) + lap(W, F, F.shift, p, q, false);
              acc = acc + F.c3q * lq;
              F.v[t][m] = acc;
            }
            if (mur_order == 2) {
              F.ob[t][m] = wb;
              F.os[t][m] = ws;
            }
          }
        }
    }
  }

  // After the E update: post (mur_abc.rs:257-291) for every face, then apply
  // (mur_abc.rs:294-324) face by face.
  void mur_post_apply() {
    for (MurFace& F : mur) {
      const int comp[2] = {F.nyp, F.nypp};
      for (int64_t p = 0; p < F.size0; ++p)
        for (int64_t q = 0; q < F.size1; ++q) {
          const size_t m = (size_t)(p * F.size1 + q);
          if (p < F.lo0 || q < F.lo1) continue;
          for (int t = 0; t < 2; ++t) {
            const T a = F.coeff * E[comp[t]][mur_idx(F, F.shift, p, q)];
            F.v[t][m] = F.v[t][m] + a;
          }
        }
    }
    for (MurFace& F : mur) {
      const int comp[2] = {F.nyp, F.nypp};
      for (int64_t p = 0; p < F.size0; ++p)
        for (int64_t q = 0; q < F.size1; ++q) {
          const size_t m = (size_t)(p * F.size1 + q);
          if (p < F.lo0 || q < F.lo1) continue;
          for (int t = 0; t < 2; ++t) E[comp[t]][mur_idx(F, F.line, p, q)] = F.v[t][m];
        }
    }
  }

  // src/arrays/field.rs:219-221, :314-316
  static double sumsq(const std::vector<T>& a) {
    double s = 0.0;
    for (T v : a) s += (double)v * (double)v;
    return s;
  }
  void energies(double* e, double* h) const {
    *e = sumsq(E[0]) + sumsq(E[1]) + sumsq(E[2]);
    *h = sumsq(H[0]) + sumsq(H[1]) + sumsq(H[2]);
  }

  // TF/SF plane source as the reference (src/extensions/tfsf.rs:115-355):
  // a 1D auxiliary grid in f32 driven by sin at its first H node and closed
  // by a first-order Mur end; before every H update the whole plane `pos`
  // of the H component gets h - db e_inc, before every E update the plane
  // of the E component gets e + cb h_inc (the 1D values at pos).
  struct Tfsf {
    bool on = false;
    int kind = 0;  // 0 the reference's update, 1 corrected (see tfsf_pre_h)
    int prop = 0, e_axis = 1, h_axis = 2;
    int64_t pos = 10;
    double freq = 0.0, amp = 0.0, v = kC0;
    std::vector<float> e1d, h1d;
    uint64_t t = 0;
  } tf;

  void tfsf_step_1d() {
    const double dx = delta[tf.prop];
    const size_t len = tf.h1d.size();
    for (size_t i = 0; i + 1 < len; ++i) {
      const float db = (float)(-(dt / (kMu0 * dx)));
      tf.h1d[i] += db * (tf.e1d[i + 1] - tf.e1d[i]);
    }
    const double t = (double)tf.t * dt;
    const double eta = std::sqrt(kMu0 / kEps0);
    tf.h1d[0] = (float)((tf.amp / eta) * std::sin(2.0 * kPi * tf.freq * t));
    for (size_t i = 1; i < len; ++i) {
      const float cb = (float)(dt / (kEps0 * dx));
      tf.e1d[i] += cb * (tf.h1d[i] - tf.h1d[i - 1]);
    }
    const float coeff = (float)((tf.v * dt - dx) / (tf.v * dt + dx));
    tf.e1d[len - 1] = coeff * tf.e1d[len - 2];
  }

  // Corrected 1D step: hard E source at node 0 at time n, H to n + 1/2,
  // E to n + 1 with the sign of the wave equation (the reference's E update
  // has the opposite sign and grows exponentially), first-order Mur at the
  // last node.  e_inc: E at node pos, time n; h_inc: H at pos - 1/2, n + 1/2.
  void tfsf_step_1d_fixed(float& e_inc, float& h_inc) {
    const double dx = delta[tf.prop];
    const size_t len = tf.e1d.size();
    const float db = (float)(-(dt / (kMu0 * dx))), cb = (float)(dt / (kEps0 * dx));
    tf.e1d[0] = (float)(tf.amp * std::sin(2.0 * kPi * tf.freq * ((double)tf.t * dt)));
    e_inc = tf.e1d[tf.pos];
    for (size_t i = 0; i + 1 < len; ++i) tf.h1d[i] += db * (tf.e1d[i + 1] - tf.e1d[i]);
    h_inc = tf.h1d[tf.pos - 1];
    const float en1 = tf.e1d[len - 2], en = tf.e1d[len - 1];
    for (size_t i = 1; i < len; ++i) tf.e1d[i] -= cb * (tf.h1d[i] - tf.h1d[i - 1]);
    const float coeff = (float)((tf.v * dt - dx) / (tf.v * dt + dx));
    tf.e1d[len - 1] = en1 + coeff * (tf.e1d[len - 2] - en);
    tf.t += 1;
  }
  float tf_h_inc = 0.0f;  // kind 1: H sample of the current step for the E correction

  // every cell of plane `plane` along the propagation axis of component
  // array f: f = f + coef * v (add) or f - coef * v
  // (first = 1 skips the index-0 lines the E update never writes)
  void tfsf_plane(std::vector<T>& f, T coef, T val, bool add, int64_t plane, int64_t first = 0) {
    const int64_t nn[3] = {nx, ny, nz};
    int64_t lo[3] = {first, first, first}, hi[3] = {nn[0], nn[1], nn[2]};
    lo[tf.prop] = plane;
    hi[tf.prop] = plane + 1;
    for (int64_t i = lo[0]; i < hi[0]; ++i)
      for (int64_t j = lo[1]; j < hi[1]; ++j)
        for (int64_t k = lo[2]; k < hi[2]; ++k) {
          T& x = f[(i * ny + j) * nz + k];
          x = add ? x + coef * val : x - coef * val;
        }
  }

  // Kind 1 corrections: the scattered-side H plane pos - 1 sees total E at
  // pos, so it gets -Db E_inc (= +dt/(mu0 dx) E_inc for Transverse1, where
  // the 1D H is the 3D H component; -dt/(mu0 dx) E_inc for Transverse2,
  // where it is minus it); the total-side E plane pos sees scattered H at
  // pos - 1, so it gets +Cb H_inc.
  void tfsf_pre_h() {
    if (tf.kind == 1) {
      float e_inc = 0.0f;
      tfsf_step_1d_fixed(e_inc, tf_h_inc);
      const float c = (float)(dt / (kMu0 * delta[tf.prop]));
      tfsf_plane(H[tf.h_axis], (T)c, (T)e_inc, tf.e_axis == (tf.prop + 1) % 3, tf.pos - 1);
      return;
    }
    tfsf_step_1d();
    const float e_inc = (size_t)tf.pos < tf.e1d.size() ? tf.e1d[tf.pos] : 0.0f;
    const float db = (float)(-(dt / (kMu0 * delta[tf.prop])));
    tfsf_plane(H[tf.h_axis], (T)db, (T)e_inc, false, tf.pos);
  }

  void tfsf_pre_e() {
    const float cb = (float)(dt / (kEps0 * delta[tf.prop]));
    if (tf.kind == 1) {
      tfsf_plane(E[tf.e_axis], (T)cb, (T)tf_h_inc, true, tf.pos, 1);
      return;
    }
    const float h_inc = (size_t)tf.pos < tf.h1d.size() ? tf.h1d[tf.pos] : 0.0f;
    tfsf_plane(E[tf.e_axis], (T)cb, (T)h_inc, true, tf.pos);
    tf.t += 1;
  }

  int enable_tfsf(int direction, int polarization, double freq, double amp, int64_t layer, double vphase,
                  int kind) {
    if (direction < 0 || direction > 5 || polarization < 0 || polarization > 1 || kind < 0 || kind > 1) return -1;
    tf.prop = direction / 2;
    const int64_t nn[3] = {nx, ny, nz};
    if (layer < 0 || layer >= nn[tf.prop]) return -2;
    if (kind == 1 && (layer < 1 || direction % 2 != 0)) return -3;
    tf.kind = kind;
    tf.on = true;
    tf.e_axis = polarization == 0 ? (tf.prop + 1) % 3 : (tf.prop + 2) % 3;
    tf.h_axis = polarization == 0 ? (tf.prop + 2) % 3 : (tf.prop + 1) % 3;
    tf.pos = layer;
    tf.freq = freq;
    tf.amp = amp;
    tf.v = vphase > 0.0 ? vphase : kC0;
    tf.e1d.assign(nn[tf.prop] + 1, 0.0f);
    tf.h1d.assign(nn[tf.prop] + 1, 0.0f);
    tf.t = 0;
    return 0;
  }

  // src/fdtd/basic_engine.rs:56-163
  int run_batch(uint64_t num_steps, uint64_t sample_interval, bool track_peak,
                uint64_t check_interval, bool has_decay, double decay_db, double peak0,
                orc_batch_result* res) {
    double peak = peak0;
    uint64_t executed = 0;
    int reason = 0;
    double final_db = 0.0;
    energy.clear();
    traces.clear();
    for (uint64_t step = 0; step < num_steps; ++step) {
      uint64_t cur = timestep;
      if (tf.on) tfsf_pre_h();
      if (!upml.empty()) upml_hook(true, true);
      update_h();
      if (!upml.empty()) upml_hook(true, false);
      if (tf.on) tfsf_pre_e();
      if (!mur.empty()) mur_pre();
      if (!disp.empty()) capture_dispersive();
      if (!upml.empty()) upml_hook(false, true);
      update_e();
      if (!upml.empty()) upml_hook(false, false);
      if (!mur.empty()) mur_post_apply();
      if (!disp.empty()) apply_dispersive();
      if (!rlc.empty()) apply_rlc();
      apply_excitations(step);
      record_probes(timestep + 1);
      record_fd(timestep + 1);
      timestep += 1;
      executed += 1;
      if (sample_interval > 0 && cur % sample_interval == 0) {
        orc_energy_sample smp;
        smp.timestep = cur;
        energies(&smp.e_energy, &smp.h_energy);
        smp.total_energy = smp.e_energy + smp.h_energy;
        if (track_peak) peak = std::max(peak, smp.total_energy);
        energy.push_back(smp);
      }
      if (check_interval > 0 && cur > 0 && cur % check_interval == 0) {
        if (has_decay) {
          double e, h;
          energies(&e, &h);
          double curE = e + h;
          if (peak > 0.0 && curE > 0.0) {
            double d = 10.0 * std::log10(curE / peak);
            if (d < -std::fabs(decay_db)) {
              reason = 1;
              final_db = d;
              break;
            }
          }
        }
      }
    }
    res->timesteps_executed = executed;
    res->termination_reason = reason;
    res->pad_ = 0;
    res->final_decay_db = final_db;
    res->num_energy_samples = energy.size();
    res->peak_energy = peak;
    return 0;
  }
};

struct Any {
  int precision;
  Sim<float>* f = nullptr;
  Sim<double>* d = nullptr;
};

}  // namespace

struct orc_sim {
  Any a;
};

#define DISPATCH(s, ...)             \
  do {                               \
    if ((s)->a.precision == 32) {    \
      auto* S = (s)->a.f;            \
      __VA_ARGS__;                   \
    } else {                         \
      auto* S = (s)->a.d;            \
      __VA_ARGS__;                   \
    }                                \
  } while (0)

extern "C" {

void orc_grid_timestep(const double* xl, int64_t nxl, const double* yl, int64_t nyl,
                       const double* zl, int64_t nzl, double unit, double* dt_out,
                       double* delta_out3) {
  double dx = min_delta(xl, nxl) * unit;
  double dy = min_delta(yl, nyl) * unit;
  double dz = min_delta(zl, nzl) * unit;
  double inv_sum = 1.0 / (dx * dx) + 1.0 / (dy * dy) + 1.0 / (dz * dz);
  double dt_max = 1.0 / (kC0 * std::sqrt(inv_sum));
  *dt_out = 0.99 * dt_max;
  delta_out3[0] = dx;
  delta_out3[1] = dy;
  delta_out3[2] = dz;
}

double orc_excitation_eval(int32_t kind, const double* params, double amplitude, double t) {
  return eval_excitation(kind, params, amplitude, t);
}

orc_sim* orc_new(int32_t precision, int64_t nx, int64_t ny, int64_t nz, double dt, double dx,
                 double dy, double dz) {
  if (nx <= 0 || ny <= 0 || nz <= 0) return nullptr;
  orc_sim* s = new orc_sim;
  s->a.precision = precision == 64 ? 64 : 32;
  if (s->a.precision == 32)
    s->a.f = new Sim<float>(nx, ny, nz, dt, dx, dy, dz);
  else
    s->a.d = new Sim<double>(nx, ny, nz, dt, dx, dy, dz);
  return s;
}

void orc_free(orc_sim* s) {
  if (!s) return;
  delete s->a.f;
  delete s->a.d;
  delete s;
}

void orc_set_threads(orc_sim* s, int32_t threads) { DISPATCH(s, S->threads = threads < 1 ? 1 : threads); }
void orc_set_zline(orc_sim* s, int32_t on) { DISPATCH(s, S->zline = on != 0); }

void orc_set_material(orc_sim* s, double eps_r, double mu_r, double sigma_e, double sigma_m,
                      const int64_t* r) {
  DISPATCH(s, S->set_material(eps_r, mu_r, sigma_e, sigma_m, r));
}

void orc_set_pec(orc_sim* s, const int64_t* r) { DISPATCH(s, S->set_pec(r)); }

void orc_get_coefficients(const orc_sim* s, void* out12) {
  DISPATCH(s, {
    using T = std::remove_reference_t<decltype(S->E[0][0])>;
    T* o = (T*)out12;
    const std::vector<T>* arr[12] = {&S->ca[0], &S->ca[1], &S->ca[2], &S->cb[0], &S->cb[1], &S->cb[2],
                                     &S->da[0], &S->da[1], &S->da[2], &S->db[0], &S->db[1], &S->db[2]};
    for (int a = 0; a < 12; ++a) std::memcpy(o + a * S->n, arr[a]->data(), sizeof(T) * S->n);
  });
}

void orc_set_coefficients(orc_sim* s, const void* in12) {
  DISPATCH(s, {
    using T = std::remove_reference_t<decltype(S->E[0][0])>;
    const T* p = (const T*)in12;
    std::vector<T>* arr[12] = {&S->ca[0], &S->ca[1], &S->ca[2], &S->cb[0], &S->cb[1], &S->cb[2],
                               &S->da[0], &S->da[1], &S->da[2], &S->db[0], &S->db[1], &S->db[2]};
    for (int a = 0; a < 12; ++a) std::memcpy(arr[a]->data(), p + a * S->n, sizeof(T) * S->n);
  });
}

void orc_get_fields(const orc_sim* s, void* out6) {
  DISPATCH(s, {
    using T = std::remove_reference_t<decltype(S->E[0][0])>;
    T* o = (T*)out6;
    for (int c = 0; c < 3; ++c) {
      std::memcpy(o + c * S->n, S->E[c].data(), sizeof(T) * S->n);
      std::memcpy(o + (3 + c) * S->n, S->H[c].data(), sizeof(T) * S->n);
    }
  });
}

void orc_set_fields(orc_sim* s, const void* in6) {
  DISPATCH(s, {
    using T = std::remove_reference_t<decltype(S->E[0][0])>;
    const T* p = (const T*)in6;
    for (int c = 0; c < 3; ++c) {
      std::memcpy(S->E[c].data(), p + c * S->n, sizeof(T) * S->n);
      std::memcpy(S->H[c].data(), p + (3 + c) * S->n, sizeof(T) * S->n);
    }
  });
}

void orc_reset(orc_sim* s) {
  DISPATCH(s, {
    using T = std::remove_reference_t<decltype(S->E[0][0])>;
    for (int c = 0; c < 3; ++c) {
      std::fill(S->E[c].begin(), S->E[c].end(), T(0));
      std::fill(S->H[c].begin(), S->H[c].end(), T(0));
    }
    for (int q = 0; q < 6; ++q) {
      std::fill(S->psi_h[q].begin(), S->psi_h[q].end(), T(0));
      std::fill(S->psi_e[q].begin(), S->psi_e[q].end(), T(0));
    }
    for (auto& D : S->disp)
      for (int c = 0; c < 3; ++c) {
        std::fill(D.j[c].begin(), D.j[c].end(), T(0));
        std::fill(D.pp[c].begin(), D.pp[c].end(), T(0));
        std::fill(D.ep[c].begin(), D.ep[c].end(), T(0));
      }
    for (auto& r : S->rlc) r.i_int = T(0);
    for (auto& d : S->fdumps) std::fill(d.acc.begin(), d.acc.end(), 0.0);
    for (auto& R : S->upml)
      for (int c = 0; c < 3; ++c) {
        std::fill(R.vflux[c].begin(), R.vflux[c].end(), T(0));
        std::fill(R.iflux[c].begin(), R.iflux[c].end(), T(0));
      }
    for (auto& B : S->boxes)
      for (auto& v : B.acc) std::fill(v.begin(), v.end(), 0.0);
    for (auto& F : S->mur)
      for (int t = 0; t < 2; ++t) {
        std::fill(F.v[t].begin(), F.v[t].end(), T(0));
        std::fill(F.ob[t].begin(), F.ob[t].end(), T(0));
        std::fill(F.os[t].begin(), F.os[t].end(), T(0));
      }
    std::fill(S->tf.e1d.begin(), S->tf.e1d.end(), 0.0f);
    std::fill(S->tf.h1d.begin(), S->tf.h1d.end(), 0.0f);
    S->tf.t = 0;
    S->timestep = 0;
  });
}

uint64_t orc_timestep(const orc_sim* s) {
  uint64_t t = 0;
  DISPATCH(s, t = S->timestep);
  return t;
}

void orc_clear_excitations(orc_sim* s) { DISPATCH(s, S->excs.clear()); }

void orc_add_excitation_sampled(orc_sim* s, const int64_t* pos3, int32_t dir, int32_t soft,
                                const void* samples, int64_t n) {
  DISPATCH(s, {
    using T = std::remove_reference_t<decltype(S->E[0][0])>;
    typename std::remove_reference_t<decltype(*S)>::Exc x;
    x.i = pos3[0];
    x.j = pos3[1];
    x.k = pos3[2];
    x.dir = dir;
    x.soft = soft != 0;
    x.samples.assign((const T*)samples, (const T*)samples + n);
    S->excs.push_back(x);
  });
}

// src/fdtd/batch.rs:110-129: t = (start + step) * dt, value = evaluate(t)
// rounded to the sim precision.
void orc_add_excitation_analytic(orc_sim* s, const int64_t* pos3, int32_t dir, int32_t soft,
                                 int32_t kind, const double* params, double amplitude,
                                 uint64_t start_timestep, int64_t n) {
  DISPATCH(s, {
    using T = std::remove_reference_t<decltype(S->E[0][0])>;
    typename std::remove_reference_t<decltype(*S)>::Exc x;
    x.i = pos3[0];
    x.j = pos3[1];
    x.k = pos3[2];
    x.dir = dir;
    x.soft = soft != 0;
    x.samples.resize(n);
    for (int64_t st = 0; st < n; ++st) {
      double t = (double)(start_timestep + (uint64_t)st) * S->dt;
      x.samples[st] = T(eval_excitation(kind, params, amplitude, t));
    }
    S->excs.push_back(x);
  });
}

void orc_add_point_probe(orc_sim* s, int32_t comp, const int64_t* pos3) {
  const double w = 1.0;
  orc_add_probe(s, &comp, pos3, &w, 1, 0);
}

int32_t orc_add_probe(orc_sim* s, const int32_t* comps, const int64_t* pos, const double* weights, int64_t nterms,
                      int32_t mode) {
  int32_t id = -1;
  DISPATCH(s, {
    typename std::remove_reference_t<decltype(*S)>::Probe p;
    p.mode = mode;
    bool all_h = nterms > 0;
    for (int64_t t = 0; t < nterms; ++t) {
      p.comp.push_back(comps[t]);
      p.q.push_back(S->idx(pos[3 * t], pos[3 * t + 1], pos[3 * t + 2]));
      p.w.push_back(weights[t]);
      all_h = all_h && comps[t] >= 3;
    }
    p.half = all_h ? 0.5 : 0.0;
    S->probes.push_back(p);
    id = (int32_t)S->probes.size() - 1;
  });
  return id;
}

void orc_eval_probes(orc_sim* s, double* out) {
  DISPATCH(s, {
    const size_t base = S->traces.size();
    auto saved = S->dfts;
    S->dfts.clear();
    S->record_probes(S->timestep);
    S->dfts = saved;
    for (size_t p = 0; p < S->probes.size(); ++p) out[p] = S->traces[base + p];
    S->traces.resize(base);
  });
}

void orc_get_probe_traces(const orc_sim* s, double* out, int64_t max_steps) {
  DISPATCH(s, {
    int64_t cnt = std::min<int64_t>((int64_t)S->traces.size(), max_steps * (int64_t)S->probes.size());
    std::memcpy(out, S->traces.data(), sizeof(double) * cnt);
  });
}

int32_t orc_add_probe_dft(orc_sim* s, int32_t probe, const double* freqs, int64_t nfreq) {
  int32_t id = -1;
  DISPATCH(s, {
    if (probe < 0 || probe >= (int32_t)S->probes.size()) return -1;
    typename std::remove_reference_t<decltype(*S)>::ProbeDft d;
    d.probe = probe;
    d.freqs.assign(freqs, freqs + nfreq);
    d.re.assign(nfreq, 0.0);
    d.im.assign(nfreq, 0.0);
    S->dfts.push_back(d);
    id = (int32_t)S->dfts.size() - 1;
  });
  return id;
}

void orc_get_probe_dft(const orc_sim* s, int32_t dft, double* out) {
  DISPATCH(s, {
    const auto& d = S->dfts[dft];
    for (size_t f = 0; f < d.freqs.size(); ++f) {
      out[2 * f] = d.re[f];
      out[2 * f + 1] = d.im[f];
    }
  });
}

int32_t orc_add_field_dft(orc_sim* s, const int64_t* region6, const int64_t* sub3, uint32_t comp_mask,
                          const double* freqs, int64_t nfreq, uint64_t interval) {
  int32_t id = -1;
  DISPATCH(s, {
    typename std::remove_reference_t<decltype(*S)>::FieldDft d;
    const int64_t ext[3] = {S->nx, S->ny, S->nz};
    d.npts = 1;
    for (int a = 0; a < 3; ++a) {
      d.r[2 * a] = std::min(region6[2 * a], ext[a]);
      d.r[2 * a + 1] = std::min(region6[2 * a + 1], ext[a]);
      d.ss[a] = std::max<int64_t>(sub3[a], 1);
      const int64_t len = std::max<int64_t>(d.r[2 * a + 1] - d.r[2 * a], 0);
      d.n[a] = (len + d.ss[a] - 1) / d.ss[a];
      d.npts *= d.n[a];
    }
    for (int c = 0; c < 6; ++c)
      if (comp_mask & (1u << c)) d.comps.push_back(c);
    d.interval = std::max<uint64_t>(interval, 1);
    d.freqs.assign(freqs, freqs + nfreq);
    d.acc.assign(2 * (size_t)nfreq * d.comps.size() * (size_t)d.npts, 0.0);
    S->fdumps.push_back(std::move(d));
    id = (int32_t)S->fdumps.size() - 1;
  });
  return id;
}

int64_t orc_field_dft_points(const orc_sim* s, int32_t id) {
  int64_t n = 0;
  DISPATCH(s, n = S->fdumps[id].npts);
  return n;
}

void orc_get_field_dft(const orc_sim* s, int32_t id, int64_t f, int64_t comp_slot, double* out) {
  DISPATCH(s, {
    const auto& d = S->fdumps[id];
    const size_t off = 2 * (f * d.comps.size() + comp_slot) * (size_t)d.npts;
    std::memcpy(out, d.acc.data() + off, 2 * sizeof(double) * d.npts);
  });
}

int32_t orc_add_nf2ff_box(orc_sim* s, const int64_t* lo3, const int64_t* hi3, const int32_t* dirs6,
                          const double* freqs, int64_t nfreq, uint64_t interval) {
  int32_t id = -1;
  DISPATCH(s, {
    typename std::remove_reference_t<decltype(*S)>::Nf2ffBox B;
    const int64_t ext[3] = {S->nx, S->ny, S->nz};
    for (int a = 0; a < 3; ++a) {
      if (lo3[a] < 1 || hi3[a] <= lo3[a] || hi3[a] > ext[a] - 1) return -1;
      B.lo[a] = lo3[a];
      B.hi[a] = hi3[a];
    }
    B.interval = std::max<uint64_t>(interval, 1);
    B.freqs.assign(freqs, freqs + nfreq);
    for (int f = 0; f < 6; ++f) {
      B.dirs[f] = dirs6[f] != 0;
      if (!B.dirs[f]) continue;
      const int a = f / 2, b = (a + 1) % 3, c = (a + 2) % 3;
      const int64_t np = (B.hi[b] - B.lo[b] + 1) * (B.hi[c] - B.lo[c] + 1);
      B.faces.push_back(f);
      B.acc.emplace_back(8 * (size_t)nfreq * (size_t)np, 0.0);
    }
    S->boxes.push_back(std::move(B));
    id = (int32_t)S->boxes.size() - 1;
  });
  return id;
}

/* out: 4 arrays (Eb, Ec, Hb, Hc) of nb * nc (re, im); returns nb * nc, 0 if
 * the face is not recorded. */
int64_t orc_get_nf2ff_face(const orc_sim* s, int32_t id, int32_t face, int64_t f, double* out) {
  int64_t np = 0;
  DISPATCH(s, {
    const auto& B = S->boxes[id];
    for (size_t fs = 0; fs < B.faces.size(); ++fs) {
      if (B.faces[fs] != face) continue;
      const int a = face / 2, b = (a + 1) % 3, c = (a + 2) % 3;
      np = (B.hi[b] - B.lo[b] + 1) * (B.hi[c] - B.lo[c] + 1);
      std::memcpy(out, B.acc[fs].data() + f * 8 * (size_t)np, 8 * sizeof(double) * np);
    }
  });
  return np;
}

int32_t orc_enable_cpml(orc_sim* s, const int32_t* layers6, double m, double R, double alpha_max,
                        double kappa_max) {
  int rc = 0;
  DISPATCH(s, rc = S->enable_cpml(layers6, m, R, alpha_max, kappa_max));
  return rc;
}

int32_t orc_cpml_profile(const orc_sim* s, int32_t f, double* out) {
  int L = 0;
  DISPATCH(s, {
    if (!S->cpml || f < 0 || f >= 6) return 0;
    const CpmlFace& F = S->face[f];
    L = F.layers;
    for (int l = 0; l < L; ++l) {
      out[0 * L + l] = F.b_e[l];
      out[1 * L + l] = F.c_e[l];
      out[2 * L + l] = F.ik_e[l];
      out[3 * L + l] = F.b_h[l];
      out[4 * L + l] = F.c_h[l];
      out[5 * L + l] = F.ik_h[l];
    }
  });
  return L;
}

int32_t orc_add_dispersive(orc_sim* s, int32_t kind, const double* p, double eps_inf, const int64_t* cells,
                           int64_t ncells) {
  if (kind < 0 || kind > 4 || !(eps_inf > 0.0)) return -1;
  int32_t rc = 0;
  DISPATCH(s, {
    typename std::remove_reference_t<decltype(*S)>::Dispersive D;
    D.kind = kind;
    const double dt = S->dt;
    if (kind == 0) {  // DrudeMaterial::new (dispersive.rs:476-498)
      const double wp = p[0], g = p[1], den = 1.0 + g * dt / 2.0;
      D.a = (float)((1.0 - g * dt / 2.0) / den);
      D.b = (float)(kEps0 * wp * wp * dt / den);
      D.c = (float)(dt / (kEps0 * eps_inf));
    } else if (kind == 1 || kind == 3) {  // LorentzMaterial::new (dispersive.rs:134-159)
      const double w0 = p[0], g = p[1], de = p[2], den = 1.0 + g * dt / 2.0;
      D.a = (float)((2.0 - w0 * w0 * dt * dt) / den);
      D.b = (float)((g * dt / 2.0 - 1.0) / den);
      D.c = (float)(kEps0 * de * w0 * w0 * dt * dt / den);
      D.c2 = (float)(1.0 / (kEps0 * eps_inf));
    } else if (kind == 4) {  // Drude as a P recursion: P'' + g P' = eps0 wp^2 E
      const double wp = p[0], g = p[1], den = 1.0 + g * dt / 2.0;
      D.a = (float)(2.0 / den);
      D.b = (float)((g * dt / 2.0 - 1.0) / den);
      D.c = (float)(kEps0 * wp * wp * dt * dt / den);
      D.c2 = (float)(1.0 / (kEps0 * eps_inf));
    } else {  // DebyeMaterial::new (dispersive.rs:570-592)
      const double tau = p[0], de = p[1], den = 2.0 * tau + dt;
      D.a = (float)((2.0 * tau - dt) / den);
      D.b = (float)(2.0 * kEps0 * de * dt / den);
      D.c = (float)(dt / (kEps0 * eps_inf));
    }
    for (int64_t m = 0; m < ncells; ++m) D.q.push_back(S->idx(cells[3 * m], cells[3 * m + 1], cells[3 * m + 2]));
    for (int c = 0; c < 3; ++c) {
      D.j[c].assign(ncells, 0);
      D.pp[c].assign(ncells, 0);
      D.ep[c].assign(ncells, 0);
    }
    S->disp.push_back(D);
  });
  return rc;
}

int32_t orc_add_lumped_rlc(orc_sim* s, const int64_t* pos, int32_t dir, int32_t type, double r, double l,
                           double c) {
  DISPATCH(s, {
    typename std::remove_reference_t<decltype(*S)>::Rlc e;
    const double dt = S->dt, dl = S->delta[dir], da = dl * dl;
    double v_vv, v_il;
    if (type == 0) {  // calc_parallel_coeffs (lumped_rlc.rs:190-216)
      const double g = r > 0 ? 1.0 / r : 0.0;
      const double inv_l = l > 0 ? dt / l : 0.0;
      const double cc = c > 0 ? c : 0.0;
      const double g_eff = g * dl / da;
      const double c_eff = cc * dl / da + kEps0 * dl / da;
      const double den = 2.0 * c_eff + g_eff * dt;
      v_vv = (2.0 * c_eff - g_eff * dt) / den;
      v_il = inv_l * dl / da;
    } else {  // calc_series_coeffs (lumped_rlc.rs:219-250)
      const double rr = r > 0 ? r : 0.0, ll = l > 0 ? l : 0.0;
      const double inv_c = c > 0 ? dt / c : 0.0;
      const double den = 2.0 * (ll * da / dl) + (rr * da / dl) * dt;
      v_vv = 1.0;
      v_il = std::fabs(den) < 1e-20 ? 0.0 : inv_c * da / dl;
    }
    e.q = S->idx(pos[0], pos[1], pos[2]);
    e.dir = dir;
    e.v_vv = (float)v_vv;
    e.v_il = (float)v_il;
    e.i_int = 0;
    S->rlc.push_back(e);
  });
  return 0;
}

double orc_set_lumped(orc_sim* s, const int64_t* pos, int32_t dir, double r, double c, double eps_r,
                      double sigma) {
  double scale = 0.0;
  DISPATCH(s, {
    using T = std::remove_reference_t<decltype(S->E[0][0])>;
    const int a = (dir + 1) % 3, b = (dir + 2) % 3;
    const double dl = S->delta[dir], area = S->delta[a] * S->delta[b], dt = S->dt;
    const double eps = eps_r * kEps0 + (c > 0 ? c * dl / area : 0.0);
    const double sig = sigma + (r > 0 ? dl / (r * area) : 0.0);
    const double loss = sig * dt / (2.0 * eps);
    const int64_t q = S->idx(pos[0], pos[1], pos[2]);
    S->ca[dir][q] = T((1.0 - loss) / (1.0 + loss));
    S->cb[dir][q] = T((dt / eps) / (1.0 + loss) / dl);
    scale = r > 0 ? (dt / eps) / (1.0 + loss) / (r * area) : 0.0;
  });
  return scale;
}

int32_t orc_enable_upml(orc_sim* s, const int64_t* layers6, double grading_order, double reflection_coeff,
                        int32_t kind) {
  if (kind != 0 && kind != 1) return -1;
  int n = 0;
  DISPATCH(s, n = S->enable_upml(layers6, grading_order, reflection_coeff, kind));
  return n;
}

void orc_upml_kappa(const orc_sim* s, int32_t comp, int32_t dir, const int64_t* pos3, int32_t is_min,
                    int64_t layers, double width, double smax, double m, double* kv, double* ki) {
  DISPATCH(s, S->upml_kappa(comp, dir, pos3, is_min != 0, layers, width, smax, m, kv, ki));
}

int32_t orc_enable_mur(orc_sim* s, const int32_t* enabled6, int32_t order, double phase_velocity) {
  if (order != 1 && order != 2) return -2;
  int rc = 0;
  DISPATCH(s, rc = S->enable_mur(enabled6, order, phase_velocity));
  return rc;
}

int32_t orc_enable_tfsf(orc_sim* s, int32_t direction, int32_t polarization, double frequency, double amplitude,
                        int64_t boundary_layer, double phase_velocity, int32_t kind) {
  int rc = 0;
  DISPATCH(s, rc = S->enable_tfsf(direction, polarization, frequency, amplitude, boundary_layer, phase_velocity,
                                  kind));
  return rc;
}

int32_t orc_run_batch(orc_sim* s, uint64_t num_steps, uint64_t sample_interval, int32_t track_peak,
                      uint64_t check_interval, int32_t has_decay, double decay_db,
                      double initial_peak, orc_batch_result* res) {
  int rc = 0;
  DISPATCH(s, rc = S->run_batch(num_steps, sample_interval, track_peak != 0, check_interval,
                                has_decay != 0, decay_db, initial_peak, res));
  return rc;
}

void orc_get_energy_samples(const orc_sim* s, orc_energy_sample* out, uint64_t cap) {
  DISPATCH(s, {
    uint64_t cnt = std::min<uint64_t>(cap, S->energy.size());
    std::memcpy(out, S->energy.data(), sizeof(orc_energy_sample) * cnt);
  });
}

void orc_energy(const orc_sim* s, double* e, double* h) { DISPATCH(s, S->energies(e, h)); }

}  // extern "C"
