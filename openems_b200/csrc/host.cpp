// host.cpp -- C++ host-side mirror of the reference's Grid / Operator /
// Excitation / Simulation surface (declared for C callers in
// include/oems_host.h).  Everything here runs on the CPU once per setup or per
// batch; the timestep loop itself runs on the GPU behind include/oems.h.
#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstring>
#include <limits>
#include <memory>
#include <string>
#include <thread>
#include <unordered_map>
#include <vector>

#include "../../include/oems.h"
#include "../../include/oems_host.h"

namespace oems {
extern thread_local std::string g_last_error;
}

namespace {

using oems::g_last_error;

oems_status hfail(oems_status st, const char* msg) {
  g_last_error = msg;
  return st;
}

// src/constants.rs:8-14
constexpr double kC0 = 299792458.0;
constexpr double kEps0 = 8.854187817e-12;
constexpr double kMu0 = 1.256637062e-6;
constexpr double kPi = 3.14159265358979323846;

// Grid (src/geometry/mod.rs): mesh lines per axis, scaled by unit.
struct Grid {
  std::vector<double> lines[3];
  double unit = 1.0;

  // cells = lines - 1, at least 1 (src/geometry/mod.rs:85-92)
  uint64_t cells(int a) const { return lines[a].size() > 1 ? lines[a].size() - 1 : 1; }

  // minimum positive spacing (src/geometry/mod.rs:113-119, :242-255)
  double min_delta(int a) const {
    const auto& l = lines[a];
    if (l.size() < 2) return 1.0 * unit;
    double m = std::numeric_limits<double>::max();
    for (size_t i = 0; i + 1 < l.size(); ++i) {
      const double d = l[i + 1] - l[i];
      if (d > 0.0 && d < m) m = d;
    }
    return m * unit;
  }
};

}  // namespace

// Operator (src/fdtd/operator.rs:42-263).
struct oems_operator {
  Grid grid;
  uint64_t n[3] = {0, 0, 0};
  double dt = 0.0;
  double delta[3] = {0, 0, 0};
  std::vector<float> c[12];  // ca0..2 cb0..2 da0..2 db0..2

  size_t idx(uint64_t i, uint64_t j, uint64_t k) const { return (size_t)((i * n[1] + j) * n[2] + k); }

  void init() {
    for (int a = 0; a < 3; ++a) {
      n[a] = grid.cells(a);
      delta[a] = grid.min_delta(a);
    }
    // src/fdtd/operator.rs:82-89: dt = 0.99 / (c0 * sqrt(sum 1/d^2))
    const double inv_sum = 1.0 / (delta[0] * delta[0]) + 1.0 / (delta[1] * delta[1]) + 1.0 / (delta[2] * delta[2]);
    dt = 0.99 * (1.0 / (kC0 * std::sqrt(inv_sum)));
    const size_t cells = (size_t)(n[0] * n[1] * n[2]);
    // src/fdtd/operator.rs:92-141: vacuum Ca = Da = 1, Cb = dt/(eps0 d), Db = -dt/(mu0 d)
    float v[12];
    for (int a = 0; a < 3; ++a) {
      v[a] = 1.0f;
      v[3 + a] = (float)(dt / (kEps0 * delta[a]));
      v[6 + a] = 1.0f;
      v[9 + a] = -(float)(dt / (kMu0 * delta[a]));
    }
    // the twelve arrays are independent: fill them on parallel threads when
    // they are large (hundreds of MB at 256^3)
    auto fill = [&](int a) { c[a].assign(cells, v[a]); };
    if (cells < (size_t)1 << 20) {
      for (int a = 0; a < 12; ++a) fill(a);
    } else {
      std::vector<std::thread> t;
      for (int a = 1; a < 12; ++a) t.emplace_back(fill, a);
      fill(0);
      for (auto& x : t) x.join();
    }
  }
};

struct oems_simulation {
  oems_operator op;
  int32_t device = -1;
  uint32_t flags = 0;
  std::vector<oems_excitation> excitations;
  int32_t end_kind = OEMS_END_TIMESTEPS;
  double end_value = 10000.0;  // EndCondition::default (src/fdtd/simulation.rs:45-49)
  uint64_t batch_size = 0;
  bool has_cpml = false;
  oems_cpml_desc cpml{};
  oems_engine* engine = nullptr;
  bool ran = false;
};

namespace {

bool clip_region(const oems_operator* op, const uint64_t* r, uint64_t* out) {
  for (int a = 0; a < 3; ++a) {
    out[2 * a] = std::min(r[2 * a], op->n[a]);
    out[2 * a + 1] = std::min(r[2 * a + 1], op->n[a]);
  }
  return true;
}

double eval(const oems_excitation* x, double t) {
  // src/fdtd/excitation.rs:150-200
  double v = 0.0;
  switch (x->kind) {
    case OEMS_EXC_GAUSSIAN: {
      const double arg = (t - x->params[0]) / x->params[1];
      v = std::exp(-arg * arg);
      break;
    }
    case OEMS_EXC_SINUSOIDAL:
      v = std::sin(2.0 * kPi * x->params[0] * t);
      break;
    case OEMS_EXC_GAUSSIAN_MODULATED: {
      const double arg = (t - x->params[1]) / x->params[2];
      const double env = std::exp(-arg * arg);
      const double car = std::sin(2.0 * kPi * x->params[0] * t);
      v = env * car;
      break;
    }
    case OEMS_EXC_DIRAC:
      v = std::fabs(t) < 1e-15 ? 1.0 : 0.0;
      break;
    case OEMS_EXC_STEP:
      v = t >= 0.0 ? 1.0 : 0.0;
      break;
    default:
      v = 0.0;
  }
  return x->amplitude * v;
}

void fill_exc(int32_t kind, uint32_t dir, const uint64_t* pos, oems_excitation* out) {
  *out = oems_excitation{};
  out->kind = kind;
  out->direction = dir;
  for (int a = 0; a < 3; ++a) out->position[a] = pos[a];
  out->amplitude = 1.0;
  out->soft_source = 1;
}

}  // namespace

extern "C" {

// ---- compressed coefficients (src/fdtd/compressed.rs:125-192) -------------
// Exact (bitwise) deduplication of each cell's 12 coefficients into a table:
// the reference quantises at 1e-10 (compressed.rs:11-31), below one f32 ulp
// of every coefficient magnitude the operator produces, so both find the
// same sets.  Ids are assigned in cell order.
namespace {
struct CoefSet {
  float v[12];
  bool operator==(const CoefSet& o) const { return std::memcmp(v, o.v, sizeof(v)) == 0; }
};
struct CoefSetHash {
  size_t operator()(const CoefSet& k) const {
    uint64_t h = 1469598103934665603ull;  // FNV-1a over the 48 bytes
    const unsigned char* p = reinterpret_cast<const unsigned char*>(k.v);
    for (size_t i = 0; i < sizeof(k.v); ++i) h = (h ^ p[i]) * 1099511628211ull;
    return (size_t)h;
  }
};
}  // namespace

oems_status oems_compress_coefficients(const float* const coef[12], uint64_t ncells, uint16_t* ids, float* table,
                                       uint32_t table_cap, uint32_t* nunique) {
  if (!coef || !nunique) return hfail(OEMS_ERR_INVALID_ARGUMENT, "NULL argument");
  for (int a = 0; a < 12; ++a)
    if (!coef[a] && ncells) return hfail(OEMS_ERR_INVALID_ARGUMENT, "coefficient array pointer is NULL");
  std::unordered_map<CoefSet, uint32_t, CoefSetHash> map;
  for (uint64_t q = 0; q < ncells; ++q) {
    CoefSet key;
    for (int a = 0; a < 12; ++a) key.v[a] = coef[a][q];
    auto it = map.find(key);
    uint32_t id;
    if (it == map.end()) {
      id = (uint32_t)map.size();
      if (id >= 65536)
        return hfail(OEMS_ERR_MATERIAL, "more than 65536 unique coefficient sets; compressed storage refused");
      map.emplace(key, id);
      if (table && id < table_cap) std::memcpy(table + (size_t)id * 12, key.v, sizeof(key.v));
    } else {
      id = it->second;
    }
    if (ids) ids[q] = (uint16_t)id;
  }
  *nunique = (uint32_t)map.size();
  return OEMS_OK;
}

oems_status oems_operator_create(const double* xl, uint64_t nxl, const double* yl, uint64_t nyl, const double* zl,
                                 uint64_t nzl, double unit, oems_operator** out) {
  if (!out || !xl || !yl || !zl) return hfail(OEMS_ERR_INVALID_ARGUMENT, "NULL argument");
  *out = nullptr;
  if (nxl < 2 || nyl < 2 || nzl < 2) return hfail(OEMS_ERR_GRID, "each axis needs at least two mesh lines");
  if (!(unit > 0.0)) return hfail(OEMS_ERR_GRID, "unit must be positive");
  std::unique_ptr<oems_operator> op(new oems_operator);
  op->grid.lines[0].assign(xl, xl + nxl);
  op->grid.lines[1].assign(yl, yl + nyl);
  op->grid.lines[2].assign(zl, zl + nzl);
  op->grid.unit = unit;
  for (int a = 0; a < 3; ++a) {
    const auto& l = op->grid.lines[a];
    for (size_t i = 0; i + 1 < l.size(); ++i)
      if (!(l[i + 1] > l[i])) return hfail(OEMS_ERR_GRID, "mesh lines must be strictly increasing");
  }
  op->init();
  *out = op.release();
  return OEMS_OK;
}

oems_status oems_operator_create_uniform(uint64_t nx, uint64_t ny, uint64_t nz, double delta, oems_operator** out) {
  if (!out) return hfail(OEMS_ERR_INVALID_ARGUMENT, "NULL argument");
  if (nx == 0 || ny == 0 || nz == 0) return hfail(OEMS_ERR_GRID, "grid dimensions must be positive");
  if (!(delta > 0.0)) return hfail(OEMS_ERR_GRID, "cell size must be positive");
  // src/geometry/mod.rs:60-66: lines = i * delta
  std::vector<double> l[3];
  const uint64_t n[3] = {nx, ny, nz};
  for (int a = 0; a < 3; ++a) {
    l[a].resize(n[a] + 1);
    for (uint64_t i = 0; i <= n[a]; ++i) l[a][i] = (double)i * delta;
  }
  return oems_operator_create(l[0].data(), l[0].size(), l[1].data(), l[1].size(), l[2].data(), l[2].size(), 1.0,
                              out);
}

void oems_operator_destroy(oems_operator* op) { delete op; }

// Finite, positive permittivity and permeability, finite non-negative
// conductivities: anything else (NaN or infinite parameters included)
// would put non-finite numbers into the coefficients.
static bool material_ok(double eps_r, double mu_r, double sigma_e, double sigma_m) {
  return std::isfinite(eps_r) && eps_r > 0.0 && std::isfinite(mu_r) && mu_r > 0.0 && std::isfinite(sigma_e) &&
         sigma_e >= 0.0 && std::isfinite(sigma_m) && sigma_m >= 0.0;
}

oems_status oems_operator_set_material(oems_operator* op, double eps_r, double mu_r, double sigma_e, double sigma_m,
                                       const uint64_t region[6]) {
  if (!op || !region) return hfail(OEMS_ERR_INVALID_ARGUMENT, "NULL argument");
  if (!material_ok(eps_r, mu_r, sigma_e, sigma_m))
    return hfail(OEMS_ERR_MATERIAL, "eps_r and mu_r must be positive, conductivities non-negative, all finite");
  uint64_t r[6];
  clip_region(op, region, r);
  // src/fdtd/operator.rs:195-220
  const double dt = op->dt;
  const double eps = eps_r * kEps0;
  const double loss_e = sigma_e * dt / (2.0 * eps);
  const float ca_mat = (float)((1.0 - loss_e) / (1.0 + loss_e));
  const double cb_factor = (dt / eps) / (1.0 + loss_e);
  const float cbv[3] = {(float)(cb_factor / op->delta[0]), (float)(cb_factor / op->delta[1]),
                        (float)(cb_factor / op->delta[2])};
  const double mu = mu_r * kMu0;
  const double loss_m = sigma_m * dt / (2.0 * mu);
  const float da_mat = (float)((1.0 - loss_m) / (1.0 + loss_m));
  const double db_factor = -(dt / mu) / (1.0 + loss_m);
  const float dbv[3] = {(float)(db_factor / op->delta[0]), (float)(db_factor / op->delta[1]),
                        (float)(db_factor / op->delta[2])};
  for (uint64_t i = r[0]; i < r[1]; ++i)
    for (uint64_t j = r[2]; j < r[3]; ++j) {
      const size_t q0 = op->idx(i, j, 0);
      for (int a = 0; a < 3; ++a) {
        std::fill(op->c[a].begin() + q0 + r[4], op->c[a].begin() + q0 + r[5], ca_mat);
        std::fill(op->c[3 + a].begin() + q0 + r[4], op->c[3 + a].begin() + q0 + r[5], cbv[a]);
        std::fill(op->c[6 + a].begin() + q0 + r[4], op->c[6 + a].begin() + q0 + r[5], da_mat);
        std::fill(op->c[9 + a].begin() + q0 + r[4], op->c[9 + a].begin() + q0 + r[5], dbv[a]);
      }
    }
  return OEMS_OK;
}

oems_status oems_operator_set_material_cells(oems_operator* op, double eps_r, double mu_r, double sigma_e,
                                             double sigma_m, const uint64_t* cells, uint64_t ncells) {
  if (!op || (!cells && ncells)) return hfail(OEMS_ERR_INVALID_ARGUMENT, "NULL argument");
  if (!material_ok(eps_r, mu_r, sigma_e, sigma_m))
    return hfail(OEMS_ERR_MATERIAL, "eps_r and mu_r must be positive, conductivities non-negative, all finite");
  for (uint64_t m = 0; m < ncells; ++m)
    if (cells[3 * m] >= op->n[0] || cells[3 * m + 1] >= op->n[1] || cells[3 * m + 2] >= op->n[2])
      return hfail(OEMS_ERR_MATERIAL, "material cell outside the grid");
  // the same coefficients as set_material (src/fdtd/operator.rs:195-220) on
  // each listed cell
  const double dt = op->dt;
  const double eps = eps_r * kEps0;
  const double loss_e = sigma_e * dt / (2.0 * eps);
  const float ca_mat = (float)((1.0 - loss_e) / (1.0 + loss_e));
  const double cb_factor = (dt / eps) / (1.0 + loss_e);
  const double mu = mu_r * kMu0;
  const double loss_m = sigma_m * dt / (2.0 * mu);
  const float da_mat = (float)((1.0 - loss_m) / (1.0 + loss_m));
  const double db_factor = -(dt / mu) / (1.0 + loss_m);
  float cbv[3], dbv[3];
  for (int a = 0; a < 3; ++a) {
    cbv[a] = (float)(cb_factor / op->delta[a]);
    dbv[a] = (float)(db_factor / op->delta[a]);
  }
  for (uint64_t m = 0; m < ncells; ++m) {
    const size_t q = op->idx(cells[3 * m], cells[3 * m + 1], cells[3 * m + 2]);
    for (int a = 0; a < 3; ++a) {
      op->c[a][q] = ca_mat;
      op->c[3 + a][q] = cbv[a];
      op->c[6 + a][q] = da_mat;
      op->c[9 + a][q] = dbv[a];
    }
  }
  return OEMS_OK;
}

oems_status oems_operator_set_pec(oems_operator* op, const uint64_t region[6]) {
  if (!op || !region) return hfail(OEMS_ERR_INVALID_ARGUMENT, "NULL argument");
  uint64_t r[6];
  clip_region(op, region, r);
  // src/fdtd/operator.rs:249-263: Ca = Cb = 0
  for (uint64_t i = r[0]; i < r[1]; ++i)
    for (uint64_t j = r[2]; j < r[3]; ++j) {
      const size_t q0 = op->idx(i, j, 0);
      for (int a = 0; a < 6; ++a) std::fill(op->c[a].begin() + q0 + r[4], op->c[a].begin() + q0 + r[5], 0.0f);
    }
  return OEMS_OK;
}

oems_status oems_operator_set_lumped(oems_operator* op, const uint64_t pos[3], int32_t dir, double r, double c,
                                     double eps_r, double sigma, double* source_scale) {
  if (!op || !pos) return hfail(OEMS_ERR_INVALID_ARGUMENT, "NULL argument");
  if (dir < 0 || dir > 2) return hfail(OEMS_ERR_CONFIG, "lumped element direction must be 0, 1 or 2");
  for (int a = 0; a < 3; ++a)
    if (pos[a] >= op->n[a]) return hfail(OEMS_ERR_CONFIG, "lumped element outside the grid");
  if (!(eps_r > 0.0) || sigma < 0.0) return hfail(OEMS_ERR_MATERIAL, "eps_r must be positive, sigma >= 0");
  const int a = (dir + 1) % 3, b = (dir + 2) % 3;
  const double dl = op->delta[dir], area = op->delta[a] * op->delta[b], dt = op->dt;
  const double eps = eps_r * kEps0 + (c > 0 ? c * dl / area : 0.0);
  const double sig = sigma + (r > 0 ? dl / (r * area) : 0.0);
  const double loss = sig * dt / (2.0 * eps);
  const size_t q = op->idx(pos[0], pos[1], pos[2]);
  op->c[dir][q] = (float)((1.0 - loss) / (1.0 + loss));
  op->c[3 + dir][q] = (float)((dt / eps) / (1.0 + loss) / dl);
  if (source_scale) *source_scale = r > 0 ? (dt / eps) / (1.0 + loss) / (r * area) : 0.0;
  return OEMS_OK;
}

oems_status oems_operator_clone(const oems_operator* op, oems_operator** out) {
  if (!op || !out) return hfail(OEMS_ERR_INVALID_ARGUMENT, "NULL argument");
  *out = new oems_operator(*op);
  return OEMS_OK;
}

oems_status oems_operator_info(const oems_operator* op, uint64_t dims[3], double* dt, double delta[3]) {
  if (!op) return hfail(OEMS_ERR_INVALID_ARGUMENT, "NULL operator");
  for (int a = 0; a < 3; ++a) {
    if (dims) dims[a] = op->n[a];
    if (delta) delta[a] = op->delta[a];
  }
  if (dt) *dt = op->dt;
  return OEMS_OK;
}

oems_status oems_operator_coefficients(const oems_operator* op, const float* out[12]) {
  if (!op || !out) return hfail(OEMS_ERR_INVALID_ARGUMENT, "NULL argument");
  for (int a = 0; a < 12; ++a) out[a] = op->c[a].data();
  return OEMS_OK;
}

oems_status oems_operator_engine_desc(const oems_operator* op, int32_t device, uint32_t flags, oems_operator_desc* d) {
  if (!op || !d) return hfail(OEMS_ERR_INVALID_ARGUMENT, "NULL argument");
  *d = oems_operator_desc{};
  d->nx = op->n[0];
  d->ny = op->n[1];
  d->nz = op->n[2];
  d->dt = op->dt;
  for (int a = 0; a < 3; ++a) {
    d->delta[a] = op->delta[a];
    d->ca[a] = op->c[a].data();
    d->cb[a] = op->c[3 + a].data();
    d->da[a] = op->c[6 + a].data();
    d->db[a] = op->c[9 + a].data();
  }
  d->device = device;
  d->flags = flags;
  return OEMS_OK;
}

// src/fdtd/excitation.rs:67-85
oems_status oems_excitation_gaussian(double center_freq, double bandwidth, uint32_t direction,
                                     const uint64_t position[3], oems_excitation* out) {
  if (!out || !position) return hfail(OEMS_ERR_INVALID_ARGUMENT, "NULL argument");
  fill_exc(OEMS_EXC_GAUSSIAN, direction, position, out);
  const double f_max = center_freq * (1.0 + 0.5 * bandwidth);
  const double tau = 1.0 / (kPi * f_max);
  out->params[0] = 4.0 * tau;
  out->params[1] = tau;
  return OEMS_OK;
}

// src/fdtd/excitation.rs:88-108
oems_status oems_excitation_gaussian_modulated(double center_freq, double bandwidth, uint32_t direction,
                                               const uint64_t position[3], oems_excitation* out) {
  if (!out || !position) return hfail(OEMS_ERR_INVALID_ARGUMENT, "NULL argument");
  fill_exc(OEMS_EXC_GAUSSIAN_MODULATED, direction, position, out);
  const double tau = 1.0 / (kPi * center_freq * bandwidth);
  out->params[0] = center_freq;
  out->params[1] = 4.0 * tau;
  out->params[2] = tau;
  return OEMS_OK;
}

// src/fdtd/excitation.rs:111-119
oems_status oems_excitation_sinusoidal(double frequency, uint32_t direction, const uint64_t position[3],
                                       oems_excitation* out) {
  if (!out || !position) return hfail(OEMS_ERR_INVALID_ARGUMENT, "NULL argument");
  fill_exc(OEMS_EXC_SINUSOIDAL, direction, position, out);
  out->params[0] = frequency;
  return OEMS_OK;
}

// src/fdtd/excitation.rs:127-135
oems_status oems_excitation_dirac(double amplitude, uint32_t direction, const uint64_t position[3],
                                  oems_excitation* out) {
  if (!out || !position) return hfail(OEMS_ERR_INVALID_ARGUMENT, "NULL argument");
  fill_exc(OEMS_EXC_DIRAC, direction, position, out);
  out->amplitude = amplitude;
  return OEMS_OK;
}

double oems_excitation_evaluate(const oems_excitation* exc, double t) { return exc ? eval(exc, t) : 0.0; }

// src/fdtd/batch.rs:110-129
oems_status oems_excitation_sample(const oems_excitation* exc, uint64_t start, uint64_t n, double dt, float* out) {
  if (!exc || (!out && n)) return hfail(OEMS_ERR_INVALID_ARGUMENT, "NULL argument");
  for (uint64_t s = 0; s < n; ++s) out[s] = (float)eval(exc, (double)(start + s) * dt);
  return OEMS_OK;
}

// ---- probe term builders ----------------------------------------------------

namespace {

struct TermList {
  oems_probe_term* out;
  uint64_t cap, n = 0;
  void add(int comp, uint64_t i, uint64_t j, uint64_t k, double w) {
    if (n < cap) {
      oems_probe_term& t = out[n];
      t = oems_probe_term{};
      t.component = comp;
      t.position[0] = i;
      t.position[1] = j;
      t.position[2] = k;
      t.weight = w;
    }
    ++n;
  }
};

// Grid::delta_x/y/z (src/geometry/mod.rs:281-313)
double grid_delta(const oems_operator* op, int a, uint64_t i) {
  const auto& l = op->grid.lines[a];
  if (i + 1 < l.size()) return (l[i + 1] - l[i]) * op->grid.unit;
  if (i > 0) return (l[i] - l[i - 1]) * op->grid.unit;
  return op->grid.unit;
}

oems_status finish(TermList& L, uint64_t* n) {
  if (n) *n = L.n;
  return OEMS_OK;
}

}  // namespace

oems_status oems_probe_voltage_terms(const uint64_t s[3], const uint64_t e[3], int32_t dir, oems_probe_term* out,
                                     uint64_t cap, uint64_t* n) {
  if (!s || !e || (!out && cap)) return hfail(OEMS_ERR_INVALID_ARGUMENT, "NULL argument");
  TermList L{out, cap};
  // src/processing/probes.rs:107-127: inclusive ranges, value 0 for other directions
  if (dir == 0)
    for (uint64_t i = s[0]; i <= e[0]; ++i) L.add(0, i, s[1], s[2], 1.0);
  else if (dir == 1)
    for (uint64_t j = s[1]; j <= e[1]; ++j) L.add(1, s[0], j, s[2], 1.0);
  else if (dir == 2)
    for (uint64_t k = s[2]; k <= e[2]; ++k) L.add(2, s[0], s[1], k, 1.0);
  return finish(L, n);
}

oems_status oems_probe_current_terms(const uint64_t s[3], const uint64_t e[3], int32_t normal, oems_probe_term* out,
                                     uint64_t cap, uint64_t* n) {
  if (!s || !e || (!out && cap)) return hfail(OEMS_ERR_INVALID_ARGUMENT, "NULL argument");
  TermList L{out, cap};
  // src/processing/probes.rs:204-236: current += H_a; current -= H_b, in loop order
  if (normal == 0) {
    for (uint64_t j = s[1]; j <= e[1]; ++j)
      for (uint64_t k = s[2]; k <= e[2]; ++k) {
        L.add(4, s[0], j, k, 1.0);
        L.add(5, s[0], j, k, -1.0);
      }
  } else if (normal == 1) {
    for (uint64_t i = s[0]; i <= e[0]; ++i)
      for (uint64_t k = s[2]; k <= e[2]; ++k) {
        L.add(5, i, s[1], k, 1.0);
        L.add(3, i, s[1], k, -1.0);
      }
  } else if (normal == 2) {
    for (uint64_t i = s[0]; i <= e[0]; ++i)
      for (uint64_t j = s[1]; j <= e[1]; ++j) {
        L.add(3, i, j, s[2], 1.0);
        L.add(4, i, j, s[2], -1.0);
      }
  }
  return finish(L, n);
}

oems_status oems_probe_voltage_integral_terms(const oems_operator* op, const uint64_t s[3], const uint64_t t[3],
                                              oems_probe_term* out, uint64_t cap, uint64_t* n) {
  if (!op || !s || !t || (!out && cap)) return hfail(OEMS_ERR_INVALID_ARGUMENT, "NULL argument");
  TermList L{out, cap};
  // src/fdtd/engine_interface.rs:208-247 (x at (j_start, k_start), y at
  // (i_stop, k_start), z at (i_stop, j_stop); indices clamped to the grid)
  for (uint64_t i = std::min(s[0], t[0]); i < std::max(s[0], t[0]); ++i) {
    const uint64_t ic = std::min(i, op->n[0] - 1);
    L.add(0, ic, s[1], s[2], -grid_delta(op, 0, ic));
  }
  for (uint64_t j = std::min(s[1], t[1]); j < std::max(s[1], t[1]); ++j) {
    const uint64_t jc = std::min(j, op->n[1] - 1);
    L.add(1, t[0], jc, s[2], -grid_delta(op, 1, jc));
  }
  for (uint64_t k = std::min(s[2], t[2]); k < std::max(s[2], t[2]); ++k) {
    const uint64_t kc = std::min(k, op->n[2] - 1);
    L.add(2, t[0], t[1], kc, -grid_delta(op, 2, kc));
  }
  return finish(L, n);
}

oems_status oems_probe_current_integral_terms(const oems_operator* op, const uint64_t s[3], const uint64_t t[3],
                                              int32_t normal, oems_probe_term* out, uint64_t cap, uint64_t* n) {
  if (!op || !s || !t || (!out && cap)) return hfail(OEMS_ERR_INVALID_ARGUMENT, "NULL argument");
  TermList L{out, cap};
  // src/fdtd/engine_interface.rs:251-305
  const uint64_t a0 = std::min(s[0], t[0]), a1 = std::max(s[0], t[0]);
  const uint64_t b0 = std::min(s[1], t[1]), b1 = std::max(s[1], t[1]);
  const uint64_t c0 = std::min(s[2], t[2]), c1 = std::max(s[2], t[2]);
  if (normal == 0) {
    for (uint64_t j = b0; j < b1; ++j)
      for (uint64_t k = c0; k < c1; ++k) {
        const uint64_t jc = std::min(j, op->n[1] - 1), kc = std::min(k, op->n[2] - 1);
        L.add(4, s[0], jc, kc, grid_delta(op, 2, kc));
        L.add(5, s[0], jc, kc, -grid_delta(op, 1, jc));
      }
  } else if (normal == 1) {
    for (uint64_t i = a0; i < a1; ++i)
      for (uint64_t k = c0; k < c1; ++k) {
        const uint64_t ic = std::min(i, op->n[0] - 1), kc = std::min(k, op->n[2] - 1);
        L.add(5, ic, s[1], kc, grid_delta(op, 0, ic));
        L.add(3, ic, s[1], kc, -grid_delta(op, 2, kc));
      }
  } else {
    for (uint64_t i = a0; i < a1; ++i)
      for (uint64_t j = b0; j < b1; ++j) {
        const uint64_t ic = std::min(i, op->n[0] - 1), jc = std::min(j, op->n[1] - 1);
        L.add(3, ic, jc, s[2], grid_delta(op, 1, jc));
        L.add(4, ic, jc, s[2], -grid_delta(op, 0, ic));
      }
  }
  return finish(L, n);
}

oems_status oems_probe_port_terms(const oems_operator* op, const uint64_t p[3], int32_t dir, int32_t kind,
                                  oems_probe_term* out, uint64_t cap, uint64_t* n) {
  if (!op || !p || (!out && cap)) return hfail(OEMS_ERR_INVALID_ARGUMENT, "NULL argument");
  if (dir < 0 || dir > 2) return hfail(OEMS_ERR_CONFIG, "port direction must be 0, 1 or 2");
  for (int a = 0; a < 3; ++a)
    if (p[a] >= op->n[a]) return hfail(OEMS_ERR_CONFIG, "port position outside the grid");
  TermList L{out, cap};
  if (kind == 0) {
    L.add(dir, p[0], p[1], p[2], -grid_delta(op, dir, p[dir]));
    return finish(L, n);
  }
  // the curl of H driving E[dir] at p (the E update's curl, times cell sides)
  const int a = (dir + 1) % 3, b = (dir + 2) % 3;  // H_b varies along a, H_a along b
  if (p[a] == 0 || p[b] == 0) return hfail(OEMS_ERR_CONFIG, "port current needs a cell before the edge");
  uint64_t m[3] = {p[0], p[1], p[2]};
  // + (H_b(p) - H_b(p - e_a)) * d_b   - (H_a(p) - H_a(p - e_b)) * d_a
  const double db = grid_delta(op, b, p[b]), da = grid_delta(op, a, p[a]);
  L.add(3 + b, p[0], p[1], p[2], db);
  m[a] -= 1;
  L.add(3 + b, m[0], m[1], m[2], -db);
  m[a] += 1;
  L.add(3 + a, p[0], p[1], p[2], -da);
  m[b] -= 1;
  L.add(3 + a, m[0], m[1], m[2], da);
  return finish(L, n);
}

oems_status oems_simulation_create(const oems_operator* op, int32_t device, uint32_t flags, oems_simulation** out) {
  if (!op || !out) return hfail(OEMS_ERR_INVALID_ARGUMENT, "NULL argument");
  std::unique_ptr<oems_simulation> s(new oems_simulation);
  s->op = *op;
  s->device = device;
  s->flags = flags;
  *out = s.release();
  return OEMS_OK;
}

void oems_simulation_destroy(oems_simulation* sim) {
  if (!sim) return;
  if (sim->engine) oems_engine_destroy(sim->engine);
  delete sim;
}

oems_status oems_simulation_add_excitation(oems_simulation* sim, const oems_excitation* exc) {
  if (!sim || !exc) return hfail(OEMS_ERR_INVALID_ARGUMENT, "NULL argument");
  sim->excitations.push_back(*exc);
  return OEMS_OK;
}

oems_status oems_simulation_set_end_condition(oems_simulation* sim, int32_t kind, double value) {
  if (!sim) return hfail(OEMS_ERR_INVALID_ARGUMENT, "NULL simulation");
  if (kind < OEMS_END_TIMESTEPS || kind > OEMS_END_SIMULATION_TIME) return hfail(OEMS_ERR_CONFIG, "unknown end condition");
  sim->end_kind = kind;
  sim->end_value = value;
  return OEMS_OK;
}

oems_status oems_simulation_set_batch_size(oems_simulation* sim, uint64_t batch_size) {
  if (!sim) return hfail(OEMS_ERR_INVALID_ARGUMENT, "NULL simulation");
  sim->batch_size = batch_size;
  return OEMS_OK;
}

oems_status oems_simulation_set_cpml(oems_simulation* sim, const oems_cpml_desc* cpml) {
  if (!sim || !cpml) return hfail(OEMS_ERR_INVALID_ARGUMENT, "NULL argument");
  if (sim->engine) return hfail(OEMS_ERR_CONFIG, "Simulation already set up");
  sim->has_cpml = true;
  sim->cpml = *cpml;
  return OEMS_OK;
}

// src/fdtd/simulation.rs:164-197
oems_status oems_simulation_setup(oems_simulation* sim) {
  if (!sim) return hfail(OEMS_ERR_INVALID_ARGUMENT, "NULL simulation");
  if (sim->engine) return hfail(OEMS_ERR_CONFIG, "Simulation already set up");
  oems_operator_desc d;
  oems_status st = oems_operator_engine_desc(&sim->op, sim->device, sim->flags, &d);
  if (st != OEMS_OK) return st;
  oems_engine* en = nullptr;
  st = oems_engine_create(&d, &en);
  if (st != OEMS_OK) return st;
  if (sim->has_cpml) {
    st = oems_engine_add_cpml(en, &sim->cpml);
    if (st != OEMS_OK) {
      oems_engine_destroy(en);
      return st;
    }
  }
  sim->engine = en;
  return OEMS_OK;
}

// src/fdtd/simulation.rs:200-360.  One deliberate difference: the peak energy
// found by earlier batches is handed to the next batch, so an EnergyDecay end
// condition can trigger (the reference restarts the peak at 0 inside every
// batch, which with its 100-step batches makes the decay never fire).
oems_status oems_simulation_run(oems_simulation* sim, oems_simulation_stats* stats) {
  if (!sim) return hfail(OEMS_ERR_INVALID_ARGUMENT, "NULL simulation");
  if (!sim->engine) {
    oems_status st = oems_simulation_setup(sim);
    if (st != OEMS_OK) return st;
  }
  if (sim->ran) return hfail(OEMS_ERR_CONFIG, "Simulation not ready to run");
  sim->ran = true;
  const double dt = sim->op.dt;
  const uint64_t batch = sim->batch_size ? sim->batch_size : 1000;
  uint64_t max_steps = 0;
  bool has_decay = false;
  double thr = 0.0;
  switch (sim->end_kind) {
    case OEMS_END_TIMESTEPS: max_steps = (uint64_t)sim->end_value; break;
    case OEMS_END_SIMULATION_TIME: max_steps = (uint64_t)std::ceil(sim->end_value / dt); break;
    default:
      max_steps = 1000000;
      has_decay = true;
      thr = sim->end_value;
  }
  const auto t0 = std::chrono::steady_clock::now();
  double peak = 0.0;
  uint64_t run = 0;
  std::vector<std::vector<float>> samples(sim->excitations.size());
  std::vector<oems_scheduled_excitation> sched(sim->excitations.size());
  std::vector<oems_energy_sample> es(64);
  while (run < max_steps) {
    const uint64_t this_batch = std::min(max_steps - run, batch);
    for (size_t x = 0; x < sim->excitations.size(); ++x) {
      const oems_excitation& e = sim->excitations[x];
      samples[x].resize(this_batch);
      oems_excitation_sample(&e, run, this_batch, dt, samples[x].data());
      sched[x] = oems_scheduled_excitation{};
      for (int a = 0; a < 3; ++a) sched[x].position[a] = e.position[a];
      sched[x].direction = e.direction;
      sched[x].soft_source = e.soft_source ? 1 : 0;
      sched[x].samples = samples[x].data();
      sched[x].num_samples = this_batch;
    }
    oems_batch b{};
    b.num_steps = this_batch;
    b.excitations = sched.data();
    b.num_excitations = (uint32_t)sched.size();
    b.has_energy_decay_db = has_decay ? 1 : 0;
    b.energy_decay_db = thr;
    b.check_interval = 100;
    b.sample_interval = 100;
    b.track_peak = 1;
    b.initial_peak_energy = peak;
    oems_batch_result r{};
    es.resize(this_batch / 100 + 2);
    r.energy_samples = es.data();
    r.energy_capacity = es.size();
    oems_status st = oems_engine_run_batch(sim->engine, &b, &r);
    if (st != OEMS_OK) return st;
    run += r.timesteps_executed;
    peak = std::max(peak, r.peak_energy);
    if (r.termination_reason != OEMS_TERMINATION_STEPS_COMPLETED) break;
    if (r.timesteps_executed == 0) break;
  }
  const double wall = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
  double e = 0.0, h = 0.0;
  oems_status st = oems_engine_energy(sim->engine, &e, &h);
  if (st != OEMS_OK) return st;
  if (stats) {
    const double cells = (double)sim->op.n[0] * (double)sim->op.n[1] * (double)sim->op.n[2];
    stats->timesteps = run;
    stats->sim_time = (double)run * dt;
    stats->wall_time = wall;
    stats->peak_energy = peak;
    stats->final_energy = e + h;
    stats->speed_mcells_per_sec = wall > 0.0 ? (double)run * cells / wall / 1e6 : 0.0;
  }
  return OEMS_OK;
}

oems_engine* oems_simulation_engine(oems_simulation* sim) { return sim ? sim->engine : nullptr; }

}  // extern "C"
