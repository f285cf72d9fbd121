// cylindrical.cu -- the cylindrical-coordinate FDTD engine (rho, alpha, z).
//
// Restates CylindricalEngine (src/fdtd/cylindrical.rs:394-638) on the GPU:
// per-cell coefficients vi = dt / (eps0 area) and iv = dt / (mu0 length)
// (computed on the host, openems_b200/cylindrical.py), vv = ii = 1, curls
// as plain differences with clamped edges and alpha wrap-around on a closed
// mesh, and the R = 0 fix-up after the voltage update (E_alpha = 0,
// E_z(0) = E_z(1) / 2).  The voltage pass reads only H and the current pass
// only E, so one thread per cell gives the reference's sequential loops bit
// for bit; products and sums are rounded separately as the reference's f32.
// Layout: [rho][alpha][z], z fastest, no padding.

#include <cuda_runtime.h>
#include <stdint.h>

#include <nvtx3/nvToolsExt.h>

#include <algorithm>
#include <string>

#include "../../include/oems.h"

namespace oems {
extern thread_local std::string g_last_error;
}

struct oems_cyl_engine {
  int device = 0;
  cudaStream_t stream = nullptr;
  long long nr = 0, na = 0, nz = 0, n = 0;
  int closed = 0, r0 = 0;
  double dt = 0.0, time = 0.0;
  uint64_t timestep = 0;
  float* buf = nullptr;  // E[3] H[3] vi[3] iv[3], n floats each
  cudaEvent_t ev[2] = {nullptr, nullptr};
  float last_ms = 0.0f;  // device time of the last oems_cyl_step
  float* at(int a) const { return buf + (size_t)a * n; }
};

namespace {

oems_status cfail(oems_status st, const std::string& m) {
  oems::g_last_error = m;
  return st;
}

#define CYL_CUDA(x)                                                              \
  do {                                                                           \
    cudaError_t e_ = (x);                                                        \
    if (e_ != cudaSuccess) return cfail(OEMS_ERR_CUDA, cudaGetErrorString(e_)); \
  } while (0)

constexpr int kCylRowThreads = 128;  // z cells per block in the row form
constexpr unsigned kCylRowMinZ = 128;  // shorter z rows use the flat form

struct CylArgs {
  float* e[3];
  float* h[3];
  const float* co[3];  // vi (voltage pass) or iv (current pass)
  unsigned nr, na, nz;  // n_rho * n_alpha * n_z <= 1.5e9 (checked at create)
  int closed, r0;
};

// One cell of update_voltage (src/fdtd/cylindrical.rs:422-497).  H and vi
// are read-only during the pass.
__device__ __forceinline__ void voltage_cell(const CylArgs& a, unsigned i, unsigned j, unsigned k) {
  const unsigned q = (i * a.na + j) * a.nz + k;
  const unsigned jp = j == 0 ? (a.closed ? a.na - 1 : 0) : j - 1;
  const unsigned kp = k > 0 ? k - 1 : 0, ip = i > 0 ? i - 1 : 0;
  const unsigned qj = (i * a.na + jp) * a.nz + k, qk = q - k + kp, qi = (ip * a.na + j) * a.nz + k;
  const float* __restrict__ hr = a.h[0];
  const float* __restrict__ ha = a.h[1];
  const float* __restrict__ hz = a.h[2];
  const float hr_q = __ldg(hr + q), ha_q = __ldg(ha + q), hz_q = __ldg(hz + q);
  const bool axis = i == 0 && a.r0;
  const float c_rho = axis ? 0.0f : __fsub_rn(__fsub_rn(hz_q, __ldg(hz + qj)), __fsub_rn(ha_q, __ldg(ha + qk)));
  const float c_alpha = __fsub_rn(__fsub_rn(hr_q, __ldg(hr + qk)), __fsub_rn(hz_q, __ldg(hz + qi)));
  const float c_z = axis ? 0.0f : __fsub_rn(__fsub_rn(ha_q, __ldg(ha + qi)), __fsub_rn(hr_q, __ldg(hr + qj)));
  a.e[0][q] = __fadd_rn(a.e[0][q], __fmul_rn(__ldg(a.co[0] + q), c_rho));
  a.e[1][q] = __fadd_rn(a.e[1][q], __fmul_rn(__ldg(a.co[1] + q), c_alpha));
  a.e[2][q] = __fadd_rn(a.e[2][q], __fmul_rn(__ldg(a.co[2] + q), c_z));
}

// One cell of update_current (src/fdtd/cylindrical.rs:524-591).  E and iv
// are read-only during the pass.
__device__ __forceinline__ void current_cell(const CylArgs& a, unsigned i, unsigned j, unsigned k) {
  const unsigned q = (i * a.na + j) * a.nz + k;
  const unsigned jn = j + 1 >= a.na ? (a.closed ? 0 : a.na - 1) : j + 1;
  const unsigned kn = k + 1 < a.nz ? k + 1 : a.nz - 1, in = i + 1 < a.nr ? i + 1 : a.nr - 1;
  const unsigned qj = (i * a.na + jn) * a.nz + k, qk = q - k + kn, qi = (in * a.na + j) * a.nz + k;
  const float* __restrict__ er = a.e[0];
  const float* __restrict__ ea = a.e[1];
  const float* __restrict__ ez = a.e[2];
  const float er_q = __ldg(er + q), ea_q = __ldg(ea + q), ez_q = __ldg(ez + q);
  const float c_rho = __fsub_rn(__fsub_rn(__ldg(ea + qk), ea_q), __fsub_rn(__ldg(ez + qj), ez_q));
  const float c_alpha = __fsub_rn(__fsub_rn(__ldg(ez + qi), ez_q), __fsub_rn(__ldg(er + qk), er_q));
  const float c_z = __fsub_rn(__fsub_rn(__ldg(er + qj), er_q), __fsub_rn(__ldg(ea + qi), ea_q));
  a.h[0][q] = __fadd_rn(a.h[0][q], __fmul_rn(__ldg(a.co[0] + q), c_rho));
  a.h[1][q] = __fadd_rn(a.h[1][q], __fmul_rn(__ldg(a.co[1] + q), c_alpha));
  a.h[2][q] = __fadd_rn(a.h[2][q], __fmul_rn(__ldg(a.co[2] + q), c_z));
}

// Flat form: one thread per cell over the whole array (short z rows).
template <bool kVoltage>
__global__ void __launch_bounds__(256) k_cyl_flat(const CylArgs a) {
  const unsigned n = a.nr * a.na * a.nz;
  for (unsigned q = blockIdx.x * blockDim.x + threadIdx.x; q < n; q += gridDim.x * blockDim.x) {
    const unsigned k = q % a.nz, ij = q / a.nz, j = ij % a.na, i = ij / a.na;
    if (kVoltage)
      voltage_cell(a, i, j, k);
    else
      current_cell(a, i, j, k);
  }
}

// Row form: blockIdx.y walks the (rho, alpha) rows, threads the z cells of
// a row, so no per-cell division and every row access is coalesced.
template <bool kVoltage>
__global__ void __launch_bounds__(kCylRowThreads) k_cyl_rows(const CylArgs a) {
  const unsigned rows = a.nr * a.na;
  for (unsigned row = blockIdx.y; row < rows; row += gridDim.y) {
    const unsigned i = row / a.na, j = row - i * a.na;
    for (unsigned k = blockIdx.x * blockDim.x + threadIdx.x; k < a.nz; k += gridDim.x * blockDim.x) {
      if (kVoltage)
        voltage_cell(a, i, j, k);
      else
        current_cell(a, i, j, k);
    }
  }
}

// src/fdtd/cylindrical.rs:499-520, after the voltage pass
__global__ void k_cyl_r0(const CylArgs a) {
  const unsigned m = a.na * a.nz;
  for (unsigned t = blockIdx.x * blockDim.x + threadIdx.x; t < m; t += gridDim.x * blockDim.x) {
    a.e[1][t] = 0.0f;                            // (0, j, k)
    a.e[2][t] = __fmul_rn(a.e[2][m + t], 0.5f);  // E_z(1, j, k) / 2
  }
}

CylArgs args(const oems_cyl_engine* en, bool voltage) {
  CylArgs a{};
  for (int c = 0; c < 3; ++c) {
    a.e[c] = en->at(c);
    a.h[c] = en->at(3 + c);
    a.co[c] = en->at(voltage ? 6 + c : 9 + c);
  }
  a.nr = (unsigned)en->nr;
  a.na = (unsigned)en->na;
  a.nz = (unsigned)en->nz;
  a.closed = en->closed;
  a.r0 = en->r0;
  return a;
}

int grid_of(long long n) { return (int)std::min<long long>((n + 255) / 256, 148 * 16); }

struct Dev {
  int prev = -1;
  explicit Dev(int d) {
    cudaGetDevice(&prev);
    if (prev != d) cudaSetDevice(d);
  }
  ~Dev() {
    if (prev >= 0) cudaSetDevice(prev);
  }
};

}  // namespace

extern "C" {

oems_status oems_cyl_create(const oems_cyl_desc* d, oems_cyl_engine** out) {
  if (!d || !out) return cfail(OEMS_ERR_INVALID_ARGUMENT, "NULL argument");
  *out = nullptr;
  if (d->n_rho == 0 || d->n_alpha == 0 || d->n_z == 0) return cfail(OEMS_ERR_GRID, "grid dimensions must be positive");
  if (d->r0_included && d->n_rho < 2) return cfail(OEMS_ERR_GRID, "a grid through R = 0 needs two rho cells");
  if ((double)d->n_rho * d->n_alpha * d->n_z > 1.5e9) return cfail(OEMS_ERR_GRID, "grid too large");
  for (int c = 0; c < 3; ++c)
    if (!d->vi[c] || !d->iv[c]) return cfail(OEMS_ERR_INVALID_ARGUMENT, "coefficient array pointer is NULL");
  int dev = d->device;
  if (dev < 0) CYL_CUDA(cudaGetDevice(&dev));
  Dev g(dev);
  auto* en = new oems_cyl_engine;
  en->device = dev;
  en->nr = (long long)d->n_rho;
  en->na = (long long)d->n_alpha;
  en->nz = (long long)d->n_z;
  en->n = en->nr * en->na * en->nz;
  en->closed = d->closed_alpha ? 1 : 0;
  en->r0 = d->r0_included ? 1 : 0;
  en->dt = d->dt;
  const size_t bytes = (size_t)en->n * sizeof(float);
  cudaError_t e = cudaStreamCreateWithFlags(&en->stream, cudaStreamNonBlocking);
  if (e == cudaSuccess) e = cudaEventCreate(&en->ev[0]);
  if (e == cudaSuccess) e = cudaEventCreate(&en->ev[1]);
  if (e == cudaSuccess) e = cudaMalloc(&en->buf, 12 * bytes);
  if (e == cudaSuccess) e = cudaMemsetAsync(en->buf, 0, 6 * bytes, en->stream);
  for (int c = 0; c < 3 && e == cudaSuccess; ++c) {
    e = cudaMemcpyAsync(en->at(6 + c), d->vi[c], bytes, cudaMemcpyHostToDevice, en->stream);
    if (e == cudaSuccess) e = cudaMemcpyAsync(en->at(9 + c), d->iv[c], bytes, cudaMemcpyHostToDevice, en->stream);
  }
  if (e == cudaSuccess) e = cudaStreamSynchronize(en->stream);
  if (e != cudaSuccess) {
    oems_cyl_destroy(en);
    return cfail(OEMS_ERR_CUDA, cudaGetErrorString(e));
  }
  *out = en;
  return OEMS_OK;
}

void oems_cyl_destroy(oems_cyl_engine* en) {
  if (!en) return;
  Dev g(en->device);
  if (en->stream) cudaStreamSynchronize(en->stream);
  if (en->buf) cudaFree(en->buf);
  for (cudaEvent_t ev : en->ev)
    if (ev) cudaEventDestroy(ev);
  if (en->stream) cudaStreamDestroy(en->stream);
  delete en;
}

static oems_status cyl_launch(oems_cyl_engine* en, uint64_t steps) {
  Dev g(en->device);
  const CylArgs v = args(en, true), c = args(en, false);
  const int gn = grid_of(en->n), gr = grid_of(en->na * en->nz);
  const bool rows = (unsigned)en->nz >= kCylRowMinZ;
  const long long nrows = en->nr * en->na, per = (nrows + 65534) / 65535;  // gridDim.y <= 65535
  const dim3 grow((unsigned)((en->nz + kCylRowThreads - 1) / kCylRowThreads), (unsigned)((nrows + per - 1) / per));
  CYL_CUDA(cudaEventRecord(en->ev[0], en->stream));
  for (uint64_t s = 0; s < steps; ++s) {
    if (rows)
      k_cyl_rows<true><<<grow, kCylRowThreads, 0, en->stream>>>(v);
    else
      k_cyl_flat<true><<<gn, 256, 0, en->stream>>>(v);
    if (en->r0) k_cyl_r0<<<gr, 256, 0, en->stream>>>(v);
    if (rows)
      k_cyl_rows<false><<<grow, kCylRowThreads, 0, en->stream>>>(c);
    else
      k_cyl_flat<false><<<gn, 256, 0, en->stream>>>(c);
    en->timestep += 1;
    en->time += en->dt;
  }
  CYL_CUDA(cudaGetLastError());
  CYL_CUDA(cudaEventRecord(en->ev[1], en->stream));
  CYL_CUDA(cudaStreamSynchronize(en->stream));
  CYL_CUDA(cudaEventElapsedTime(&en->last_ms, en->ev[0], en->ev[1]));
  return OEMS_OK;
}

oems_status oems_cyl_step(oems_cyl_engine* en, uint64_t steps) {
  if (!en) return cfail(OEMS_ERR_INVALID_ARGUMENT, "NULL engine");
  nvtxRangePushA("oems_cyl_step");
  const oems_status st = cyl_launch(en, steps);
  nvtxRangePop();
  return st;
}

static oems_status cyl_copy(oems_cyl_engine* en, float* const* host6, bool to_host) {
  if (!en || !host6) return cfail(OEMS_ERR_INVALID_ARGUMENT, "NULL argument");
  Dev g(en->device);
  const size_t bytes = (size_t)en->n * sizeof(float);
  for (int c = 0; c < 6; ++c) {
    if (!host6[c]) return cfail(OEMS_ERR_INVALID_ARGUMENT, "field pointer is NULL");
    if (to_host)
      CYL_CUDA(cudaMemcpyAsync(host6[c], en->at(c), bytes, cudaMemcpyDeviceToHost, en->stream));
    else
      CYL_CUDA(cudaMemcpyAsync(en->at(c), host6[c], bytes, cudaMemcpyHostToDevice, en->stream));
  }
  CYL_CUDA(cudaStreamSynchronize(en->stream));
  return OEMS_OK;
}

oems_status oems_cyl_read_fields(oems_cyl_engine* en, float* const e[3], float* const h[3]) {
  if (!e || !h) return cfail(OEMS_ERR_INVALID_ARGUMENT, "NULL argument");
  float* all[6] = {e[0], e[1], e[2], h[0], h[1], h[2]};
  return cyl_copy(en, all, true);
}

oems_status oems_cyl_write_fields(oems_cyl_engine* en, const float* const e[3], const float* const h[3]) {
  if (!e || !h) return cfail(OEMS_ERR_INVALID_ARGUMENT, "NULL argument");
  float* all[6] = {const_cast<float*>(e[0]), const_cast<float*>(e[1]), const_cast<float*>(e[2]),
                   const_cast<float*>(h[0]), const_cast<float*>(h[1]), const_cast<float*>(h[2])};
  return cyl_copy(en, all, false);
}

oems_status oems_cyl_reset(oems_cyl_engine* en) {
  if (!en) return cfail(OEMS_ERR_INVALID_ARGUMENT, "NULL engine");
  Dev g(en->device);
  CYL_CUDA(cudaMemsetAsync(en->buf, 0, 6 * (size_t)en->n * sizeof(float), en->stream));
  CYL_CUDA(cudaStreamSynchronize(en->stream));
  en->timestep = 0;
  en->time = 0.0;
  return OEMS_OK;
}

oems_status oems_cyl_last_step_ms(const oems_cyl_engine* en, float* ms) {
  if (!en || !ms) return cfail(OEMS_ERR_INVALID_ARGUMENT, "NULL argument");
  *ms = en->last_ms;
  return OEMS_OK;
}

oems_status oems_cyl_time(const oems_cyl_engine* en, uint64_t* timestep, double* time) {
  if (!en) return cfail(OEMS_ERR_INVALID_ARGUMENT, "NULL engine");
  if (timestep) *timestep = en->timestep;
  if (time) *time = en->time;
  return OEMS_OK;
}

}  // extern "C"
