// engine.cu -- the B200 FDTD engine behind the C ABI in include/oems.h.
//
// One engine = one grid on one GPU.  All state (fields, coefficients, CPML psi,
// probe traces, energy samples, excitation waveforms) stays resident in HBM;
// the host only uploads the operator once, the sampled waveforms per batch, and
// reads back small results.  A batch is planned on the host into spans of
// timesteps between energy samples / termination checks; each span replays a
// captured CUDA graph (H kernel, E kernel, post-step kernel per timestep), so
// the per-step launch cost is that of graph nodes.
//
// Step order per timestep (src/fdtd/basic_engine.rs:83-147):
//   H update -> E update -> excitations -> probes -> timestep += 1 ->
//   energy sample if cur % sample_interval == 0 ->
//   energy-decay check if cur > 0 && cur % check_interval == 0.
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstring>

#include <nvtx3/nvToolsExt.h>  // header-only; the ranges cost nothing without a profiler attached
#include <map>
#include <memory>
#include <mutex>
#include <string>
#include <tuple>
#include <type_traits>
#include <unordered_map>
#include <vector>

#include "../../include/oems.h"
#include "../../include/oems_host.h"
#include "yee_kernels.cuh"
#include "yee_pipe.cuh"
#include "yee_tma.cuh"
#include "mur.cuh"
#include "lumped_ade.cuh"
#include "fd_nf2ff.cuh"
#include "upml.cuh"
#include "interface.cuh"

namespace oems {

// ---------------------------------------------------------------------------
// error plumbing
// ---------------------------------------------------------------------------

thread_local std::string g_last_error;

static oems_status fail(oems_status st, const std::string& msg) {
  g_last_error = msg;
  return st;
}

#define OEMS_CUDA(call)                                                                        \
  do {                                                                                         \
    cudaError_t err_ = (call);                                                                 \
    if (err_ != cudaSuccess) {                                                                 \
      return fail(OEMS_ERR_CUDA, std::string(#call) + ": " + cudaGetErrorString(err_));       \
    }                                                                                          \
  } while (0)

#define OEMS_TRY(expr)              \
  do {                              \
    oems_status st_ = (expr);       \
    if (st_ != OEMS_OK) return st_; \
  } while (0)

// ---------------------------------------------------------------------------
// small device kernels
// ---------------------------------------------------------------------------

// Post-step work of one timestep: excitations (serially, in list order, so
// duplicate positions behave like the reference's sequential loop,
// basic_engine.rs:318-394), then probes.  A probe is a list of terms
// (component, cell, weight): mode 0 sums the values in order in f32 with
// weights +-1 (VoltageProbe / CurrentProbe::sample, src/processing/probes.rs:
// 98-239), mode 1 sums weight * value in f64 (EngineInterface integrals,
// src/fdtd/engine_interface.rs:208-305).  Traces are f64.
struct PostArgs {
  float* e[3];
  const float* h[3];
  int nexc;
  const long long* exc_idx;    // device linear index (padded layout)
  const int* exc_meta;         // dir | soft << 2
  const long long* exc_off;    // offset into exc_samples
  const long long* exc_count;  // number of samples
  const float* exc_samples;
  int nprobe;
  const int* probe_off;        // [nprobe + 1] term ranges
  const int* probe_mode;
  const long long* term_idx;
  const int* term_comp;
  const double* term_w;
  double* traces;              // [batch step][probe]
  const long long* d_base;     // batch step of local step 0
  int local;
  float h_inv;                 // 2-byte storage: 1 / the H scale
};

// One field value of component c at linear index q (H stored scaled in the
// 2-byte storage modes: multiplied back by h_inv, a power of two).
template <typename T>
__device__ __forceinline__ float field_value(const PostArgs& a, int c, long long q) {
  if constexpr (std::is_same<T, float>::value) {
    return (c < 3 ? a.e[c] : a.h[c - 3])[q];
  } else {
    const float v = FieldIO<T>::ld1(c < 3 ? a.e[c] : a.h[c - 3], q);
    return c < 3 ? v : v * a.h_inv;
  }
}

// Post-step work of batch step s (one CTA).
template <typename T>
__device__ __forceinline__ void post_step_body(const PostArgs& a, long long s) {
  if (threadIdx.x == 0) {
    for (int x = 0; x < a.nexc; ++x) {
      if (s >= a.exc_count[x]) continue;
      const float v = a.exc_samples[a.exc_off[x] + s];
      const int meta = a.exc_meta[x];
      if constexpr (std::is_same<T, float>::value) {
        float* p = a.e[meta & 3] + a.exc_idx[x];
        *p = (meta >> 2) ? __fadd_rn(*p, v) : v;
      } else {
        float* b = a.e[meta & 3];
        const float cur = FieldIO<T>::ld1(b, a.exc_idx[x]);
        FieldIO<T>::st1(b, a.exc_idx[x], (meta >> 2) ? __fadd_rn(cur, v) : v);
      }
    }
  }
  __syncthreads();
  for (int p = threadIdx.x; p < a.nprobe; p += blockDim.x) {
    double val;
    if (a.probe_mode[p] == 0) {
      float acc = 0.0f;
      for (int t = a.probe_off[p]; t < a.probe_off[p + 1]; ++t) {
        const float v = field_value<T>(a, a.term_comp[t], a.term_idx[t]);
        acc = a.term_w[t] >= 0.0 ? __fadd_rn(acc, v) : __fsub_rn(acc, v);
      }
      val = (double)acc;
    } else {
      double acc = 0.0;
      for (int t = a.probe_off[p]; t < a.probe_off[p + 1]; ++t) {
        const float v = field_value<T>(a, a.term_comp[t], a.term_idx[t]);
        acc = __dadd_rn(acc, __dmul_rn(a.term_w[t], (double)v));
      }
      val = acc;
    }
    a.traces[s * a.nprobe + p] = val;
  }
}

template <typename T = float>
__global__ void k_post_step(const PostArgs a) {
  post_step_body<T>(a, *a.d_base + a.local);
}

// The post-step work of several grids (a pack): CTA b does grid b's.
template <typename T = float>
__global__ void k_post_step_pack(const PostArgs* args, const long long* d_base, int local) {
  post_step_body<T>(args[blockIdx.x], *d_base + local);
}

// Running DFT of probe traces over the steps of a batch
// (src/processing/fields_fd.rs:149-217): X(f) += x(t) exp(-j 2 pi f t) 2 dt,
// t = (t_after - half) dt.  One thread per (dft, frequency), steps in order.
struct DftArgs {
  int nentries;             // total (dft, frequency) pairs
  const int* entry_probe;   // probe of each pair
  const double* entry_freq;
  const double* entry_half;
  double* acc;              // [nentries][2]
  const double* traces;
  int nprobe;
  long long steps;
  long long t0;             // timestep before the batch
  double dt;
};

__global__ void k_probe_dft(const DftArgs a) {
  const int e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= a.nentries) return;
  const int p = a.entry_probe[e];
  const double f = a.entry_freq[e];
  const double scale = 2.0 * a.dt;
  double re = a.acc[2 * e], im = a.acc[2 * e + 1];
  for (long long s = 0; s < a.steps; ++s) {
    const double x = a.traces[s * a.nprobe + p];
    const double t = ((double)(a.t0 + s + 1) - a.entry_half[e]) * a.dt;
    double sn, cs;
    sincos(-2.0 * 3.14159265358979323846 * f * t, &sn, &cs);
    re += x * (cs * scale);
    im += x * (sn * scale);
  }
  a.acc[2 * e] = re;
  a.acc[2 * e + 1] = im;
}

__global__ void k_set_i64(long long* p, long long v) { *p = v; }

// TF/SF plane injection (src/extensions/tfsf.rs:241-355): every cell of one
// plane of one field component gets f + coef * v (add) or f - coef * v, v the
// 1D grid's value of batch step *d_base + local (computed on the host).
struct TfsfArgs {
  float* f;
  long long plane_off, s1, s2;  // first cell, strides of the two in-plane axes
  int n1, n2;
  float coef;
  int add;
  const float* samples;
  const long long* d_base;
  int local;
};

__global__ void k_tfsf_plane(const TfsfArgs a) {
  const float v = a.samples[*a.d_base + a.local];
  const float d = __fmul_rn(a.coef, v);
  const long long n = (long long)a.n1 * a.n2;
  for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < n; t += (long long)gridDim.x * blockDim.x) {
    const long long u = t / a.n2, w = t - u * a.n2;
    float* p = a.f + a.plane_off + u * a.s1 + w * a.s2;
    *p = a.add ? __fadd_rn(*p, d) : __fsub_rn(*p, d);
  }
}

// Energy: per-block partial sums of x^2 in f64 over one array (blockIdx.y),
// then a fixed-order final sum (deterministic run to run).
constexpr int kEnergyBlocks = 296;
constexpr int kEnergyThreads = 256;

struct EnergyArgs {
  const float* arr[6];
  long long n4;          // float4 count per array
  double* partials;      // [6][kEnergyBlocks]
};

template <typename T>
__device__ __forceinline__ void energy_partial_body(const EnergyArgs& a) {
  const float4* p = reinterpret_cast<const float4*>(a.arr[blockIdx.y]);
  double s = 0.0;
  for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < a.n4;
       t += (long long)gridDim.x * blockDim.x) {
    float4 v;
    if constexpr (std::is_same<T, float>::value)
      v = __ldcs(p + t);
    else
      v = FieldIO<T>::ldg4(a.arr[blockIdx.y], 4 * t);
    s += (double)v.x * (double)v.x + (double)v.y * (double)v.y + (double)v.z * (double)v.z +
         (double)v.w * (double)v.w;
  }
  __shared__ double red[kEnergyThreads];
  red[threadIdx.x] = s;
  __syncthreads();
  for (int w = kEnergyThreads / 2; w > 0; w >>= 1) {
    if ((int)threadIdx.x < w) red[threadIdx.x] += red[threadIdx.x + w];
    __syncthreads();
  }
  if (threadIdx.x == 0) a.partials[blockIdx.y * kEnergyBlocks + blockIdx.x] = red[0];
}

template <typename T = float>
__global__ void __launch_bounds__(kEnergyThreads) k_energy_partial(const EnergyArgs a) {
  energy_partial_body<T>(a);
}

// Several grids: blockIdx.z picks the grid; each grid's partition and sum
// order are those of k_energy_partial, so its energies are the same bits.
template <typename T = float>
__global__ void __launch_bounds__(kEnergyThreads) k_energy_partial_pack(const EnergyArgs* args) {
  energy_partial_body<T>(args[blockIdx.z]);
}

// out[0] = E energy, out[1] = H energy (each the sum over its 3 components in
// component order, like VectorField3D::energy, src/arrays/field.rs:314-316).
// h_inv2: 1 / the square of the H storage scale (1 for float storage; a
// power of two, so exact).
__device__ __forceinline__ void energy_final_body(const double* partials, double* out, double h_inv2) {
  __shared__ double comp[6];
  const int c = threadIdx.x;
  if (c < 6) {
    double s = 0.0;
    for (int b = 0; b < kEnergyBlocks; ++b) s += partials[c * kEnergyBlocks + b];
    comp[c] = c < 3 ? s : s * h_inv2;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    out[0] = comp[0] + comp[1] + comp[2];
    out[1] = comp[3] + comp[4] + comp[5];
  }
}

__global__ void k_energy_final(const double* partials, double* out, double h_inv2) {
  energy_final_body(partials, out, h_inv2);
}

// Several grids: CTA b sums grid b's partials into out[2 b], out[2 b + 1].
__global__ void k_energy_final_pack(const EnergyArgs* args, double* out, double h_inv2) {
  energy_final_body(args[blockIdx.x].partials, out + 2 * blockIdx.x, h_inv2);
}

// ---------------------------------------------------------------------------
// engine
// ---------------------------------------------------------------------------

// Launch shape of the update kernels.  tma = false: register kernels
// (yee_kernels.cuh) with `block` threads; tma = true: bulk-async staged
// kernels (yee_tma.cuh) with `nconsumer` + 32 threads and `smem` bytes.
struct LaunchShape {
  int block = 256;
  int ichunk = 8;
  int pf = 0;  // L2 prefetch distance (register kernels)
  // split: staged kernels (tma) on the interior box, register CPML kernels
  // with these settings on the x / y slabs
  bool split = false;
  // zsplit: plain register kernels (no CPML) on the CPML-free box and the
  // CPML kernels (sh_block, sh_ichunk) on every slab cell (x, y and z)
  bool zsplit = false;
  int occ = 0;      // register budget of the (interior) register kernels
  int sh_occ = 0;   // ... of the CPML slab kernels of a z-split
  // z-split only: the slab launch runs on a second stream beside the
  // interior launch (fork / join by events, captured into the graphs), the
  // interior grid cut by `cut` CTAs per SM to leave room for it
  bool fork = false;
  int cut = 0;
  int sh_block = 256, sh_ichunk = 8, grid_sh = 0, grid_se = 0;
  int grid_h = 0;
  int grid_e = 0;
  bool tma = false;
  // pipe: the pipelined register kernels (yee_pipe.cuh), 256 threads, one
  // CTA per SM, pipe_ns shared-memory stages
  bool pipe = false;
  int pipe_ns = 4;
  int nconsumer = 256;
  TmaGeom tg{};
  size_t smem = 0;
};

// ---------------------------------------------------------------------------
// device and pinned host memory
// ---------------------------------------------------------------------------
// An engine's device buffers come from one stream-ordered pool per device
// (cudaMallocFromPoolAsync / cudaFreeAsync on the engine's stream).  cudaFree
// waits for every stream of the device, so with several engines in flight
// (a sweep) each engine teardown would stall all the others; a stream-ordered
// free does not, and the freed blocks stay in the pool for the next engine
// (oems_release_cached_memory hands them back to the driver).  A buffer is
// allocated on the stream of the engine whose entry point is running
// (EngineScope); outside an engine it falls back to cudaMalloc / cudaFree.

thread_local cudaStream_t t_alloc_stream = nullptr;

constexpr int kMaxDevices = 64;
struct PoolTable {
  std::mutex mu;
  cudaMemPool_t pool[kMaxDevices] = {};
};
static PoolTable& pool_table() {
  static PoolTable t;
  return t;
}

static cudaError_t device_pool(int dev, bool create, cudaMemPool_t* out) {
  *out = nullptr;
  if (dev < 0 || dev >= kMaxDevices) return cudaErrorInvalidDevice;
  PoolTable& t = pool_table();
  std::lock_guard<std::mutex> lk(t.mu);
  if (!t.pool[dev] && create) {
    cudaMemPoolProps props{};
    props.allocType = cudaMemAllocationTypePinned;
    props.handleTypes = cudaMemHandleTypeNone;
    props.location.type = cudaMemLocationTypeDevice;
    props.location.id = dev;
    cudaMemPool_t p = nullptr;
    cudaError_t e = cudaMemPoolCreate(&p, &props);
    if (e != cudaSuccess) return e;
    uint64_t keep = UINT64_MAX;  // freed blocks stay for reuse until trimmed
    if ((e = cudaMemPoolSetAttribute(p, cudaMemPoolAttrReleaseThreshold, &keep)) != cudaSuccess) {
      cudaMemPoolDestroy(p);
      return e;
    }
    t.pool[dev] = p;
  }
  *out = t.pool[dev];
  return cudaSuccess;
}

// `bytes` of device memory ordered on stream s (the current device's pool).
static cudaError_t pool_alloc(void** p, size_t bytes, cudaStream_t s) {
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  cudaMemPool_t pool = nullptr;
  if ((e = device_pool(dev, true, &pool)) != cudaSuccess) return e;
  return cudaMallocFromPoolAsync(p, std::max<size_t>(bytes, 1), pool, s);
}

template <typename T>
struct DevBuf {
  T* p = nullptr;
  size_t n = 0;
  cudaStream_t s = nullptr;  // stream of a pooled allocation (null: cudaMalloc)
  DevBuf() = default;
  DevBuf(const DevBuf&) = delete;
  DevBuf& operator=(const DevBuf&) = delete;
  ~DevBuf() { release(); }
  void release() {
    if (p) {
      if (s)
        cudaFreeAsync(p, s);
      else
        cudaFree(p);
    }
    p = nullptr;
    n = 0;
    s = nullptr;
  }
  cudaError_t ensure(size_t count) {
    if (count <= n && p) return cudaSuccess;
    release();
    const size_t c = std::max<size_t>(count, 1);
    void* q = nullptr;
    cudaError_t e = t_alloc_stream ? pool_alloc(&q, c * sizeof(T), t_alloc_stream) : cudaMalloc(&q, c * sizeof(T));
    if (e != cudaSuccess) return e;
    p = static_cast<T*>(q);
    n = c;
    s = t_alloc_stream;
    return cudaSuccess;
  }
};

// Pinned host buffers are cached by power-of-two size class: cudaFreeHost
// synchronises the device like cudaFree.
struct PinnedCache {
  std::mutex mu;
  std::multimap<size_t, void*> free;
};
static PinnedCache& pinned_cache() {
  static PinnedCache c;
  return c;
}
static size_t pinned_class(size_t bytes) {
  size_t c = 4096;
  while (c < bytes) c <<= 1;
  return c;
}
static cudaError_t pinned_get(void** p, size_t bytes) {
  const size_t c = pinned_class(bytes);
  PinnedCache& pc = pinned_cache();
  {
    std::lock_guard<std::mutex> lk(pc.mu);
    auto it = pc.free.find(c);
    if (it != pc.free.end()) {
      *p = it->second;
      pc.free.erase(it);
      return cudaSuccess;
    }
  }
  return cudaMallocHost(p, c);
}
static void pinned_put(void* p, size_t bytes) {
  if (!p) return;
  PinnedCache& pc = pinned_cache();
  std::lock_guard<std::mutex> lk(pc.mu);
  pc.free.emplace(pinned_class(bytes), p);
}

struct DeviceGuard {
  int prev = -1;
  explicit DeviceGuard(int dev) {
    cudaGetDevice(&prev);
    if (prev != dev) cudaSetDevice(dev);
  }
  ~DeviceGuard() {
    int cur = -1;
    cudaGetDevice(&cur);
    if (prev >= 0 && cur != prev) cudaSetDevice(prev);
  }
};

struct CpmlHost {
  bool on = false;
  oems_cpml_desc desc{};
  CpmlArgs args{};
  DevBuf<float> prof;
  DevBuf<float> psi;  // one allocation holding every psi array
  std::vector<size_t> psi_sizes;
};

struct MurHost {
  bool on = false;
  MurArgs args{};
  DevBuf<float> state;  // v, ob, os: 3 x 2 x total
};

struct DispHost {
  DispArgs args{};
  std::unique_ptr<DevBuf<long long>> q{new DevBuf<long long>};
  std::unique_ptr<DevBuf<float>> state{new DevBuf<float>};  // st then pp
};

struct RlcHost {
  std::vector<long long> q;
  std::vector<int> dir;
  std::vector<float> v_vv, v_il;
  DevBuf<long long> d_q;
  DevBuf<int> d_dir;
  DevBuf<float> d_vv, d_vil, d_int;
};

// Per-batch twiddle table of one frequency-domain recorder: [step][f][4] and
// the steps that sample.
struct FdTable {
  DevBuf<double> tw;
  DevBuf<int> sampled;
  std::vector<double> h_tw;
  std::vector<int> h_sampled;
};

struct FieldDftHost {
  FieldDftArgs args{};
  std::vector<double> freqs;
  std::vector<int> comps;
  uint32_t interval = 1;
  std::unique_ptr<DevBuf<double>> acc{new DevBuf<double>};
  std::unique_ptr<FdTable> tab{new FdTable};
};

struct Nf2ffHost {
  Nf2ffAccArgs args{};
  long long lo[3], hi[3];
  int sign[6];
  std::vector<double> freqs;
  uint32_t interval = 1;
  std::unique_ptr<DevBuf<double>> acc{new DevBuf<double>};
  std::unique_ptr<FdTable> tab{new FdTable};
};

// TF/SF plane source: the 1D auxiliary grid lives on the host (it does not
// depend on the 3D fields); each batch uploads its per-step values at the
// boundary plane: [e_inc of every step | h_inc of every step].
struct TfsfHost {
  bool on = false;
  int kind = 0;  // 0 the reference's update, 1 corrected
  int prop = 0, e_axis = 1, h_axis = 2;
  long long pos = 10;
  double freq = 0.0, amp = 0.0, v = 0.0;
  std::vector<float> e1d, h1d;
  uint64_t t = 0;
  uint64_t cap = 0;  // steps per half of `samples`
  DevBuf<float> samples;
};

struct UpmlHost {
  bool on = false;
  UpmlArgs e{}, h{};                 // E (voltage) and H (current) halves
  DevBuf<float> coef, flux;          // [E coef | H coef], [E flux | H flux]
};

}  // namespace oems

struct oems_engine {
  int device = 0;
  cudaStream_t stream = nullptr;
  uint32_t flags = 0;
  oems::Geom g{};
  int nx = 0, ny = 0, nz = 0;
  double dt = 0.0;
  double delta[3] = {0, 0, 0};
  uint64_t timestep = 0;
  long long ncells_padded = 0;

  // fields and coefficients (one allocation each)
  float* fields = nullptr;  // 6 * ncells_padded
  float* coeffs = nullptr;  // 12 * ncells_padded (full mode)
  void* ids = nullptr;      // compressed mode
  int id_bytes = 0;         // 0 full, 1 uint8, 2 uint16
  float* table = nullptr;
  int ntable = 0;

  oems::CpmlHost cpml;
  oems::MurHost mur;
  std::vector<oems::DispHost> disp;
  oems::RlcHost rlc;
  oems::UpmlHost upml;
  oems::TfsfHost tfsf;
  std::vector<oems::FieldDftHost> fdumps;
  std::vector<oems::Nf2ffHost> boxes;

  // probes: term tables (host copies and device mirrors) and f64 traces
  std::vector<int> probe_off{0}, probe_mode, term_comp;
  std::vector<long long> term_idx;
  std::vector<double> term_w, probe_half;
  oems::DevBuf<int> d_probe_off, d_probe_mode, d_term_comp;
  oems::DevBuf<long long> d_term_idx;
  oems::DevBuf<double> d_term_w;
  oems::DevBuf<double> d_traces;
  uint64_t traces_steps = 0;
  int nprobe() const { return (int)probe_mode.size(); }
  // probe DFTs: one entry per (dft, frequency)
  std::vector<int> dft_first, dft_count;  // entry range of each dft
  std::vector<int> entry_probe;
  std::vector<double> entry_freq, entry_half;
  oems::DevBuf<int> d_entry_probe;
  oems::DevBuf<double> d_entry_freq, d_entry_half, d_dft_acc;

  // excitations for the current batch
  oems::DevBuf<long long> d_exc_idx, d_exc_off, d_exc_count;
  oems::DevBuf<int> d_exc_meta;
  oems::DevBuf<float> d_exc_samples;
  int nexc = 0;

  // energy
  oems::DevBuf<double> d_partials;
  oems::DevBuf<double> d_energy;  // [sample][2]
  double* h_energy = nullptr;     // pinned mirror (cached pinned buffer)
  size_t h_energy_cap = 0;        // samples

  oems::DevBuf<long long> d_base;
  oems::DevBuf<int> d_err;  // device error word (bounded waits that gave up)
  oems::DevBuf<unsigned long long> d_iface;  // queries and results of the interface reads, 8-byte words

  oems::LaunchShape shape;
  oems::Geom gs{};  // shell segments of a split shape
  bool tuned = false;
  std::vector<oems_tune_entry> tune_report;  // candidates timed by the last tuning

  // graphs keyed by span length; invalidated when any baked pointer changes
  std::map<int, cudaGraphExec_t> graphs;
  uint64_t graph_epoch = 0, built_epoch = ~0ull;

  // per-kernel profiling
  bool profiling = false;
  std::vector<cudaEvent_t> prof_ev;  // 4 per step: h0 h1 e0 e1
  double prof_h_s = 0.0, prof_e_s = 0.0;
  uint64_t prof_h_n = 0, prof_e_n = 0;

  uint64_t last_launches = 0;
  double last_device_seconds = 0.0;
  cudaEvent_t ev0 = nullptr, ev1 = nullptr;
  // second stream of a forked z-split and its fork / join events
  cudaStream_t side = nullptr;
  cudaEvent_t fork_ev = nullptr, join_ev = nullptr;

  // field storage: 0 float, 1 half, 2 bfloat16 (arithmetic in float); with
  // 2-byte storage H is kept multiplied by h_scale (a power of two)
  int storage = 0;
  size_t elem = sizeof(float);
  float h_scale = 1.0f;
  float* at(size_t c) { return reinterpret_cast<float*>(reinterpret_cast<char*>(fields) + c * ncells_padded * elem); }
  float* E(int c) { return at((size_t)c); }
  float* H(int c) { return at((size_t)(3 + c)); }
  size_t field_bytes() const { return 6 * (size_t)ncells_padded * elem; }
  float* C(int a) { return coeffs + (size_t)a * ncells_padded; }
};

namespace oems {

// Runs an entry point of an engine: its device is current and new buffers
// are allocated on its stream.
struct EngineScope {
  DeviceGuard dev;
  cudaStream_t prev;
  explicit EngineScope(const oems_engine* en) : dev(en->device), prev(t_alloc_stream) {
    t_alloc_stream = en->stream;
  }
  ~EngineScope() { t_alloc_stream = prev; }
};

static void drop_graphs(oems_engine* en) {
  for (auto& kv : en->graphs) cudaGraphExecDestroy(kv.second);
  en->graphs.clear();
}

static Geom make_geom(const oems_engine* en, int block, int ichunk) {
  Geom g{};
  g.nx = en->nx;
  g.ny = en->ny;
  g.nz = en->nz;
  g.nzp = (en->nz + 3) / 4 * 4;
  g.nzq = g.nzp / 4;
  g.plane = (long long)g.ny * g.nzp;
  g.plane4 = g.ny * g.nzq;
  g.tiles = (g.plane4 + block - 1) / block;
  g.ichunk = ichunk;
  g.nchunks = (g.nx + ichunk - 1) / ichunk;
  g.work = g.tiles * g.nchunks;
  g.nseg = 1;
  g.seg[0] = Seg{0, g.nx, 0, 0, g.nzq, g.plane4, g.tiles, 0};
  return g;
}

// Appends segment planes [i0, i1) x rows [j0, j1) x chunks [q0, q1) of each
// row (skipped when empty).
static void add_seg(Geom& g, int block, int ichunk, int i0, int i1, int j0, int j1, int q0, int q1) {
  if (i1 <= i0 || j1 <= j0 || q1 <= q0) return;
  Seg S;
  S.i0 = i0;
  S.i1 = i1;
  S.j0 = j0;
  S.q0 = q0;
  S.w = q1 - q0;
  S.n = (j1 - j0) * S.w;
  S.tiles = (S.n + block - 1) / block;
  S.work0 = g.work;
  g.work += S.tiles * ((i1 - i0 + ichunk - 1) / ichunk);
  g.seg[g.nseg++] = S;
}

// Chunks [qa, qb) of a row touch neither z slab: chunk q (cells 4q..4q+3)
// meets the z-min slab when 4q < L and the z-max slab when 4q + 3 >= its
// first cell.
static void zfree_chunks(const oems_engine* en, int* qa, int* qb) {
  const int nzq = (en->nz + 3) / 4;
  const CpmlArgs& cp = en->cpml.args;
  *qa = (cp.L[4] + 3) / 4;
  *qb = cp.L[5] > 0 ? (std::max(cp.start[5] - 3, 0) + 3) / 4 : nzq;
  *qb = std::min(*qb, nzq);
}

// Interior box between the x and y CPML slabs: planes [i_lo, i_hi), rows
// [j_lo, j_hi) (all of z).  Empty when the slabs leave nothing between them.
static bool cpml_interior(const oems_engine* en, int* i_lo, int* i_hi, int* j_lo, int* j_hi) {
  if (!en->cpml.on) return false;
  const CpmlArgs& cp = en->cpml.args;
  *i_lo = cp.L[0];
  *i_hi = en->nx - cp.L[1];
  *j_lo = cp.L[2];
  *j_hi = en->ny - cp.L[3];
  return *i_lo < *i_hi && *j_lo < *j_hi;
}

// The x / y slabs as register-kernel segments: whole planes of the x slabs,
// slab rows of the planes between them; with_z adds the z-slab chunks of the
// interior rows (the chunks the plain interior launch of a z-split leaves).
static Geom make_shell_geom(const oems_engine* en, int block, int ichunk, bool with_z = false) {
  Geom g = make_geom(en, block, ichunk);
  int ilo = 0, ihi = 0, jlo = 0, jhi = 0;
  cpml_interior(en, &ilo, &ihi, &jlo, &jhi);
  const int nq = g.nzq;
  g.nseg = 0;
  g.work = 0;
  add_seg(g, block, ichunk, 0, ilo, 0, g.ny, 0, nq);
  add_seg(g, block, ichunk, ihi, g.nx, 0, g.ny, 0, nq);
  add_seg(g, block, ichunk, ilo, ihi, 0, jlo, 0, nq);
  add_seg(g, block, ichunk, ilo, ihi, jhi, g.ny, 0, nq);
  if (with_z) {
    int qa = 0, qb = 0;
    zfree_chunks(en, &qa, &qb);
    qb = std::max(qa, qb);  // never twice over a chunk
    add_seg(g, block, ichunk, ilo, ihi, jlo, jhi, 0, qa);
    add_seg(g, block, ichunk, ilo, ihi, jlo, jhi, qb, nq);
  }
  return g;
}

// The CPML-free box: planes and rows between the x / y slabs, chunks clear
// of both z slabs, as one segment for the plain (no CPML) kernels.
static Geom make_interior_geom(const oems_engine* en, int block, int ichunk) {
  Geom g = make_geom(en, block, ichunk);
  g.nseg = 0;
  g.work = 0;
  int ilo = 0, ihi = 0, jlo = 0, jhi = 0;
  if (!cpml_interior(en, &ilo, &ihi, &jlo, &jhi)) return g;
  int qa = 0, qb = 0;
  zfree_chunks(en, &qa, &qb);
  add_seg(g, block, ichunk, ilo, ihi, jlo, jhi, qa, qb);
  return g;
}

// A z-split needs a non-empty CPML-free box.
static bool can_zsplit(const oems_engine* en) {
  return en->cpml.on && make_interior_geom(en, 256, 8).work > 0;
}

static HArgs h_args(oems_engine* en) {
  HArgs a{};
  a.g = en->g;
  a.ex = en->E(0);
  a.ey = en->E(1);
  a.ez = en->E(2);
  a.hx = en->H(0);
  a.hy = en->H(1);
  a.hz = en->H(2);
  if (en->id_bytes == 0) {
    for (int c = 0; c < 3; ++c) {
      a.da[c] = en->C(6 + c);
      a.db[c] = en->C(9 + c);
    }
  }
  a.ids = en->ids;
  a.table = en->table;
  a.ntable = en->ntable;
  a.cp = en->cpml.args;
  return a;
}

static EArgs e_args(oems_engine* en) {
  EArgs a{};
  a.g = en->g;
  a.ex = en->E(0);
  a.ey = en->E(1);
  a.ez = en->E(2);
  a.hx = en->H(0);
  a.hy = en->H(1);
  a.hz = en->H(2);
  if (en->id_bytes == 0) {
    for (int c = 0; c < 3; ++c) {
      a.ca[c] = en->C(c);
      a.cb[c] = en->C(3 + c);
    }
  }
  a.ids = en->ids;
  a.table = en->table;
  a.ntable = en->ntable;
  a.cp = en->cpml.args;
  return a;
}

using HKernel = void (*)(HArgs);
using EKernel = void (*)(EArgs);

template <typename T>
static HKernel pick_h_t(int id_bytes, bool cpml) {
  if (id_bytes == 0) return cpml ? k_update_h<0, true, T> : k_update_h<0, false, T>;
  if (id_bytes == 1) return cpml ? k_update_h<1, true, T> : k_update_h<1, false, T>;
  return cpml ? k_update_h<2, true, T> : k_update_h<2, false, T>;
}
template <typename T>
static EKernel pick_e_t(int id_bytes, bool cpml) {
  if (id_bytes == 0) return cpml ? k_update_e<0, true, T> : k_update_e<0, false, T>;
  if (id_bytes == 1) return cpml ? k_update_e<1, true, T> : k_update_e<1, false, T>;
  return cpml ? k_update_e<2, true, T> : k_update_e<2, false, T>;
}
// occ: register budget variant, 0 the uncapped kernels, 1 / 2 the capped
// ones (k_update_*_cap with 3 / 4 CTAs of 256 per SM), built for float
// storage and full coefficients, the benchmark's kernels; other variants
// ignore it.
static HKernel pick_h(int id_bytes, bool cpml, int storage = 0, int occ = 0) {
  if (storage == 1) return pick_h_t<__half>(id_bytes, cpml);
  if (storage == 2) return pick_h_t<__nv_bfloat16>(id_bytes, cpml);
  if (id_bytes == 0 && occ == 1) return cpml ? k_update_h_cap<true, 3> : k_update_h_cap<false, 3>;
  if (id_bytes == 0 && occ == 2) return cpml ? k_update_h_cap<true, 4> : k_update_h_cap<false, 4>;
  return pick_h_t<float>(id_bytes, cpml);
}
static EKernel pick_e(int id_bytes, bool cpml, int storage = 0, int occ = 0) {
  if (storage == 1) return pick_e_t<__half>(id_bytes, cpml);
  if (storage == 2) return pick_e_t<__nv_bfloat16>(id_bytes, cpml);
  if (id_bytes == 0 && occ == 1) return cpml ? k_update_e_cap<true, 3> : k_update_e_cap<false, 3>;
  if (id_bytes == 0 && occ == 2) return cpml ? k_update_e_cap<true, 4> : k_update_e_cap<false, 4>;
  return pick_e_t<float>(id_bytes, cpml);
}

static HKernel pick_h_pipe(bool cpml, int ns) {
  if (ns >= 4) return cpml ? k_update_h_pipe<true, 4> : k_update_h_pipe<false, 4>;
  return cpml ? k_update_h_pipe<true, 3> : k_update_h_pipe<false, 3>;
}
static EKernel pick_e_pipe(bool cpml, int ns) {
  if (ns >= 4) return cpml ? k_update_e_pipe<true, 4> : k_update_e_pipe<false, 4>;
  return cpml ? k_update_e_pipe<true, 3> : k_update_e_pipe<false, 3>;
}

// Stage count of the pipelined kernels for this grid (4, 3) or 0 where they
// do not apply: float fields, full coefficient arrays, a halo row of at most
// one CTA's chunks, and the stages within the opt-in shared memory.
static int pipe_stages(const oems_engine* en, size_t optin) {
  if (en->id_bytes != 0 || en->storage != 0) return 0;
  const int nzq = (en->nz + 3) / 4;
  if (nzq > kPipeThreads) return 0;
  for (int ns : {4, 3})
    if (pipe_smem_bytes(ns, nzq) <= optin) return ns;
  return 0;
}

static size_t table_smem(const oems_engine* en) {
  return en->id_bytes == 1 ? (size_t)en->ntable * 12 * sizeof(float) : 0;
}

// Stage layout of the bulk-staged kernels for tiles of TJ rows.  Returns the
// dynamic shared memory in bytes, 0 if fewer than 2 stages fit in `limit`.
static size_t make_tma_geom(const oems_engine* en, int TJ, int ichunk, int nconsumer, size_t limit, int ns_max,
                            TmaGeom& t, bool interior = false) {
  const int nzp = en->g.nzp;
  t = TmaGeom{};
  t.i_lo = 0;
  t.i_hi = en->nx;
  t.j_lo = 0;
  t.j_hi = en->ny;
  if (interior && !cpml_interior(en, &t.i_lo, &t.i_hi, &t.j_lo, &t.j_hi)) return 0;
  t.xy_psi = en->cpml.on && !interior;
  t.TJ = TJ;
  t.ntiles = (t.j_hi - t.j_lo + TJ - 1) / TJ;
  t.ichunk = ichunk;
  t.nitems = t.ntiles * ((t.i_hi - t.i_lo + ichunk - 1) / ichunk);
  t.nconsumer = nconsumer;
  int off = 0;
  t.off_f = off;
  off += 3 * (TJ + 1) * nzp;
  t.off_u = off;
  off += 3 * TJ * nzp;
  t.off_c = off;
  off += 6 * TJ * nzp;
  t.off_px = t.off_py = t.off_pz = off;
  if (en->cpml.on) {
    const CpmlArgs& cp = en->cpml.args;
    t.zwmax = std::max(cp.zw[0], cp.zw[1]);
    t.off_px = off;
    if (t.xy_psi) off += 2 * TJ * nzp;
    t.off_py = off;
    if (t.xy_psi) off += 2 * TJ * nzp;
    t.off_pz = off;
    off += 4 * TJ * t.zwmax;
    t.prof_floats = 0;
    for (int f = 0; f < 6; ++f) t.prof_floats += 6 * cp.L[f];
  }
  t.stage_floats = (off + 31) / 32 * 32;  // 128-byte aligned stages
  const size_t fixed = (size_t)((t.prof_floats + 3) / 4 * 4) * sizeof(float) + 64;
  int ns = 0;
  for (int s = ns_max; s >= 2; --s)
    if ((size_t)s * t.stage_floats * sizeof(float) + fixed + 2 * s * sizeof(uint64_t) <= limit) {
      ns = s;
      break;
    }
  if (ns == 0) return 0;
  t.NS = ns;
  return (size_t)ns * t.stage_floats * sizeof(float) + fixed + 2 * ns * sizeof(uint64_t);
}

static oems_status tma_smem_limit(const oems_engine* en, size_t* limit) {
  int optin = 0;
  OEMS_CUDA(cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, en->device));
  *limit = (size_t)optin;
  return OEMS_OK;
}

static oems_status prepare_tma_kernels(size_t smem) {
  OEMS_CUDA(cudaFuncSetAttribute((const void*)k_update_tma<true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)smem));
  OEMS_CUDA(cudaFuncSetAttribute((const void*)k_update_tma<false>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)smem));
  return OEMS_OK;
}

// Grid = resident CTAs (occupancy x SMs), capped by the work item count.
static oems_status size_grid(oems_engine* en, LaunchShape& s) {
  int sms = 0;
  OEMS_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, en->device));
  if (s.pipe) {
    const int nzq = (en->nz + 3) / 4;
    const size_t smem = pipe_smem_bytes(s.pipe_ns, nzq);
    const bool cp = en->cpml.on;
    // the attribute is per function and shared by every engine: allow up to
    // the opt-in limit, so a grid with wider rows never shrinks it under
    // another engine's launches
    size_t limit = 0;
    OEMS_TRY(tma_smem_limit(en, &limit));
    OEMS_CUDA(cudaFuncSetAttribute((const void*)pick_h_pipe(cp, s.pipe_ns),
                                   cudaFuncAttributeMaxDynamicSharedMemorySize, (int)limit));
    OEMS_CUDA(cudaFuncSetAttribute((const void*)pick_e_pipe(cp, s.pipe_ns),
                                   cudaFuncAttributeMaxDynamicSharedMemorySize, (int)limit));
    int oh = 0, oe = 0;
    OEMS_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&oh, (const void*)pick_h_pipe(cp, s.pipe_ns),
                                                            kPipeThreads, smem));
    OEMS_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&oe, (const void*)pick_e_pipe(cp, s.pipe_ns),
                                                            kPipeThreads, smem));
    s.block = kPipeThreads;
    s.smem = smem;
    const Geom g = make_geom(en, kPipeThreads, s.ichunk);
    s.grid_h = std::max(1, std::min(g.work, std::max(1, oh) * sms));
    s.grid_e = std::max(1, std::min(g.work, std::max(1, oe) * sms));
    return OEMS_OK;
  }
  if (s.tma) {
    // allow any stage count up to the opt-in limit (the attribute is per
    // function, shared by every engine and tuning candidate)
    size_t limit = 0;
    OEMS_TRY(tma_smem_limit(en, &limit));
    OEMS_TRY(prepare_tma_kernels(limit));
    int occ = 0;
    OEMS_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, (const void*)k_update_tma<true>,
                                                            s.nconsumer + 32, s.smem));
    s.grid_h = s.grid_e = std::max(1, std::min(s.tg.nitems, std::max(1, occ) * sms));
    if (s.split) {
      int oh = 0, oe = 0;
      OEMS_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&oh, (const void*)pick_h(0, true), s.sh_block, 0));
      OEMS_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&oe, (const void*)pick_e(0, true), s.sh_block, 0));
      const Geom gs = make_shell_geom(en, s.sh_block, s.sh_ichunk);
      s.grid_sh = std::max(1, std::min(gs.work, std::max(1, oh) * sms));
      s.grid_se = std::max(1, std::min(gs.work, std::max(1, oe) * sms));
    }
    return OEMS_OK;
  }
  const size_t smem = table_smem(en);
  int occ_h = 0, occ_e = 0;
  const bool mode = en->cpml.on && !s.zsplit;
  OEMS_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(
      &occ_h, (const void*)pick_h(en->id_bytes, mode, en->storage, s.occ), s.block, smem));
  OEMS_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(
      &occ_e, (const void*)pick_e(en->id_bytes, mode, en->storage, s.occ), s.block, smem));
  const Geom g = s.zsplit ? make_interior_geom(en, s.block, s.ichunk) : make_geom(en, s.block, s.ichunk);
  const int cut = s.zsplit && s.fork ? s.cut : 0;
  s.grid_h = std::max(1, std::min(g.work, std::max(1, occ_h - cut) * sms));
  s.grid_e = std::max(1, std::min(g.work, std::max(1, occ_e - cut) * sms));
  if (s.zsplit) {
    int oh = 0, oe = 0;
    OEMS_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(
        &oh, (const void*)pick_h(en->id_bytes, true, en->storage, s.sh_occ), s.sh_block, smem));
    OEMS_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(
        &oe, (const void*)pick_e(en->id_bytes, true, en->storage, s.sh_occ), s.sh_block, smem));
    const Geom gs = make_shell_geom(en, s.sh_block, s.sh_ichunk, true);
    s.grid_sh = std::max(1, std::min(gs.work, std::max(1, oh) * sms));
    s.grid_se = std::max(1, std::min(gs.work, std::max(1, oe) * sms));
  }
  return OEMS_OK;
}

static void apply_shape(oems_engine* en, const LaunchShape& s) {
  if (s.fork && !en->side) {
    // created on first use; failures leave the shape unforked
    if (cudaStreamCreateWithFlags(&en->side, cudaStreamNonBlocking) != cudaSuccess ||
        cudaEventCreateWithFlags(&en->fork_ev, cudaEventDisableTiming) != cudaSuccess ||
        cudaEventCreateWithFlags(&en->join_ev, cudaEventDisableTiming) != cudaSuccess)
      cudaGetLastError();
  }
  en->shape = s;
  if (s.fork && !(en->side && en->fork_ev && en->join_ev)) en->shape.fork = false;
  en->g = s.zsplit ? make_interior_geom(en, s.block, s.ichunk) : make_geom(en, s.block, s.ichunk);
  en->g.pf = (s.tma || s.pipe) ? 0 : s.pf;
  if (s.split || s.zsplit) en->gs = make_shell_geom(en, s.sh_block, s.sh_ichunk, s.zsplit);
  en->graph_epoch++;
}

static TmaArgs tma_args(oems_engine* en, bool is_h) {
  TmaArgs a{};
  a.g = en->g;
  a.t = en->shape.tg;
  for (int c = 0; c < 3; ++c) {
    a.f[c] = is_h ? en->E(c) : en->H(c);
    a.u[c] = is_h ? en->H(c) : en->E(c);
    a.c[c] = en->C(is_h ? 6 + c : c);
    a.c[3 + c] = en->C(is_h ? 9 + c : 3 + c);
  }
  a.cp = en->cpml.args;
  a.cpml = en->cpml.on;
  a.err = en->d_err.p;
  return a;
}

static cudaError_t launch_h(oems_engine* en) {
  if (en->shape.pipe) {
    HArgs a = h_args(en);
    pick_h_pipe(en->cpml.on, en->shape.pipe_ns)<<<en->shape.grid_h, kPipeThreads, en->shape.smem, en->stream>>>(a);
    return cudaGetLastError();
  }
  if (en->shape.tma) {
    TmaArgs a = tma_args(en, true);
    k_update_tma<true><<<en->shape.grid_h, en->shape.nconsumer + 32, en->shape.smem, en->stream>>>(a);
    if (en->shape.split) {
      HArgs b = h_args(en);
      b.g = en->gs;
      pick_h(0, true)<<<en->shape.grid_sh, en->shape.sh_block, 0, en->stream>>>(b);
    }
    return cudaGetLastError();
  }
  HArgs a = h_args(en);
  if (en->shape.zsplit) {
    const bool fork = en->shape.fork && en->gs.work > 0;
    cudaStream_t ss = fork ? en->side : en->stream;
    if (fork) {
      cudaEventRecord(en->fork_ev, en->stream);
      cudaStreamWaitEvent(ss, en->fork_ev, 0);
    }
    pick_h(en->id_bytes, false, en->storage, en->shape.occ)<<<en->shape.grid_h, en->shape.block, table_smem(en),
                                                              en->stream>>>(a);
    if (en->gs.work > 0) {
      HArgs b = a;
      b.g = en->gs;
      pick_h(en->id_bytes, true, en->storage, en->shape.sh_occ)<<<en->shape.grid_sh, en->shape.sh_block,
                                                                 table_smem(en), ss>>>(b);
    }
    if (fork) {
      cudaEventRecord(en->join_ev, ss);
      cudaStreamWaitEvent(en->stream, en->join_ev, 0);
    }
    return cudaGetLastError();
  }
  pick_h(en->id_bytes, en->cpml.on, en->storage, en->shape.occ)<<<en->shape.grid_h, en->shape.block, table_smem(en),
                                                                  en->stream>>>(a);
  return cudaGetLastError();
}
static cudaError_t launch_e(oems_engine* en) {
  if (en->shape.pipe) {
    EArgs a = e_args(en);
    pick_e_pipe(en->cpml.on, en->shape.pipe_ns)<<<en->shape.grid_e, kPipeThreads, en->shape.smem, en->stream>>>(a);
    return cudaGetLastError();
  }
  if (en->shape.tma) {
    TmaArgs a = tma_args(en, false);
    k_update_tma<false><<<en->shape.grid_e, en->shape.nconsumer + 32, en->shape.smem, en->stream>>>(a);
    if (en->shape.split) {
      EArgs b = e_args(en);
      b.g = en->gs;
      pick_e(0, true)<<<en->shape.grid_se, en->shape.sh_block, 0, en->stream>>>(b);
    }
    return cudaGetLastError();
  }
  EArgs a = e_args(en);
  if (en->shape.zsplit) {
    const bool fork = en->shape.fork && en->gs.work > 0;
    cudaStream_t ss = fork ? en->side : en->stream;
    if (fork) {
      cudaEventRecord(en->fork_ev, en->stream);
      cudaStreamWaitEvent(ss, en->fork_ev, 0);
    }
    pick_e(en->id_bytes, false, en->storage, en->shape.occ)<<<en->shape.grid_e, en->shape.block, table_smem(en),
                                                              en->stream>>>(a);
    if (en->gs.work > 0) {
      EArgs b = a;
      b.g = en->gs;
      pick_e(en->id_bytes, true, en->storage, en->shape.sh_occ)<<<en->shape.grid_se, en->shape.sh_block,
                                                                 table_smem(en), ss>>>(b);
    }
    if (fork) {
      cudaEventRecord(en->join_ev, ss);
      cudaStreamWaitEvent(en->stream, en->join_ev, 0);
    }
    return cudaGetLastError();
  }
  pick_e(en->id_bytes, en->cpml.on, en->storage, en->shape.occ)<<<en->shape.grid_e, en->shape.block, table_smem(en),
                                                                  en->stream>>>(a);
  return cudaGetLastError();
}

static int post_kernels(const oems_engine* en) {
  return (en->nexc > 0 || en->nprobe() > 0 ? 1 : 0) + (int)en->fdumps.size() + (int)en->boxes.size();
}
static bool need_post(const oems_engine* en) { return post_kernels(en) > 0; }

static cudaError_t launch_fd(oems_engine* en, int local) {
  for (FieldDftHost& d : en->fdumps) {
    FieldDftArgs a = d.args;
    a.tw = d.tab->tw.p;
    a.sampled = d.tab->sampled.p;
    a.d_base = en->d_base.p;
    a.local = local;
    k_field_dft<<<(int)((a.npts + 255) / 256), 256, 0, en->stream>>>(a);
  }
  for (Nf2ffHost& b : en->boxes) {
    Nf2ffAccArgs a = b.args;
    a.tw = b.tab->tw.p;
    a.sampled = b.tab->sampled.p;
    a.d_base = en->d_base.p;
    a.local = local;
    k_nf2ff_acc<<<(int)((a.off[a.nfaces] + 255) / 256), 256, 0, en->stream>>>(a);
  }
  return cudaGetLastError();
}

static cudaError_t launch_post(oems_engine* en, int local) {
  if (en->nexc == 0 && en->nprobe() == 0) return launch_fd(en, local);
  PostArgs a{};
  for (int c = 0; c < 3; ++c) {
    a.e[c] = en->E(c);
    a.h[c] = en->H(c);
  }
  a.nexc = en->nexc;
  a.exc_idx = en->d_exc_idx.p;
  a.exc_meta = en->d_exc_meta.p;
  a.exc_off = en->d_exc_off.p;
  a.exc_count = en->d_exc_count.p;
  a.exc_samples = en->d_exc_samples.p;
  a.nprobe = en->nprobe();
  a.probe_off = en->d_probe_off.p;
  a.probe_mode = en->d_probe_mode.p;
  a.term_idx = en->d_term_idx.p;
  a.term_comp = en->d_term_comp.p;
  a.term_w = en->d_term_w.p;
  a.traces = en->d_traces.p;
  a.d_base = en->d_base.p;
  a.local = local;
  a.h_inv = 1.0f / en->h_scale;
  if (en->storage == 1)
    k_post_step<__half><<<1, 128, 0, en->stream>>>(a);
  else if (en->storage == 2)
    k_post_step<__nv_bfloat16><<<1, 128, 0, en->stream>>>(a);
  else
    k_post_step<float><<<1, 128, 0, en->stream>>>(a);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return e;
  return launch_fd(en, local);
}

// Extension kernels between the H and E updates (Mur pre) and after the E
// update (Mur post and apply), in the reference's hook order.
static int blocks_for(long long n, int threads) { return (int)((n + threads - 1) / threads); }

static cudaError_t launch_upml(oems_engine* en, bool h, bool pre);

static int second_order_disp(const oems_engine* en) {
  int k = 0;
  for (const DispHost& d : en->disp) k += d.args.kind >= 3 ? 1 : 0;
  return k;
}

static cudaError_t launch_pre_e(oems_engine* en) {
  if (en->mur.on) {
    k_mur_pre<<<blocks_for(en->mur.args.total, 256), 256, 0, en->stream>>>(en->mur.args);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
  }
  for (const DispHost& d : en->disp)
    if (d.args.kind >= 3) k_dispersive_pre<<<blocks_for(d.args.n, 256), 256, 0, en->stream>>>(d.args);
  // UPML innermost: its pre hook right before the E update
  if (en->upml.on) return launch_upml(en, false, true);
  return cudaSuccess;
}

static cudaError_t launch_post_e(oems_engine* en) {
  if (en->upml.on) {
    cudaError_t e = launch_upml(en, false, false);
    if (e != cudaSuccess) return e;
  }
  if (en->mur.on) {
    const int b = blocks_for(en->mur.args.total, 256);
    k_mur_post<<<b, 256, 0, en->stream>>>(en->mur.args);
    k_mur_apply<<<b, 256, 0, en->stream>>>(en->mur.args);
  }
  // materials one launch each, in the order they were added
  for (const DispHost& d : en->disp) k_dispersive<<<blocks_for(d.args.n, 256), 256, 0, en->stream>>>(d.args);
  if (!en->rlc.q.empty()) {
    RlcArgs r{};
    r.n = (int)en->rlc.q.size();
    r.q = en->rlc.d_q.p;
    r.dir = en->rlc.d_dir.p;
    r.v_vv = en->rlc.d_vv.p;
    r.v_il = en->rlc.d_vil.p;
    r.i_int = en->rlc.d_int.p;
    r.dtf = (float)en->dt;
    for (int c = 0; c < 3; ++c) r.e[c] = en->E(c);
    k_lumped_rlc<<<1, 32, 0, en->stream>>>(r);
  }
  return cudaGetLastError();
}

static int ext_kernels(const oems_engine* en) {
  return (en->mur.on ? 3 : 0) + (en->upml.on ? 4 : 0) + (int)en->disp.size() + second_order_disp(en) +
         (en->rlc.q.empty() ? 0 : 1) + (en->tfsf.on ? 2 : 0);
}

static int kernels_per_step(const oems_engine* en) {
  const int upd = en->shape.split ? 4 : en->shape.zsplit ? (en->gs.work > 0 ? 4 : 2) : 2;
  return upd + ext_kernels(en) + post_kernels(en);
}

// Launches `steps` timesteps directly (no graph).
static cudaError_t launch_upml(oems_engine* en, bool h, bool pre) {
  const UpmlArgs& a = h ? en->upml.h : en->upml.e;
  const int b = blocks_for(a.total, 256);
  if (pre)
    k_upml_pre<<<b, 256, 0, en->stream>>>(a);
  else
    k_upml_post<<<b, 256, 0, en->stream>>>(a);
  return cudaGetLastError();
}

// H update with the UPML current hooks around it (pml.rs:586-655).
static cudaError_t launch_h_step(oems_engine* en) {
  cudaError_t e;
  if (en->upml.on && (e = launch_upml(en, true, true)) != cudaSuccess) return e;
  if ((e = launch_h(en)) != cudaSuccess) return e;
  if (en->upml.on) return launch_upml(en, true, false);
  return cudaSuccess;
}

// One step of the TF/SF 1D grid (src/extensions/tfsf.rs:204-238), f32 as
// the reference: H update, sin source at the first H node, E update, Mur end.
static void tfsf_step_1d(TfsfHost& T, double dt, double dx) {
  constexpr double kMu0 = 1.256637062e-6, kEps0 = 8.854187817e-12, kPi = 3.14159265358979323846;
  const size_t len = T.h1d.size();
  for (size_t i = 0; i + 1 < len; ++i) {
    const float db = (float)(-(dt / (kMu0 * dx)));
    T.h1d[i] += db * (T.e1d[i + 1] - T.e1d[i]);
  }
  const double t = (double)T.t * dt;
  const double eta = std::sqrt(kMu0 / kEps0);
  T.h1d[0] = (float)((T.amp / eta) * std::sin(2.0 * kPi * T.freq * t));
  for (size_t i = 1; i < len; ++i) {
    const float cb = (float)(dt / (kEps0 * dx));
    T.e1d[i] += cb * (T.h1d[i] - T.h1d[i - 1]);
  }
  const float coeff = (float)((T.v * dt - dx) / (T.v * dt + dx));
  T.e1d[len - 1] = coeff * T.e1d[len - 2];
  T.t += 1;
}

// Corrected 1D step (kind 1): hard E source at node 0 at time n, H to
// n + 1/2, E to n + 1 with the wave equation's sign (the reference's E
// update has the opposite sign and grows exponentially), first-order Mur at
// the last node.  e_inc: E at node pos, time n; h_inc: H at pos - 1/2.
static void tfsf_step_1d_fixed(TfsfHost& T, double dt, double dx, float* e_inc, float* h_inc) {
  constexpr double kMu0 = 1.256637062e-6, kEps0 = 8.854187817e-12, kPi = 3.14159265358979323846;
  const size_t len = T.e1d.size();
  const float db = (float)(-(dt / (kMu0 * dx))), cb = (float)(dt / (kEps0 * dx));
  T.e1d[0] = (float)(T.amp * std::sin(2.0 * kPi * T.freq * ((double)T.t * dt)));
  *e_inc = T.e1d[T.pos];
  for (size_t i = 0; i + 1 < len; ++i) T.h1d[i] += db * (T.e1d[i + 1] - T.e1d[i]);
  *h_inc = T.h1d[T.pos - 1];
  const float en1 = T.e1d[len - 2], en = T.e1d[len - 1];
  for (size_t i = 1; i < len; ++i) T.e1d[i] -= cb * (T.h1d[i] - T.h1d[i - 1]);
  const float coeff = (float)((T.v * dt - dx) / (T.v * dt + dx));
  T.e1d[len - 1] = en1 + coeff * (T.e1d[len - 2] - en);
  T.t += 1;
}

// One step of the 1D grid of either kind; the values the two planes get.
static void tfsf_advance(TfsfHost& T, double dt, double dx, float* e_inc, float* h_inc) {
  if (T.kind == 1) {
    tfsf_step_1d_fixed(T, dt, dx, e_inc, h_inc);
    return;
  }
  tfsf_step_1d(T, dt, dx);
  *e_inc = (size_t)T.pos < T.e1d.size() ? T.e1d[T.pos] : 0.0f;
  *h_inc = (size_t)T.pos < T.h1d.size() ? T.h1d[T.pos] : 0.0f;
}

// TF/SF hook of batch step `local`: before H (h_pre) or before E.  Kind 0:
// both planes at pos, h - db e_inc and e + cb h_inc (the reference).  Kind
// 1: the scattered-side H plane pos - 1 gets -Db E_inc (+dt/(mu0 dx) E_inc
// for Transverse1, whose 1D H is the 3D H component, minus that for
// Transverse2), the total-side E plane pos gets +Cb H_inc on the cells the
// E update writes (transverse indices >= 1).
static cudaError_t launch_tfsf(oems_engine* en, bool h_pre, int local) {
  if (!en->tfsf.on) return cudaSuccess;
  const TfsfHost& T = en->tfsf;
  constexpr double kMu0 = 1.256637062e-6, kEps0 = 8.854187817e-12;
  const double dx = en->delta[T.prop];
  TfsfArgs a{};
  a.f = h_pre ? en->H(T.h_axis) : en->E(T.e_axis);
  const long long nzp = en->g.nzp, ny = en->ny;
  const long long stride[3] = {ny * nzp, nzp, 1};
  const int n[3] = {en->nx, en->ny, en->nz};
  const int a1 = T.prop == 0 ? 1 : 0, a2 = T.prop == 2 ? 1 : 2;
  const long long plane = (T.kind == 1 && h_pre) ? T.pos - 1 : T.pos;
  const int first = (T.kind == 1 && !h_pre) ? 1 : 0;
  a.plane_off = plane * stride[T.prop] + first * (stride[a1] + stride[a2]);
  a.s1 = stride[a1];
  a.s2 = stride[a2];
  a.n1 = n[a1] - first;
  a.n2 = n[a2] - first;
  if (T.kind == 1) {
    a.coef = h_pre ? (float)(en->dt / (kMu0 * dx)) : (float)(en->dt / (kEps0 * dx));
    a.add = h_pre ? (T.e_axis == (T.prop + 1) % 3 ? 1 : 0) : 1;
  } else {
    a.coef = h_pre ? (float)(-(en->dt / (kMu0 * dx))) : (float)(en->dt / (kEps0 * dx));
    a.add = h_pre ? 0 : 1;
  }
  a.samples = T.samples.p + (h_pre ? 0 : T.cap);
  a.d_base = en->d_base.p;
  a.local = local;
  const long long cells = (long long)a.n1 * a.n2;
  k_tfsf_plane<<<(int)std::min<long long>((cells + 255) / 256, 1184), 256, 0, en->stream>>>(a);
  return cudaGetLastError();
}

static oems_status launch_steps_direct(oems_engine* en, int steps) {
  for (int s = 0; s < steps; ++s) {
    OEMS_CUDA(launch_tfsf(en, true, s));
    OEMS_CUDA(launch_h_step(en));
    OEMS_CUDA(launch_tfsf(en, false, s));
    OEMS_CUDA(launch_pre_e(en));
    OEMS_CUDA(launch_e(en));
    OEMS_CUDA(launch_post_e(en));
    if (need_post(en)) OEMS_CUDA(launch_post(en, s));
  }
  return OEMS_OK;
}

// Direct launches with an event pair around every H and E kernel; the span is
// processed in chunks of at most 64 steps, reading the events after each.
static oems_status launch_steps_profiled(oems_engine* en, int steps) {
  constexpr int kChunk = 64;
  if (en->prof_ev.empty()) {
    en->prof_ev.resize(4 * kChunk, nullptr);
    for (auto& e : en->prof_ev) OEMS_CUDA(cudaEventCreate(&e));
  }
  for (int s0 = 0; s0 < steps; s0 += kChunk) {
    const int n = std::min(kChunk, steps - s0);
    for (int s = 0; s < n; ++s) {
      cudaEvent_t* ev = &en->prof_ev[4 * s];
      OEMS_CUDA(launch_tfsf(en, true, s0 + s));
      if (en->upml.on) OEMS_CUDA(launch_upml(en, true, true));
      OEMS_CUDA(cudaEventRecord(ev[0], en->stream));
      OEMS_CUDA(launch_h(en));
      OEMS_CUDA(cudaEventRecord(ev[1], en->stream));
      if (en->upml.on) OEMS_CUDA(launch_upml(en, true, false));
      OEMS_CUDA(launch_tfsf(en, false, s0 + s));
      OEMS_CUDA(launch_pre_e(en));
      OEMS_CUDA(cudaEventRecord(ev[2], en->stream));
      OEMS_CUDA(launch_e(en));
      OEMS_CUDA(cudaEventRecord(ev[3], en->stream));
      OEMS_CUDA(launch_post_e(en));
      if (need_post(en)) OEMS_CUDA(launch_post(en, s0 + s));
    }
    OEMS_CUDA(cudaEventSynchronize(en->prof_ev[4 * (n - 1) + 3]));
    for (int s = 0; s < n; ++s) {
      float h = 0.f, e = 0.f;
      OEMS_CUDA(cudaEventElapsedTime(&h, en->prof_ev[4 * s], en->prof_ev[4 * s + 1]));
      OEMS_CUDA(cudaEventElapsedTime(&e, en->prof_ev[4 * s + 2], en->prof_ev[4 * s + 3]));
      en->prof_h_s += h * 1e-3;
      en->prof_e_s += e * 1e-3;
    }
    en->prof_h_n += n;
    en->prof_e_n += n;
  }
  return OEMS_OK;
}

static oems_status get_graph(oems_engine* en, int steps, cudaGraphExec_t* out) {
  if (en->built_epoch != en->graph_epoch) {
    drop_graphs(en);
    en->built_epoch = en->graph_epoch;
  }
  auto it = en->graphs.find(steps);
  if (it != en->graphs.end()) {
    *out = it->second;
    return OEMS_OK;
  }
  if (en->graphs.size() >= 8) drop_graphs(en);
  cudaGraph_t graph = nullptr;
  OEMS_CUDA(cudaStreamBeginCapture(en->stream, cudaStreamCaptureModeThreadLocal));
  oems_status st = launch_steps_direct(en, steps);
  cudaError_t ce = cudaStreamEndCapture(en->stream, &graph);
  if (st != OEMS_OK) {
    if (graph) cudaGraphDestroy(graph);
    return st;
  }
  if (ce != cudaSuccess) return fail(OEMS_ERR_CUDA, std::string("graph capture: ") + cudaGetErrorString(ce));
  cudaGraphExec_t exec = nullptr;
  ce = cudaGraphInstantiate(&exec, graph, 0);
  cudaGraphDestroy(graph);
  if (ce != cudaSuccess) return fail(OEMS_ERR_CUDA, std::string("graph instantiate: ") + cudaGetErrorString(ce));
  en->graphs[steps] = exec;
  *out = exec;
  return OEMS_OK;
}

// Runs batch steps [base, base + steps).
static oems_status run_span(oems_engine* en, long long base, int steps) {
  if (need_post(en) || en->tfsf.on) {
    k_set_i64<<<1, 1, 0, en->stream>>>(en->d_base.p, base);
    OEMS_CUDA(cudaGetLastError());
    en->last_launches += 1;
  }
  if (en->profiling) {
    OEMS_TRY(launch_steps_profiled(en, steps));
  } else if (en->flags & OEMS_ENGINE_NO_GRAPHS) {
    OEMS_TRY(launch_steps_direct(en, steps));
  } else {
    cudaGraphExec_t exec = nullptr;
    OEMS_TRY(get_graph(en, steps, &exec));
    OEMS_CUDA(cudaGraphLaunch(exec, en->stream));
  }
  en->last_launches += (uint64_t)steps * kernels_per_step(en);
  return OEMS_OK;
}

static oems_status launch_energy(oems_engine* en, double* out2) {
  EnergyArgs a{};
  for (int c = 0; c < 6; ++c) a.arr[c] = en->at((size_t)c);
  a.n4 = en->ncells_padded / 4;
  a.partials = en->d_partials.p;
  if (en->storage == 1)
    k_energy_partial<__half><<<dim3(kEnergyBlocks, 6), kEnergyThreads, 0, en->stream>>>(a);
  else if (en->storage == 2)
    k_energy_partial<__nv_bfloat16><<<dim3(kEnergyBlocks, 6), kEnergyThreads, 0, en->stream>>>(a);
  else
    k_energy_partial<float><<<dim3(kEnergyBlocks, 6), kEnergyThreads, 0, en->stream>>>(a);
  OEMS_CUDA(cudaGetLastError());
  k_energy_final<<<1, 32, 0, en->stream>>>(en->d_partials.p, out2, 1.0 / ((double)en->h_scale * en->h_scale));
  OEMS_CUDA(cudaGetLastError());
  en->last_launches += 2;
  return OEMS_OK;
}

static oems_status ensure_host_energy(oems_engine* en, size_t samples) {
  if (samples <= en->h_energy_cap) return OEMS_OK;
  // the mirror is only read after a stream synchronisation: nothing in flight uses it
  pinned_put(en->h_energy, en->h_energy_cap * 2 * sizeof(double));
  en->h_energy = nullptr;
  en->h_energy_cap = 0;
  const size_t cap = std::max<size_t>(samples, 16);
  void* p = nullptr;
  OEMS_CUDA(pinned_get(&p, cap * 2 * sizeof(double)));
  en->h_energy = static_cast<double*>(p);
  en->h_energy_cap = cap;
  return OEMS_OK;
}

// Times `reps` H+E pairs with the current shape (device time in ms).
static oems_status time_shape(oems_engine* en, int reps, float* ms) {
  OEMS_CUDA(launch_h(en));
  OEMS_CUDA(launch_e(en));
  OEMS_CUDA(cudaEventRecord(en->ev0, en->stream));
  for (int r = 0; r < reps; ++r) {
    OEMS_CUDA(launch_h(en));
    OEMS_CUDA(launch_e(en));
  }
  OEMS_CUDA(cudaEventRecord(en->ev1, en->stream));
  OEMS_CUDA(cudaEventSynchronize(en->ev1));
  OEMS_CUDA(cudaEventElapsedTime(ms, en->ev0, en->ev1));
  return OEMS_OK;
}

// Launch shapes already tuned in this process, keyed by grid, device and
// kernel variant (like a cuDNN benchmark cache).
struct TuneKey {
  int dev, nx, ny, nz, id_bytes, cpml;
  bool operator<(const TuneKey& o) const {
    return std::tie(dev, nx, ny, nz, id_bytes, cpml) < std::tie(o.dev, o.nx, o.ny, o.nz, o.id_bytes, o.cpml);
  }
};
struct TuneResult {
  LaunchShape best;
  std::vector<oems_tune_entry> report;
};
static std::map<TuneKey, TuneResult>& tune_cache() {
  static std::map<TuneKey, TuneResult> m;
  return m;
}

static int shape_kind(const LaunchShape& s) { return s.pipe ? 4 : s.split ? 2 : s.tma ? 1 : s.zsplit ? 3 : 0; }
// engines may be driven from several host threads (one engine per thread)
static std::mutex& tune_mutex() {
  static std::mutex m;
  return m;
}

// Project autotuner: tries CTA sizes and x-chunk depths on scratch copies of
// the state (fields and psi are saved and restored), keeps the fastest.
static oems_status autotune(oems_engine* en) {
  en->tuned = true;
  int ilo = 0, ihi = 0, jlo = 0, jhi = 0;
  const bool can_split = en->id_bytes == 0 && en->storage == 0 && cpml_interior(en, &ilo, &ihi, &jlo, &jhi);
  const bool only_split = (en->flags & OEMS_ENGINE_SPLIT_KERNELS) && can_split;
  const bool only_z = (en->flags & OEMS_ENGINE_ZSPLIT_KERNELS) && !only_split && can_zsplit(en);
  size_t optin = 0;
  OEMS_TRY(tma_smem_limit(en, &optin));
  const int pipe_ns = pipe_stages(en, optin);
  const bool only_pipe = (en->flags & OEMS_ENGINE_PIPE_KERNELS) && !only_split && !only_z && pipe_ns > 0;
  const bool want_reg = (!(en->flags & OEMS_ENGINE_STAGED_KERNELS) || en->id_bytes != 0) && !only_split &&
                        !only_z && !only_pipe;
  const bool want_tma = !(en->flags & OEMS_ENGINE_REGISTER_KERNELS) && en->id_bytes == 0 && !only_split &&
                        !only_z && !only_pipe && en->storage == 0;
  // the pipelined kernels are timed only on request: at 256^3 with CPML they
  // measured 0.65 ms per step against 0.38 for the register kernels (one
  // CTA of 8 warps per SM, 204 registers, 1.5x the instructions per plane:
  // issue-bound at 34% issue activity)
  const bool want_pipe = only_pipe;
  // split shapes are tried only on request: at 256^3 with 8-layer CPML the
  // staged interior plus register slabs measured 36.8 GCells/s against 45.6
  // for the register kernels on the whole grid (the z-slab lanes of every
  // warp keep the CPML path in both families)
  const bool want_split = only_split;
  if (en->flags & OEMS_ENGINE_NO_AUTOTUNE) {
    LaunchShape s;
    if (only_split) {
      size_t limit = 0;
      OEMS_TRY(tma_smem_limit(en, &limit));
      s.tma = true;
      s.split = true;
      s.nconsumer = 256;
      s.ichunk = 16;
      s.smem = make_tma_geom(en, std::max(1, std::min(jhi - jlo, 256 / en->g.nzq)), 16, 256, limit, 4, s.tg, true);
      if (s.smem == 0) s = LaunchShape{};
    } else if (!want_reg && !only_z) {
      size_t limit = 0;
      OEMS_TRY(tma_smem_limit(en, &limit));
      s.tma = true;
      s.nconsumer = 256;
      s.ichunk = 16;
      s.smem = make_tma_geom(en, std::max(1, std::min(en->ny, 256 / en->g.nzq)), 16, 256, limit, 4, s.tg);
      if (s.smem == 0) s = LaunchShape{};
    }
    if (only_z) {
      // the untuned z-split: the slab launch forked beside the interior one
      s.zsplit = true;
      s.fork = true;
      s.sh_block = 128;
      s.sh_ichunk = 2;
    }
    if (only_pipe) {
      s.pipe = true;
      s.pipe_ns = pipe_ns;
      s.block = kPipeThreads;
      s.ichunk = 16;
    }
    if (!s.tma) {
      // small grids: shorter x-runs, then narrower CTAs, until every SM has
      // a work item (a 70^3 grid has 45 items at 256 x 8: most SMs would idle)
      int sms = 0;
      OEMS_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, en->device));
      while (make_geom(en, s.block, s.ichunk).work < sms) {
        if (s.ichunk > 1)
          s.ichunk /= 2;
        else if (s.block > 128)
          s.block /= 2;
        else
          break;
      }
    }
    OEMS_TRY(size_grid(en, s));
    apply_shape(en, s);
    return OEMS_OK;
  }
  const bool want_z = (want_reg || only_z) && can_zsplit(en);
  const TuneKey key{en->device, en->nx, en->ny, en->nz, en->id_bytes,
                    (en->cpml.on ? 1 : 0) | (want_reg ? 2 : 0) | (want_tma ? 4 : 0) | (want_split ? 8 : 0) |
                        (want_z ? 16 : 0) | (want_pipe ? 32 : 0) | (en->storage << 6)};
  {
    std::lock_guard<std::mutex> lock(tune_mutex());
    auto hit = tune_cache().find(key);
    if (hit != tune_cache().end()) {
      en->tune_report = hit->second.report;
      apply_shape(en, hit->second.best);
      return OEMS_OK;
    }
  }
  const size_t fbytes = en->field_bytes();
  const size_t pbytes = en->cpml.on ? en->cpml.psi.n * sizeof(float) : 0;
  void* save = nullptr;
  OEMS_CUDA(pool_alloc(&save, fbytes + pbytes, en->stream));
  OEMS_CUDA(cudaMemcpyAsync(save, en->fields, fbytes, cudaMemcpyDeviceToDevice, en->stream));
  if (pbytes)
    OEMS_CUDA(cudaMemcpyAsync((char*)save + fbytes, en->cpml.psi.p, pbytes, cudaMemcpyDeviceToDevice,
                              en->stream));
  const long long cells = (long long)en->nx * en->ny * en->nz;
  const int reps = (int)std::max<long long>(2, std::min<long long>(20, 200000000LL / std::max(1LL, cells)));
  LaunchShape best = en->shape;
  float best_ms = 1e30f;
  std::vector<LaunchShape> cands;
  // plain kernels on the CPML-free box plus one CPML launch over the slabs
  // (want_z): most cells run with the plain kernels' register budget (64 /
  // 92 registers against 128 with spills for the CPML forms)
  // register budgets (occ) only exist for float storage and full arrays
  const int nocc = (en->storage == 0 && en->id_bytes == 0) ? 3 : 1;
  for (int b : {256, 512})
    for (int c : {4, 8, 16, 32})
      for (int pf : {0, 2})
        for (int occ = 0; occ < nocc; ++occ) {
          if (c > 2 * en->nx && c != 4) continue;
          if (pf >= c) continue;
          if (occ > 0 && b != 256) continue;
          LaunchShape s;
          s.block = b;
          s.ichunk = c;
          s.pf = pf;
          s.occ = occ;
          if (want_reg) cands.push_back(s);
          if (want_z && b == 256 && pf == 0 && (c == 4 || c == 8)) {
            // the slab launch: its work items are short (8 layers) and its
            // z-slab parts uncoalesced, so it is latency-bound: short x-runs
            // and narrow CTAs give it more items in flight; forked, it runs
            // beside the interior launch in the room a cut interior grid
            // leaves
            s.zsplit = true;
            for (int fk = 0; fk < 3; ++fk)
              for (int sb : {128, 256})
                for (int sc : {1, 2, 4}) {
                  s.fork = fk > 0;
                  s.cut = fk == 2 ? 1 : 0;
                  s.sh_block = sb;
                  s.sh_ichunk = sc;
                  cands.push_back(s);
                }
          }
        }
  if (want_pipe) {
    // pipelined register kernels: x-runs of 4-32 planes, both stage counts
    // that fit (3 stages keep one bundle in flight, 4 two)
    for (int c : {4, 8, 16, 32})
      for (int ns = pipe_ns; ns >= 3; --ns) {
        if (c > 2 * en->nx && c != 4) continue;
        LaunchShape s;
        s.pipe = true;
        s.pipe_ns = ns;
        s.block = kPipeThreads;
        s.ichunk = c;
        cands.push_back(s);
      }
  }
  if (want_tma) {
    size_t limit = 0;
    OEMS_TRY(tma_smem_limit(en, &limit));
    for (int nc : {128, 256})
      for (int per : {1, 2}) {
        const int tj = std::max(1, std::min(en->ny, per * nc / en->g.nzq));
        for (int c : {8, 16, 32}) {
          int last_ns = 0;
          for (int ns : {4, 3}) {
            if (c > 2 * en->nx && c != 8) continue;
            LaunchShape s;
            s.tma = true;
            s.nconsumer = nc;
            s.ichunk = c;
            s.smem = make_tma_geom(en, tj, c, nc, limit, ns, s.tg);
            if (s.smem == 0) continue;
            if (s.tg.NS == last_ns) continue;  // capped by shared memory: same shape
            last_ns = s.tg.NS;
            cands.push_back(s);
          }
        }
      }
  }
  if (want_split) {
    size_t limit = 0;
    OEMS_TRY(tma_smem_limit(en, &limit));
    for (int nc : {128, 192, 256})
      for (int per : {1, 2}) {
        const int tj = std::max(1, std::min(jhi - jlo, per * nc / en->g.nzq));
        for (int c : {8, 16, 32}) {
          int last_ns = 0;
          for (int ns : {6, 5, 4, 3}) {
            if (c > 2 * en->nx && c != 8) continue;
            LaunchShape s;
            s.tma = true;
            s.split = true;
            s.nconsumer = nc;
            s.ichunk = c;
            s.smem = make_tma_geom(en, tj, c, nc, limit, ns, s.tg, true);
            if (s.smem == 0 || s.tg.NS == last_ns) continue;
            last_ns = s.tg.NS;
            cands.push_back(s);
          }
        }
      }
  }
  oems_status st = OEMS_OK;
  en->tune_report.clear();
  for (LaunchShape s : cands) {
    st = size_grid(en, s);
    if (st != OEMS_OK) break;
    apply_shape(en, s);
    float ms = 0.f;
    st = time_shape(en, reps, &ms);
    if (st != OEMS_OK) break;
    oems_tune_entry te{};
    te.kind = shape_kind(s);
    te.threads = s.tma ? s.nconsumer + 32 : s.block;
    te.ichunk = s.ichunk;
    te.extra = s.tma ? s.tg.NS
                     : s.pipe ? s.pipe_ns : s.pf + 10 * s.occ + 100 * s.sh_occ + 1000 * (s.fork ? 1 + s.cut : 0);
    te.reps = reps;
    te.ms = ms;
    en->tune_report.push_back(te);
    if (ms < best_ms) {
      best_ms = ms;
      best = s;
    }
  }
  if (st == OEMS_OK) {
    int err = 0;
    cudaMemcpyAsync(&err, en->d_err.p, sizeof(int), cudaMemcpyDeviceToHost, en->stream);
    cudaStreamSynchronize(en->stream);
    if (err) st = fail(OEMS_ERR_TIMEOUT, "a bounded device wait gave up while tuning");
  }
  apply_shape(en, best);
  if (st == OEMS_OK) {
    std::lock_guard<std::mutex> lock(tune_mutex());
    tune_cache()[key] = TuneResult{best, en->tune_report};
  }
  cudaMemcpyAsync(en->fields, save, fbytes, cudaMemcpyDeviceToDevice, en->stream);
  if (pbytes) cudaMemcpyAsync(en->cpml.psi.p, (char*)save + fbytes, pbytes, cudaMemcpyDeviceToDevice, en->stream);
  cudaFreeAsync(save, en->stream);
  cudaStreamSynchronize(en->stream);
  return st;
}

// Factor applied to coefficient array a (ca0..2 cb0..2 da0..2 db0..2) when H
// is stored multiplied by h_scale: Cb / s (E sees H / s) and Db * s.
static float coef_storage_factor(const oems_engine* en, int a) {
  if (en->h_scale == 1.0f) return 1.0f;
  if (a >= 3 && a < 6) return 1.0f / en->h_scale;
  if (a >= 9) return en->h_scale;
  return 1.0f;
}

static oems_status upload_coefficients(oems_engine* en, const oems_operator_desc* d) {
  const size_t nzp = en->g.nzp;
  const size_t rows = (size_t)en->nx * en->ny;
  const float* src[12] = {d->ca[0], d->ca[1], d->ca[2], d->cb[0], d->cb[1], d->cb[2],
                          d->da[0], d->da[1], d->da[2], d->db[0], d->db[1], d->db[2]};
  for (int a = 0; a < 12; ++a)
    if (!src[a]) return fail(OEMS_ERR_INVALID_ARGUMENT, "coefficient array pointer is NULL");
  if (!(en->flags & OEMS_ENGINE_COMPRESSED)) {
    OEMS_CUDA(pool_alloc(reinterpret_cast<void**>(&en->coeffs), (size_t)12 * en->ncells_padded * sizeof(float),
                         en->stream));
    OEMS_CUDA(cudaMemsetAsync(en->coeffs, 0, (size_t)12 * en->ncells_padded * sizeof(float), en->stream));
    std::vector<float> scaled;
    for (int a = 0; a < 12; ++a) {
      const float* from = src[a];
      const float f = coef_storage_factor(en, a);
      if (f != 1.0f) {
        // Cb / s and Db * s for H kept scaled by s (a power of two: exact)
        scaled.resize(rows * en->nz);
        for (size_t q = 0; q < scaled.size(); ++q) scaled[q] = src[a][q] * f;
        from = scaled.data();
      }
      OEMS_CUDA(cudaMemcpy2DAsync(en->C(a), nzp * sizeof(float), from, en->nz * sizeof(float),
                                  en->nz * sizeof(float), rows, cudaMemcpyHostToDevice, en->stream));
      if (f != 1.0f) OEMS_CUDA(cudaStreamSynchronize(en->stream));
    }
    OEMS_CUDA(cudaStreamSynchronize(en->stream));
    return OEMS_OK;
  }
  // Compressed: the 12 coefficients of each cell deduplicated bit for bit
  // into a table (oems_compress_coefficients, the host routine of
  // CompressedCoefficients::from_fields), ids padded to the row pitch
  const size_t n = (size_t)en->nx * en->ny * en->nz;
  std::vector<uint16_t> dense(n);
  std::vector<float> table((size_t)65536 * 12);
  uint32_t nunique = 0;
  const oems_status cst = oems_compress_coefficients(src, n, dense.data(), table.data(), 65536, &nunique);
  if (cst != OEMS_OK) return cst;
  table.resize((size_t)nunique * 12);
  std::vector<uint16_t> ids16((size_t)en->ncells_padded, 0);
  for (size_t r = 0; r < rows; ++r)
    std::memcpy(ids16.data() + r * nzp, dense.data() + r * en->nz, (size_t)en->nz * sizeof(uint16_t));
  en->ntable = (int)nunique;
  for (size_t t = 0; t < table.size(); ++t) table[t] *= coef_storage_factor(en, (int)(t % 12));
  OEMS_CUDA(pool_alloc(reinterpret_cast<void**>(&en->table), table.size() * sizeof(float), en->stream));
  OEMS_CUDA(cudaMemcpyAsync(en->table, table.data(), table.size() * sizeof(float), cudaMemcpyHostToDevice,
                            en->stream));
  if (en->ntable <= 256) {
    en->id_bytes = 1;
    std::vector<uint8_t> ids8(ids16.size());
    for (size_t q = 0; q < ids16.size(); ++q) ids8[q] = (uint8_t)ids16[q];
    OEMS_CUDA(pool_alloc(&en->ids, ids8.size(), en->stream));
    OEMS_CUDA(cudaMemcpyAsync(en->ids, ids8.data(), ids8.size(), cudaMemcpyHostToDevice, en->stream));
    OEMS_CUDA(cudaStreamSynchronize(en->stream));
  } else {
    en->id_bytes = 2;
    OEMS_CUDA(pool_alloc(&en->ids, ids16.size() * sizeof(uint16_t), en->stream));
    OEMS_CUDA(cudaMemcpyAsync(en->ids, ids16.data(), ids16.size() * sizeof(uint16_t), cudaMemcpyHostToDevice,
                              en->stream));
    OEMS_CUDA(cudaStreamSynchronize(en->stream));
  }
  return OEMS_OK;
}

// Every buffer goes back to the pool on the engine's stream (the stream is
// idle by then); the stream itself is destroyed last.
static void destroy(oems_engine* en) {
  if (!en) return;
  cudaStream_t s = en->stream;
  if (s) cudaStreamSynchronize(s);
  drop_graphs(en);
  for (void* p : {(void*)en->fields, (void*)en->coeffs, en->ids, (void*)en->table})
    if (p) cudaFreeAsync(p, s);
  pinned_put(en->h_energy, en->h_energy_cap * 2 * sizeof(double));
  if (en->ev0) cudaEventDestroy(en->ev0);
  if (en->ev1) cudaEventDestroy(en->ev1);
  if (en->fork_ev) cudaEventDestroy(en->fork_ev);
  if (en->join_ev) cudaEventDestroy(en->join_ev);
  if (en->side) {
    cudaStreamSynchronize(en->side);
    cudaStreamDestroy(en->side);
  }
  for (cudaEvent_t e : en->prof_ev)
    if (e) cudaEventDestroy(e);
  delete en;  // DevBuf members free on their stream
  if (s) cudaStreamDestroy(s);
}

static oems_status create(const oems_operator_desc* d, oems_engine** out) {
  if (!d || !out) return fail(OEMS_ERR_INVALID_ARGUMENT, "NULL descriptor or output pointer");
  *out = nullptr;
  if (d->nx == 0 || d->ny == 0 || d->nz == 0) return fail(OEMS_ERR_GRID, "grid dimensions must be positive");
  if (d->nx > (1u << 30) || d->ny > (1u << 30) || d->nz > (1u << 30))
    return fail(OEMS_ERR_GRID, "grid dimension too large");
  const uint64_t nzp = (d->nz + 3) / 4 * 4;
  if ((double)d->ny * (double)nzp / 4.0 > 2.0e9) return fail(OEMS_ERR_GRID, "x-plane too large");
  if (!(d->dt > 0.0) || !std::isfinite(d->dt)) return fail(OEMS_ERR_CONFIG, "dt must be positive and finite");
  int ndev = 0;
  cudaError_t ce = cudaGetDeviceCount(&ndev);
  if (ce != cudaSuccess || ndev == 0) {
    cudaGetLastError();
    return fail(OEMS_ERR_NO_DEVICE, cudaGetErrorString(ce));
  }
  int dev = d->device;
  if (dev < 0) OEMS_CUDA(cudaGetDevice(&dev));
  if (dev >= ndev) return fail(OEMS_ERR_NO_DEVICE, "device ordinal out of range");
  DeviceGuard guard(dev);
  std::unique_ptr<oems_engine, void (*)(oems_engine*)> en(new oems_engine, destroy);
  en->device = dev;
  en->flags = d->flags;
  const uint32_t half_flags = d->flags & (OEMS_ENGINE_FIELDS_F16 | OEMS_ENGINE_FIELDS_BF16);
  if (half_flags == (OEMS_ENGINE_FIELDS_F16 | OEMS_ENGINE_FIELDS_BF16))
    return fail(OEMS_ERR_CONFIG, "choose one field storage: half or bfloat16");
  if (half_flags && (d->flags & (OEMS_ENGINE_STAGED_KERNELS | OEMS_ENGINE_SPLIT_KERNELS)))
    return fail(OEMS_ERR_CONFIG, "2-byte field storage runs the register kernels only");
  en->storage = (d->flags & OEMS_ENGINE_FIELDS_F16) ? 1 : (d->flags & OEMS_ENGINE_FIELDS_BF16) ? 2 : 0;
  en->elem = en->storage ? 2 : sizeof(float);
  en->h_scale = en->storage ? OEMS_H_STORAGE_SCALE : 1.0f;
  en->nx = (int)d->nx;
  en->ny = (int)d->ny;
  en->nz = (int)d->nz;
  en->dt = d->dt;
  for (int a = 0; a < 3; ++a) en->delta[a] = d->delta[a];
  OEMS_CUDA(cudaStreamCreateWithFlags(&en->stream, cudaStreamNonBlocking));
  EngineScope scope(en.get());
  OEMS_CUDA(cudaEventCreate(&en->ev0));
  OEMS_CUDA(cudaEventCreate(&en->ev1));
  en->g = make_geom(en.get(), 256, 8);
  en->ncells_padded = (long long)en->nx * en->ny * en->g.nzp;
  OEMS_CUDA(pool_alloc(reinterpret_cast<void**>(&en->fields), en->field_bytes(), en->stream));
  OEMS_CUDA(cudaMemsetAsync(en->fields, 0, en->field_bytes(), en->stream));
  OEMS_TRY(upload_coefficients(en.get(), d));
  OEMS_CUDA(en->d_partials.ensure(6 * kEnergyBlocks));
  OEMS_CUDA(en->d_base.ensure(1));
  OEMS_CUDA(en->d_err.ensure(1));
  OEMS_CUDA(cudaMemsetAsync(en->d_err.p, 0, sizeof(int), en->stream));
  LaunchShape s;
  OEMS_TRY(size_grid(en.get(), s));
  apply_shape(en.get(), s);
  OEMS_CUDA(cudaStreamSynchronize(en->stream));
  *out = en.release();
  return OEMS_OK;
}

static oems_status upload_excitations(oems_engine* en, const oems_batch* b) {
  en->nexc = (int)b->num_excitations;
  if (en->nexc == 0) return OEMS_OK;
  if (!b->excitations) return fail(OEMS_ERR_INVALID_ARGUMENT, "excitation list is NULL");
  std::vector<long long> idx(en->nexc), off(en->nexc), cnt(en->nexc);
  std::vector<int> meta(en->nexc);
  long long total = 0;
  for (int x = 0; x < en->nexc; ++x) {
    const oems_scheduled_excitation& e = b->excitations[x];
    if (e.position[0] >= (uint64_t)en->nx || e.position[1] >= (uint64_t)en->ny || e.position[2] >= (uint64_t)en->nz)
      return fail(OEMS_ERR_CONFIG, "excitation position outside the grid");
    if (e.direction > 2) return fail(OEMS_ERR_CONFIG, "excitation direction must be 0, 1 or 2");
    if (e.num_samples > 0 && !e.samples) return fail(OEMS_ERR_INVALID_ARGUMENT, "excitation samples are NULL");
    idx[x] = ((long long)e.position[0] * en->ny + (long long)e.position[1]) * en->g.nzp + (long long)e.position[2];
    meta[x] = (int)e.direction | ((e.soft_source ? 1 : 0) << 2);
    // only the samples this batch can use are uploaded
    cnt[x] = (long long)std::min<uint64_t>(e.num_samples, b->num_steps);
    off[x] = total;
    total += cnt[x];
  }
  bool realloc = false;
  realloc |= en->d_exc_idx.n < (size_t)en->nexc || en->d_exc_samples.n < (size_t)std::max(total, 1LL);
  OEMS_CUDA(en->d_exc_idx.ensure(en->nexc));
  OEMS_CUDA(en->d_exc_off.ensure(en->nexc));
  OEMS_CUDA(en->d_exc_count.ensure(en->nexc));
  OEMS_CUDA(en->d_exc_meta.ensure(en->nexc));
  OEMS_CUDA(en->d_exc_samples.ensure(std::max(total, 1LL)));
  if (realloc) en->graph_epoch++;
  OEMS_CUDA(cudaMemcpyAsync(en->d_exc_idx.p, idx.data(), en->nexc * sizeof(long long), cudaMemcpyHostToDevice, en->stream));
  OEMS_CUDA(cudaMemcpyAsync(en->d_exc_off.p, off.data(), en->nexc * sizeof(long long), cudaMemcpyHostToDevice, en->stream));
  OEMS_CUDA(cudaMemcpyAsync(en->d_exc_count.p, cnt.data(), en->nexc * sizeof(long long), cudaMemcpyHostToDevice, en->stream));
  OEMS_CUDA(cudaMemcpyAsync(en->d_exc_meta.p, meta.data(), en->nexc * sizeof(int), cudaMemcpyHostToDevice, en->stream));
  for (int x = 0; x < en->nexc; ++x)
    if (cnt[x] > 0)
      OEMS_CUDA(cudaMemcpyAsync(en->d_exc_samples.p + off[x], b->excitations[x].samples, cnt[x] * sizeof(float),
                                cudaMemcpyHostToDevice, en->stream));
  // the host buffers are borrowed only for this call
  OEMS_CUDA(cudaStreamSynchronize(en->stream));
  return OEMS_OK;
}

// Twiddles of the steps of the next batch: the sample after batch step s is
// timestep t = t0 + s + 1; it is taken when t is a multiple of `interval`,
// with exp(-j 2 pi f t dt) and exp(-j 2 pi f (t - 1/2) dt) times 2 dt interval
// (src/processing/fields_fd.rs:156-167), evaluated with the host libm.
static oems_status fill_twiddles(oems_engine* en, FdTable* T, const std::vector<double>& freqs,
                                 uint32_t interval, uint64_t steps) {
  const size_t nf = freqs.size(), ns = (size_t)std::max<uint64_t>(steps, 1);
  if (ns * nf * 4 * sizeof(double) > ((size_t)1 << 30))
    return fail(OEMS_ERR_CONFIG, "frequency-domain twiddle table above 1 GiB: use shorter batches");
  T->h_tw.assign(ns * nf * 4, 0.0);
  T->h_sampled.assign(ns, 0);
  const double scale = 2.0 * en->dt * (double)interval;
  for (uint64_t st = 0; st < steps; ++st) {
    const uint64_t t = en->timestep + st + 1;
    if (t % interval != 0) continue;
    T->h_sampled[st] = 1;
    double* w = T->h_tw.data() + st * nf * 4;
    for (size_t f = 0; f < nf; ++f) {
      const double pe = -2.0 * 3.14159265358979323846 * freqs[f] * ((double)t * en->dt);
      const double ph = -2.0 * 3.14159265358979323846 * freqs[f] * (((double)t - 0.5) * en->dt);
      w[4 * f] = std::cos(pe) * scale;
      w[4 * f + 1] = std::sin(pe) * scale;
      w[4 * f + 2] = std::cos(ph) * scale;
      w[4 * f + 3] = std::sin(ph) * scale;
    }
  }
  if (T->tw.n < T->h_tw.size() || T->sampled.n < ns) {
    OEMS_CUDA(T->tw.ensure(T->h_tw.size()));
    OEMS_CUDA(T->sampled.ensure(ns));
    en->graph_epoch++;
  }
  OEMS_CUDA(cudaMemcpyAsync(T->tw.p, T->h_tw.data(), T->h_tw.size() * sizeof(double), cudaMemcpyHostToDevice,
                            en->stream));
  OEMS_CUDA(cudaMemcpyAsync(T->sampled.p, T->h_sampled.data(), ns * sizeof(int), cudaMemcpyHostToDevice,
                            en->stream));
  OEMS_CUDA(cudaStreamSynchronize(en->stream));
  return OEMS_OK;
}

static oems_status run_batch(oems_engine* en, const oems_batch* b, oems_batch_result* r) {
  if (!b || !r) return fail(OEMS_ERR_INVALID_ARGUMENT, "NULL batch or result");
  EngineScope guard(en);
  const auto t_start = std::chrono::steady_clock::now();
  en->last_launches = 0;
  if (!en->tuned) OEMS_TRY(autotune(en));
  const int prev_nexc = en->nexc;
  OEMS_TRY(upload_excitations(en, b));
  if (prev_nexc != en->nexc) en->graph_epoch++;  // nexc is baked into captured graphs
  const uint64_t steps = b->num_steps;
  const int nprobe = en->nprobe();
  if (nprobe > 0) {
    const size_t need = (size_t)std::max<uint64_t>(steps, 1) * nprobe;
    if (en->d_traces.n < need) {
      OEMS_CUDA(en->d_traces.ensure(need));
      en->graph_epoch++;
    }
  }
  for (FieldDftHost& d : en->fdumps) OEMS_TRY(fill_twiddles(en, d.tab.get(), d.freqs, d.interval, steps));
  for (Nf2ffHost& x : en->boxes) OEMS_TRY(fill_twiddles(en, x.tab.get(), x.freqs, x.interval, steps));
  // TF/SF: this batch's 1D-grid values; the state is kept to replay a batch
  // that ends early
  std::vector<float> tf_e0, tf_h0;
  uint64_t tf_t0 = 0;
  if (en->tfsf.on && steps > 0) {
    TfsfHost& T = en->tfsf;
    tf_e0 = T.e1d;
    tf_h0 = T.h1d;
    tf_t0 = T.t;
    if (steps > T.cap) {
      T.cap = steps;
      OEMS_CUDA(T.samples.ensure(2 * T.cap));
      en->graph_epoch++;  // the h_inc half moved
    }
    std::vector<float> smp(2 * T.cap, 0.0f);
    const double dx = en->delta[T.prop];
    for (uint64_t q = 0; q < steps; ++q) tfsf_advance(T, en->dt, dx, &smp[q], &smp[T.cap + q]);
    OEMS_CUDA(cudaMemcpyAsync(T.samples.p, smp.data(), smp.size() * sizeof(float), cudaMemcpyHostToDevice,
                              en->stream));
    OEMS_CUDA(cudaStreamSynchronize(en->stream));
  }
  const uint64_t si = b->sample_interval, ci = b->check_interval;
  const bool has_decay = b->has_energy_decay_db != 0;
  // worst-case number of energy samples this batch can take
  const uint64_t t0 = en->timestep;
  uint64_t max_samples = 0;
  if (si > 0 && steps > 0) {
    const uint64_t first = (t0 + si - 1) / si * si;  // first multiple of si >= t0
    const uint64_t last_step = t0 + steps - 1;
    max_samples = first > last_step ? 0 : (last_step - first) / si + 1;
  }
  OEMS_CUDA(en->d_energy.ensure(2 * (max_samples + 1)));
  OEMS_TRY(ensure_host_energy(en, max_samples + 1));
  double* d_check = en->d_energy.p + 2 * max_samples;  // scratch slot for checks

  std::vector<uint64_t> sample_steps;
  double peak = b->initial_peak_energy;
  size_t peaked = 0;  // samples already folded into `peak`
  uint64_t executed = 0;
  int reason = OEMS_TERMINATION_STEPS_COMPLETED;
  double final_db = 0.0;
  bool numerical = false;
  OEMS_CUDA(cudaEventRecord(en->ev0, en->stream));
  uint64_t s = 0;
  while (s < steps) {
    const uint64_t cur = t0 + s;
    // next event step >= cur
    uint64_t ev = UINT64_MAX;
    if (si > 0) ev = std::min(ev, (cur + si - 1) / si * si);
    if (has_decay && ci > 0) {
      uint64_t c = (cur + ci - 1) / ci * ci;
      if (c == 0) c = ci;
      ev = std::min(ev, c);
    }
    uint64_t span = steps - s;
    if (ev != UINT64_MAX && ev - cur + 1 < span) span = ev - cur + 1;
    span = std::min<uint64_t>(span, 1u << 20);
    OEMS_TRY(run_span(en, (long long)s, (int)span));
    s += span;
    executed = s;
    const uint64_t last = t0 + s - 1;  // `cur` of the last executed step
    const bool do_sample = si > 0 && last % si == 0;
    const bool do_check = has_decay && ci > 0 && last > 0 && last % ci == 0;
    if (do_sample) {
      OEMS_TRY(launch_energy(en, en->d_energy.p + 2 * sample_steps.size()));
      sample_steps.push_back(last);
    }
    if (do_check) {
      double* src = do_sample ? en->d_energy.p + 2 * (sample_steps.size() - 1) : d_check;
      if (!do_sample) OEMS_TRY(launch_energy(en, d_check));
      // bring back every sample taken since the last check, plus this energy
      const size_t ns = sample_steps.size();
      if (ns > peaked)
        OEMS_CUDA(cudaMemcpyAsync(en->h_energy + 2 * peaked, en->d_energy.p + 2 * peaked,
                                  (ns - peaked) * 2 * sizeof(double), cudaMemcpyDeviceToHost, en->stream));
      double curE[2];
      OEMS_CUDA(cudaMemcpyAsync(en->h_energy + 2 * max_samples, src, 2 * sizeof(double), cudaMemcpyDeviceToHost,
                                en->stream));
      OEMS_CUDA(cudaStreamSynchronize(en->stream));
      curE[0] = en->h_energy[2 * max_samples];
      curE[1] = en->h_energy[2 * max_samples + 1];
      for (; peaked < ns; ++peaked) {
        const double tot = en->h_energy[2 * peaked] + en->h_energy[2 * peaked + 1];
        if (!std::isfinite(tot)) numerical = true;
        if (b->track_peak) peak = std::max(peak, tot);
      }
      const double tot = curE[0] + curE[1];
      if (!std::isfinite(tot)) numerical = true;
      if (numerical) break;
      if (peak > 0.0 && tot > 0.0) {
        const double d = 10.0 * std::log10(tot / peak);
        if (d < -std::fabs(b->energy_decay_db)) {
          reason = OEMS_TERMINATION_ENERGY_DECAY;
          final_db = d;
          break;
        }
      }
    }
  }
  if (!en->entry_probe.empty() && executed > 0) {
    DftArgs da{};
    da.nentries = (int)en->entry_probe.size();
    da.entry_probe = en->d_entry_probe.p;
    da.entry_freq = en->d_entry_freq.p;
    da.entry_half = en->d_entry_half.p;
    da.acc = en->d_dft_acc.p;
    da.traces = en->d_traces.p;
    da.nprobe = en->nprobe();
    da.steps = (long long)executed;
    da.t0 = (long long)t0;
    da.dt = en->dt;
    k_probe_dft<<<(da.nentries + 127) / 128, 128, 0, en->stream>>>(da);
    OEMS_CUDA(cudaGetLastError());
    en->last_launches += 1;
  }
  OEMS_CUDA(cudaEventRecord(en->ev1, en->stream));
  const size_t ns = sample_steps.size();
  if (ns > peaked)
    OEMS_CUDA(cudaMemcpyAsync(en->h_energy + 2 * peaked, en->d_energy.p + 2 * peaked,
                              (ns - peaked) * 2 * sizeof(double), cudaMemcpyDeviceToHost, en->stream));
  int dev_err = 0;
  OEMS_CUDA(cudaMemcpyAsync(&dev_err, en->d_err.p, sizeof(int), cudaMemcpyDeviceToHost, en->stream));
  OEMS_CUDA(cudaStreamSynchronize(en->stream));
  if (dev_err != 0) {
    cudaMemsetAsync(en->d_err.p, 0, sizeof(int), en->stream);
    cudaStreamSynchronize(en->stream);
    return fail(OEMS_ERR_TIMEOUT, "a bounded wait in an update kernel gave up; the fields are not valid");
  }
  for (; peaked < ns; ++peaked) {
    const double tot = en->h_energy[2 * peaked] + en->h_energy[2 * peaked + 1];
    if (!std::isfinite(tot)) numerical = true;
    if (b->track_peak) peak = std::max(peak, tot);
  }
  float ms = 0.f;
  cudaEventElapsedTime(&ms, en->ev0, en->ev1);
  en->last_device_seconds = ms * 1e-3;
  en->timestep = t0 + executed;
  if (en->tfsf.on && executed < steps) {
    TfsfHost& T = en->tfsf;
    T.e1d = tf_e0;
    T.h1d = tf_h0;
    T.t = tf_t0;
    float e_inc, h_inc;
    for (uint64_t q = 0; q < executed; ++q) tfsf_advance(T, en->dt, en->delta[T.prop], &e_inc, &h_inc);
  }
  en->traces_steps = executed;
  r->timesteps_executed = executed;
  r->termination_reason = reason;
  r->reserved0 = 0;
  r->final_decay_db = final_db;
  r->num_energy_samples = ns;
  r->peak_energy = peak;
  for (size_t q = 0; q < ns && r->energy_samples && q < r->energy_capacity; ++q) {
    r->energy_samples[q].timestep = sample_steps[q];
    r->energy_samples[q].e_energy = en->h_energy[2 * q];
    r->energy_samples[q].h_energy = en->h_energy[2 * q + 1];
    r->energy_samples[q].total_energy = en->h_energy[2 * q] + en->h_energy[2 * q + 1];
  }
  r->elapsed_seconds = std::chrono::duration<double>(std::chrono::steady_clock::now() - t_start).count();
  if (numerical) return fail(OEMS_ERR_NUMERICAL, "field energy became NaN or infinite");
  return OEMS_OK;
}

// 2-byte storage: values converted on the host (rounded to nearest on the
// way in), H scaled by h_scale on the device.
static oems_status copy_fields_2byte(oems_engine* en, float* const* host6, bool to_host) {
  const size_t rows = (size_t)en->nx * en->ny, n = rows * en->nz;
  std::vector<uint16_t> buf(n);
  for (int c = 0; c < 6; ++c) {
    if (!host6[c]) return fail(OEMS_ERR_INVALID_ARGUMENT, "field pointer is NULL");
    const float scale = c < 3 ? 1.0f : en->h_scale;
    float* dev = en->at((size_t)c);
    if (to_host) {
      OEMS_CUDA(cudaMemcpy2DAsync(buf.data(), en->nz * 2, dev, en->g.nzp * 2, en->nz * 2, rows,
                                  cudaMemcpyDeviceToHost, en->stream));
      OEMS_CUDA(cudaStreamSynchronize(en->stream));
      for (size_t q = 0; q < n; ++q) {
        const float v = en->storage == 1 ? __half2float(__ushort_as_half(buf[q]))
                                         : __bfloat162float(__ushort_as_bfloat16(buf[q]));
        host6[c][q] = v / scale;
      }
    } else {
      for (size_t q = 0; q < n; ++q) {
        const float v = host6[c][q] * scale;
        buf[q] = en->storage == 1 ? __half_as_ushort(__float2half_rn(v))
                                  : __bfloat16_as_ushort(__float2bfloat16_rn(v));
      }
      OEMS_CUDA(cudaMemcpy2DAsync(dev, en->g.nzp * 2, buf.data(), en->nz * 2, en->nz * 2, rows,
                                  cudaMemcpyHostToDevice, en->stream));
      OEMS_CUDA(cudaStreamSynchronize(en->stream));
    }
  }
  return OEMS_OK;
}

static oems_status copy_fields(oems_engine* en, float* const* host6, bool to_host) {
  EngineScope guard(en);
  if (en->storage) return copy_fields_2byte(en, host6, to_host);
  const size_t rows = (size_t)en->nx * en->ny;
  for (int c = 0; c < 6; ++c) {
    if (!host6[c]) return fail(OEMS_ERR_INVALID_ARGUMENT, "field pointer is NULL");
    float* dev = en->fields + (size_t)c * en->ncells_padded;
    if (to_host)
      OEMS_CUDA(cudaMemcpy2DAsync(host6[c], en->nz * sizeof(float), dev, en->g.nzp * sizeof(float),
                                  en->nz * sizeof(float), rows, cudaMemcpyDeviceToHost, en->stream));
    else
      OEMS_CUDA(cudaMemcpy2DAsync(dev, en->g.nzp * sizeof(float), host6[c], en->nz * sizeof(float),
                                  en->nz * sizeof(float), rows, cudaMemcpyHostToDevice, en->stream));
  }
  OEMS_CUDA(cudaStreamSynchronize(en->stream));
  return OEMS_OK;
}

// MurAbc::new (src/extensions/mur_abc.rs:175-206) and its face set-up
// (:88-151); second order as described in mur.cuh.
static oems_status add_mur(oems_engine* en, const oems_mur_desc* d) {
  if (!d) return fail(OEMS_ERR_INVALID_ARGUMENT, "NULL Mur descriptor");
  if (en->storage) return fail(OEMS_ERR_CONFIG, "Mur boundaries need float field storage");
  if (en->mur.on) return fail(OEMS_ERR_CONFIG, "Mur boundary already attached");
  if (d->order != 1 && d->order != 2) return fail(OEMS_ERR_CONFIG, "Mur order must be 1 or 2");
  EngineScope guard(en);
  const int ext[3] = {en->nx, en->ny, en->nz};
  const double kC0 = 299792458.0;
  const double c = d->phase_velocity > 0.0 ? d->phase_velocity : kC0;
  MurArgs& A = en->mur.args;
  A = MurArgs{};
  A.order = d->order;
  long long off = 0;
  for (int f = 0; f < 6; ++f) {
    if (!d->enabled[f]) continue;
    MurFaceDev F{};
    F.ny = f / 2;
    F.nyp = (F.ny + 1) % 3;
    F.nypp = (F.ny + 2) % 3;
    const bool is_max = f % 2 == 1;
    const int o = (d->order == 2 && !is_max) ? 1 : 0;
    const int n = ext[F.ny];
    if (n < 2 + o) return fail(OEMS_ERR_CONFIG, "Mur face needs at least two cells along its normal");
    F.line = is_max ? n - 1 : o;
    F.shift = is_max ? n - 2 : o + 1;
    F.size0 = ext[F.nyp];
    F.size1 = ext[F.nypp];
    F.lo0 = (d->order == 2 && d->enabled[2 * F.nyp]) ? 1 : 0;
    F.lo1 = (d->order == 2 && d->enabled[2 * F.nypp]) ? 1 : 0;
    const double cdt = c * en->dt, dn = en->delta[F.ny];
    F.coeff = (float)((cdt - dn) / (cdt + dn));
    F.c2 = (float)(2.0 * dn / (cdt + dn));
    F.c3p = (float)(cdt * cdt * dn / (2.0 * en->delta[F.nyp] * en->delta[F.nyp] * (cdt + dn)));
    F.c3q = (float)(cdt * cdt * dn / (2.0 * en->delta[F.nypp] * en->delta[F.nypp] * (cdt + dn)));
    F.off = off;
    off += (long long)F.size0 * F.size1;
    A.f[A.nfaces++] = F;
  }
  if (A.nfaces == 0) return fail(OEMS_ERR_CONFIG, "no Mur face enabled");
  A.total = off;
  OEMS_CUDA(en->mur.state.ensure((size_t)6 * off));
  OEMS_CUDA(cudaMemsetAsync(en->mur.state.p, 0, (size_t)6 * off * sizeof(float), en->stream));
  A.v = en->mur.state.p;
  A.ob = A.v + 2 * off;
  A.os = A.ob + 2 * off;
  for (int c3 = 0; c3 < 3; ++c3) A.e[c3] = en->E(c3);
  A.ny = en->ny;
  A.nzp = en->g.nzp;
  OEMS_CUDA(cudaStreamSynchronize(en->stream));
  en->mur.on = true;
  en->graph_epoch++;
  return OEMS_OK;
}

static oems_status add_cpml(oems_engine* en, const oems_cpml_desc* d) {
  if (!d) return fail(OEMS_ERR_INVALID_ARGUMENT, "NULL CPML descriptor");
  if (en->cpml.on) return fail(OEMS_ERR_CONFIG, "CPML already attached");
  EngineScope guard(en);
  const int ext[3] = {en->nx, en->ny, en->nz};
  int L[6];
  int lmax = 0;
  for (int f = 0; f < 6; ++f) {
    if (d->layers[f] < 0) return fail(OEMS_ERR_CONFIG, "negative CPML layer count");
    // src/extensions/cpml.rs:262,283: a face is active if 0 < layers < n
    L[f] = (d->layers[f] > 0 && d->layers[f] < ext[f / 2]) ? d->layers[f] : 0;
    lmax = std::max(lmax, d->layers[f]);
  }
  for (int a = 0; a < 3; ++a)
    if (L[2 * a] + L[2 * a + 1] > ext[a]) return fail(OEMS_ERR_CONFIG, "CPML slabs overlap");
  if (lmax <= 0) return fail(OEMS_ERR_CONFIG, "CPML needs at least one face with layers > 0");
  if (!(d->reflection_coeff > 0.0 && d->reflection_coeff < 1.0))
    return fail(OEMS_ERR_CONFIG, "CPML reflection coefficient must be in (0, 1)");
  // src/extensions/cpml.rs:68-72 and :236: sigma_max from the largest layer
  // count and the smallest cell size
  const double kEps0 = 8.854187817e-12, kZ0 = 376.730313668;
  const double dmin = std::min(en->delta[0], std::min(en->delta[1], en->delta[2]));
  const double width_max = (double)lmax * dmin;
  const double sigma_max = -(d->grading_order + 1.0) * std::log(d->reflection_coeff) / (2.0 * kZ0 * width_max);
  std::vector<float> prof;
  CpmlArgs& A = en->cpml.args;
  std::memset(&A, 0, sizeof(A));
  for (int f = 0; f < 6; ++f) {
    const int a = f / 2;
    const bool is_min = (f % 2) == 0;
    A.L[f] = L[f];
    A.start[f] = is_min ? 0 : ext[a] - L[f];
    A.prof_off[f] = (int)prof.size();
    if (L[f] == 0) continue;
    const double width = (double)L[f] * en->delta[a];
    std::vector<float> rows(6 * L[f]);
    for (int l = 0; l < L[f]; ++l) {
      // Depth of the E and H difference positions of layer l below the
      // slab's inner interface.  The grading formulas are those of
      // src/extensions/cpml.rs:114-155; its max-face depths ((l + 1) d for
      // E, (l + 1/2) d for H) put E one cell deeper than the H between the
      // same E nodes, a mismatch that reflects about -14 dB of a normally
      // incident wave (the reference never applies psi, so it does not show
      // there).  Here both faces use the positions of the differences: the
      // backward E difference of cell g sits at g d, the forward H
      // difference at (g + 1/2) d.
      const double depth_e = is_min ? (double)(L[f] - l) * en->delta[a] : (double)l * en->delta[a];
      const double depth_h = is_min ? depth_e - 0.5 * en->delta[a] : depth_e + 0.5 * en->delta[a];
      for (int w = 0; w < 2; ++w) {
        const double depth = w == 0 ? depth_e : depth_h;
        const double rho = std::min(1.0, std::max(0.0, depth / width));
        const double sigma = sigma_max * std::pow(rho, d->grading_order);
        const double alpha = d->alpha_max * (1.0 - rho);
        const double kappa = 1.0 + (d->kappa_max - 1.0) * std::pow(rho, d->grading_order);
        const double bb = std::exp(-(sigma / kappa / kEps0 + alpha / kEps0) * en->dt);
        const double sn = sigma / (kEps0 * kappa), an = alpha / kEps0, den = sn + an;
        const double a_ref = std::fabs(den) > 1e-20 ? sn / den * (1.0 - bb) : 0.0;
        // Roden-Gedney a = sigma/(sigma*kappa + kappa^2*alpha)*(b - 1) = -a_ref/kappa
        rows[(3 * w + 0) * L[f] + l] = (float)bb;
        rows[(3 * w + 1) * L[f] + l] = (float)(-a_ref / kappa);
        rows[(3 * w + 2) * L[f] + l] = (float)(1.0 / kappa);
      }
    }
    prof.insert(prof.end(), rows.begin(), rows.end());
  }
  OEMS_CUDA(en->cpml.prof.ensure(prof.size()));
  OEMS_CUDA(cudaMemcpyAsync(en->cpml.prof.p, prof.data(), prof.size() * sizeof(float), cudaMemcpyHostToDevice,
                            en->stream));
  A.prof = en->cpml.prof.p;
  // z faces: psi rows start at a multiple of 4 in k so chunks map to aligned float4s
  A.zbase[0] = 0;
  A.zw[0] = (L[4] + 3) / 4 * 4;
  A.zbase[1] = L[5] > 0 ? (en->nz - L[5]) / 4 * 4 : 0;
  A.zw[1] = L[5] > 0 ? en->g.nzp - A.zbase[1] : 0;
  // psi arrays: per face 2 for H and 2 for E
  const size_t nzp = en->g.nzp;
  size_t face_sz[6];
  size_t total = 0;
  for (int f = 0; f < 6; ++f) {
    const int a = f / 2;
    if (L[f] == 0) {
      face_sz[f] = 0;
      continue;
    }
    if (a == 0) face_sz[f] = (size_t)L[f] * en->ny * nzp;
    else if (a == 1) face_sz[f] = (size_t)en->nx * L[f] * nzp;
    else face_sz[f] = (size_t)en->nx * en->ny * A.zw[f - 4];
    face_sz[f] = (face_sz[f] + 3) / 4 * 4;  // keep every array 16-byte aligned
    total += 4 * face_sz[f];
  }
  OEMS_CUDA(en->cpml.psi.ensure(total));
  OEMS_CUDA(cudaMemsetAsync(en->cpml.psi.p, 0, total * sizeof(float), en->stream));
  size_t off = 0;
  for (int f = 0; f < 6; ++f) {
    for (int s = 0; s < 2; ++s) {
      A.psi_h[f][s] = face_sz[f] ? en->cpml.psi.p + off : nullptr;
      off += face_sz[f];
      A.psi_e[f][s] = face_sz[f] ? en->cpml.psi.p + off : nullptr;
      off += face_sz[f];
    }
  }
  OEMS_CUDA(cudaStreamSynchronize(en->stream));
  en->cpml.on = true;
  en->cpml.desc = *d;
  en->tuned = false;  // the CPML kernels get their own launch shape
  LaunchShape s = en->shape;
  OEMS_TRY(size_grid(en, s));
  apply_shape(en, s);
  return OEMS_OK;
}

}  // namespace oems

// ---------------------------------------------------------------------------
// C ABI
// ---------------------------------------------------------------------------

using namespace oems;

// Launch helpers of the engine-interface entry points.
namespace {
struct KSample {
  template <typename T>
  static void go(const SampleArgs& a, int b, int t, cudaStream_t s) { k_iface_sample<T><<<b, t, 0, s>>>(a); }
};
struct KTerms {
  template <typename T>
  static void go(const TermArgs& a, int b, int t, cudaStream_t s) { k_iface_terms<T><<<b, t, 0, s>>>(a); }
};
struct KIntegral {
  template <typename T>
  static void go(const IntegralArgs& a, int b, int t, cudaStream_t s) { k_iface_integral<T><<<b, t, 0, s>>>(a); }
};
struct KSet {
  template <typename T>
  static void go(const SetArgs& a, int b, int t, cudaStream_t s) { k_iface_set<T><<<b, t, 0, s>>>(a); }
};
// Launches kernel K for the engine's field storage type.
template <typename K, typename A>
void launch_storage(const oems_engine* en, const A& a, int blocks, int threads) {
  if (en->storage == 1)
    K::template go<__half>(a, blocks, threads, en->stream);
  else if (en->storage == 2)
    K::template go<__nv_bfloat16>(a, blocks, threads, en->stream);
  else
    K::template go<float>(a, blocks, threads, en->stream);
}
}  // namespace

extern "C" {

oems_status oems_engine_create(const oems_operator_desc* desc, oems_engine** out) {
  g_last_error.clear();
  return create(desc, out);
}

void oems_engine_destroy(oems_engine* engine) {
  if (!engine) return;
  EngineScope guard(engine);
  destroy(engine);
}

oems_status oems_engine_run_batch(oems_engine* engine, const oems_batch* batch, oems_batch_result* result) {
  if (!engine) return fail(OEMS_ERR_INVALID_ARGUMENT, "NULL engine");
  g_last_error.clear();
  nvtxRangePushA("oems_engine_run_batch");
  const oems_status st = run_batch(engine, batch, result);
  nvtxRangePop();
  return st;
}

oems_status oems_engine_current_timestep(const oems_engine* engine, uint64_t* timestep) {
  if (!engine || !timestep) return fail(OEMS_ERR_INVALID_ARGUMENT, "NULL argument");
  *timestep = engine->timestep;
  return OEMS_OK;
}

oems_status oems_engine_read_fields(oems_engine* engine, float* const e[3], float* const h[3]) {
  if (!engine || !e || !h) return fail(OEMS_ERR_INVALID_ARGUMENT, "NULL argument");
  float* all[6] = {e[0], e[1], e[2], h[0], h[1], h[2]};
  return copy_fields(engine, all, true);
}

oems_status oems_engine_write_fields(oems_engine* engine, const float* const e[3], const float* const h[3]) {
  if (!engine || !e || !h) return fail(OEMS_ERR_INVALID_ARGUMENT, "NULL argument");
  float* all[6] = {const_cast<float*>(e[0]), const_cast<float*>(e[1]), const_cast<float*>(e[2]),
                   const_cast<float*>(h[0]), const_cast<float*>(h[1]), const_cast<float*>(h[2])};
  return copy_fields(engine, all, false);
}

oems_status oems_engine_reset(oems_engine* engine) {
  if (!engine) return fail(OEMS_ERR_INVALID_ARGUMENT, "NULL engine");
  EngineScope guard(engine);
  OEMS_CUDA(cudaMemsetAsync(engine->fields, 0, engine->field_bytes(), engine->stream));
  if (engine->cpml.on)
    OEMS_CUDA(cudaMemsetAsync(engine->cpml.psi.p, 0, engine->cpml.psi.n * sizeof(float), engine->stream));
  if (engine->mur.on)
    OEMS_CUDA(cudaMemsetAsync(engine->mur.state.p, 0, engine->mur.state.n * sizeof(float), engine->stream));
  if (!engine->entry_probe.empty())
    OEMS_CUDA(cudaMemsetAsync(engine->d_dft_acc.p, 0, 2 * engine->entry_probe.size() * sizeof(double),
                              engine->stream));
  for (auto& d : engine->disp)
    OEMS_CUDA(cudaMemsetAsync(d.state->p, 0, d.state->n * sizeof(float), engine->stream));
  if (!engine->rlc.q.empty())
    OEMS_CUDA(cudaMemsetAsync(engine->rlc.d_int.p, 0, engine->rlc.q.size() * sizeof(float), engine->stream));
  if (engine->upml.on)
    OEMS_CUDA(cudaMemsetAsync(engine->upml.flux.p, 0, engine->upml.flux.n * sizeof(float), engine->stream));
  for (auto& d : engine->fdumps)
    OEMS_CUDA(cudaMemsetAsync(d.acc->p, 0, d.acc->n * sizeof(double), engine->stream));
  for (auto& x : engine->boxes)
    OEMS_CUDA(cudaMemsetAsync(x.acc->p, 0, x.acc->n * sizeof(double), engine->stream));
  OEMS_CUDA(cudaStreamSynchronize(engine->stream));
  std::fill(engine->tfsf.e1d.begin(), engine->tfsf.e1d.end(), 0.0f);
  std::fill(engine->tfsf.h1d.begin(), engine->tfsf.h1d.end(), 0.0f);
  engine->tfsf.t = 0;
  engine->timestep = 0;
  engine->traces_steps = 0;
  return OEMS_OK;
}

// ---- state sections (checkpoint / resume) ---------------------------------
// Exactly the buffers oems_engine_reset clears, with the same pointers and
// byte counts, in a fixed order; the TF/SF 1D grid lives on the host.
}  // extern "C"

namespace {
struct StateSection {
  uint32_t kind;
  uint32_t variant;  // OEMS_STATE_FIELDS: the storage type; 0 otherwise
  void* dev;   // device buffer, or null for a host one
  void* host;  // host buffer, or null for a device one
  size_t bytes;
};

std::vector<StateSection> state_sections(oems_engine* en) {
  std::vector<StateSection> s;
  s.push_back({OEMS_STATE_FIELDS, (uint32_t)en->storage, en->fields, nullptr, en->field_bytes()});
  if (en->cpml.on) s.push_back({OEMS_STATE_CPML, 0, en->cpml.psi.p, nullptr, en->cpml.psi.n * sizeof(float)});
  if (en->mur.on) s.push_back({OEMS_STATE_MUR, 0, en->mur.state.p, nullptr, en->mur.state.n * sizeof(float)});
  if (!en->entry_probe.empty())
    s.push_back({OEMS_STATE_PROBE_DFT, 0, en->d_dft_acc.p, nullptr, 2 * en->entry_probe.size() * sizeof(double)});
  for (auto& d : en->disp)
    s.push_back({OEMS_STATE_DISPERSIVE, 0, d.state->p, nullptr, d.state->n * sizeof(float)});
  if (!en->rlc.q.empty())
    s.push_back({OEMS_STATE_LUMPED_RLC, 0, en->rlc.d_int.p, nullptr, en->rlc.q.size() * sizeof(float)});
  if (en->upml.on) s.push_back({OEMS_STATE_UPML, 0, en->upml.flux.p, nullptr, en->upml.flux.n * sizeof(float)});
  for (auto& d : en->fdumps)
    s.push_back({OEMS_STATE_FIELD_DFT, 0, d.acc->p, nullptr, d.acc->n * sizeof(double)});
  for (auto& x : en->boxes) s.push_back({OEMS_STATE_NF2FF, 0, x.acc->p, nullptr, x.acc->n * sizeof(double)});
  if (en->tfsf.on) {
    s.push_back({OEMS_STATE_TFSF_E, 0, nullptr, en->tfsf.e1d.data(), en->tfsf.e1d.size() * sizeof(float)});
    s.push_back({OEMS_STATE_TFSF_H, 0, nullptr, en->tfsf.h1d.data(), en->tfsf.h1d.size() * sizeof(float)});
  }
  return s;
}

oems_status state_copy(oems_engine* en, uint64_t index, void* out, const void* in, uint64_t bytes,
                       uint32_t variant) {
  const std::vector<StateSection> s = state_sections(en);
  if (index >= s.size()) return fail(OEMS_ERR_INVALID_ARGUMENT, "state section index out of range");
  const StateSection& q = s[index];
  if (bytes != q.bytes) return fail(OEMS_ERR_INVALID_ARGUMENT, "state section size differs from the engine's");
  if (!out && variant != q.variant)
    return fail(OEMS_ERR_CONFIG, "state section encoding differs from the engine's (field storage type)");
  if (bytes == 0) return OEMS_OK;
  if (q.host) {
    if (out) std::memcpy(out, q.host, bytes);
    else std::memcpy(q.host, in, bytes);
    return OEMS_OK;
  }
  if (!q.dev) return fail(OEMS_ERR_CONFIG, "state section has no buffer");
  if (out)
    OEMS_CUDA(cudaMemcpyAsync(out, q.dev, bytes, cudaMemcpyDeviceToHost, en->stream));
  else
    OEMS_CUDA(cudaMemcpyAsync(q.dev, in, bytes, cudaMemcpyHostToDevice, en->stream));
  OEMS_CUDA(cudaStreamSynchronize(en->stream));
  return OEMS_OK;
}
}  // namespace

extern "C" {

oems_status oems_engine_state_sections(oems_engine* engine, oems_state_section* out, uint64_t capacity,
                                       uint64_t* count) {
  if (!engine || (!out && capacity)) return fail(OEMS_ERR_INVALID_ARGUMENT, "NULL argument");
  const std::vector<StateSection> s = state_sections(engine);
  if (count) *count = s.size();
  for (size_t k = 0; k < s.size() && k < capacity; ++k) {
    out[k].kind = s[k].kind;
    out[k].variant = s[k].variant;
    out[k].bytes = s[k].bytes;
  }
  return OEMS_OK;
}

oems_status oems_engine_read_state(oems_engine* engine, uint64_t index, void* host, uint64_t bytes) {
  if (!engine || (!host && bytes)) return fail(OEMS_ERR_INVALID_ARGUMENT, "NULL argument");
  EngineScope guard(engine);
  return state_copy(engine, index, host, nullptr, bytes, 0);
}

oems_status oems_engine_write_state(oems_engine* engine, uint64_t index, uint32_t variant, const void* host,
                                    uint64_t bytes) {
  if (!engine || (!host && bytes)) return fail(OEMS_ERR_INVALID_ARGUMENT, "NULL argument");
  EngineScope guard(engine);
  return state_copy(engine, index, nullptr, host, bytes, variant);
}

oems_status oems_engine_get_state_counters(const oems_engine* engine, uint64_t* timestep, uint64_t* tfsf_step) {
  if (!engine) return fail(OEMS_ERR_INVALID_ARGUMENT, "NULL engine");
  if (timestep) *timestep = engine->timestep;
  if (tfsf_step) *tfsf_step = engine->tfsf.t;
  return OEMS_OK;
}

oems_status oems_engine_set_state_counters(oems_engine* engine, uint64_t timestep, uint64_t tfsf_step) {
  if (!engine) return fail(OEMS_ERR_INVALID_ARGUMENT, "NULL engine");
  engine->timestep = timestep;
  engine->tfsf.t = tfsf_step;
  engine->traces_steps = 0;
  return OEMS_OK;
}

oems_status oems_engine_add_cpml(oems_engine* engine, const oems_cpml_desc* desc) {
  if (!engine) return fail(OEMS_ERR_INVALID_ARGUMENT, "NULL engine");
  return add_cpml(engine, desc);
}

oems_status oems_engine_add_dispersive(oems_engine* engine, const oems_dispersive_desc* d, const uint64_t* cells,
                                       uint64_t ncells) {
  if (!engine || !d || (!cells && ncells)) return fail(OEMS_ERR_INVALID_ARGUMENT, "NULL argument");
  if (engine->storage) return fail(OEMS_ERR_CONFIG, "dispersive materials need float field storage");
  if (d->kind < 0 || d->kind > 4) return fail(OEMS_ERR_MATERIAL, "unknown dispersive material kind");
  if (!(d->eps_inf > 0.0)) return fail(OEMS_ERR_MATERIAL, "eps_inf must be positive");
  if (ncells == 0) return fail(OEMS_ERR_MATERIAL, "a dispersive material needs at least one cell");
  EngineScope guard(engine);
  DispHost h;
  DispArgs& A = h.args;
  A.kind = d->kind;
  const double dt = engine->dt, kEps0 = 8.854187817e-12;
  const double* p = d->params;
  if (d->kind == 0) {  // DrudeMaterial::new (src/extensions/dispersive.rs:476-498)
    const double den = 1.0 + p[1] * dt / 2.0;
    A.a = (float)((1.0 - p[1] * dt / 2.0) / den);
    A.b = (float)(kEps0 * p[0] * p[0] * dt / den);
    A.c = (float)(dt / (kEps0 * d->eps_inf));
  } else if (d->kind == 1 || d->kind == 3) {  // LorentzMaterial::new (:134-159)
    const double den = 1.0 + p[1] * dt / 2.0;
    A.a = (float)((2.0 - p[0] * p[0] * dt * dt) / den);
    A.b = (float)((p[1] * dt / 2.0 - 1.0) / den);
    A.c = (float)(kEps0 * p[2] * p[0] * p[0] * dt * dt / den);
    A.c2 = (float)(1.0 / (kEps0 * d->eps_inf));
  } else if (d->kind == 4) {  // Drude as a P recursion: P'' + g P' = eps0 wp^2 E
    const double den = 1.0 + p[1] * dt / 2.0;
    A.a = (float)(2.0 / den);
    A.b = (float)((p[1] * dt / 2.0 - 1.0) / den);
    A.c = (float)(kEps0 * p[0] * p[0] * dt * dt / den);
    A.c2 = (float)(1.0 / (kEps0 * d->eps_inf));
  } else {  // DebyeMaterial::new (:570-592)
    const double den = 2.0 * p[0] + dt;
    A.a = (float)((2.0 * p[0] - dt) / den);
    A.b = (float)(2.0 * kEps0 * p[1] * dt / den);
    A.c = (float)(dt / (kEps0 * d->eps_inf));
  }
  A.dtf = (float)dt;
  std::vector<long long> q(ncells);
  for (uint64_t m = 0; m < ncells; ++m) {
    const uint64_t* c = cells + 3 * m;
    if (c[0] >= (uint64_t)engine->nx || c[1] >= (uint64_t)engine->ny || c[2] >= (uint64_t)engine->nz)
      return fail(OEMS_ERR_MATERIAL, "dispersive cell outside the grid");
    q[m] = ((long long)c[0] * engine->ny + (long long)c[1]) * engine->g.nzp + (long long)c[2];
  }
  OEMS_CUDA(h.q->ensure(ncells));
  OEMS_CUDA(h.state->ensure(9 * ncells));
  OEMS_CUDA(cudaMemcpyAsync(h.q->p, q.data(), ncells * sizeof(long long), cudaMemcpyHostToDevice, engine->stream));
  OEMS_CUDA(cudaMemsetAsync(h.state->p, 0, 9 * ncells * sizeof(float), engine->stream));
  A.n = (long long)ncells;
  A.q = h.q->p;
  A.st = h.state->p;
  A.pp = h.state->p + 3 * ncells;
  A.ep = h.state->p + 6 * ncells;
  for (int c = 0; c < 3; ++c) A.e[c] = engine->E(c);
  engine->disp.push_back(std::move(h));
  engine->graph_epoch++;
  return OEMS_OK;
}

oems_status oems_engine_add_lumped_rlc(oems_engine* engine, const oems_lumped_rlc_desc* elems, uint64_t n) {
  if (!engine || (!elems && n)) return fail(OEMS_ERR_INVALID_ARGUMENT, "NULL argument");
  if (engine->storage) return fail(OEMS_ERR_CONFIG, "lumped RLC elements need float field storage");
  EngineScope guard(engine);
  RlcHost& R = engine->rlc;
  const double dt = engine->dt, kEps0 = 8.854187817e-12;
  for (uint64_t m = 0; m < n; ++m) {  // validate the whole list before taking any of it
    const oems_lumped_rlc_desc& e = elems[m];
    if (e.direction > 2) return fail(OEMS_ERR_CONFIG, "lumped element direction must be 0, 1 or 2");
    if (e.position[0] >= (uint64_t)engine->nx || e.position[1] >= (uint64_t)engine->ny ||
        e.position[2] >= (uint64_t)engine->nz)
      return fail(OEMS_ERR_CONFIG, "lumped element outside the grid");
  }
  for (uint64_t m = 0; m < n; ++m) {
    const oems_lumped_rlc_desc& e = elems[m];
    const double dl = engine->delta[e.direction], da = dl * dl;
    double v_vv, v_il;
    if (e.type == 0) {  // calc_parallel_coeffs (src/extensions/lumped_rlc.rs:190-216)
      const double g = e.resistance > 0 ? 1.0 / e.resistance : 0.0;
      const double inv_l = e.inductance > 0 ? dt / e.inductance : 0.0;
      const double cc = e.capacitance > 0 ? e.capacitance : 0.0;
      const double g_eff = g * dl / da, c_eff = cc * dl / da + kEps0 * dl / da;
      const double den = 2.0 * c_eff + g_eff * dt;
      v_vv = (2.0 * c_eff - g_eff * dt) / den;
      v_il = inv_l * dl / da;
    } else {  // calc_series_coeffs (:219-250): v_vv = 1 always
      const double rr = e.resistance > 0 ? e.resistance : 0.0, ll = e.inductance > 0 ? e.inductance : 0.0;
      const double inv_c = e.capacitance > 0 ? dt / e.capacitance : 0.0;
      const double den = 2.0 * (ll * da / dl) + (rr * da / dl) * dt;
      v_vv = 1.0;
      v_il = std::fabs(den) < 1e-20 ? 0.0 : inv_c * da / dl;
    }
    R.q.push_back(((long long)e.position[0] * engine->ny + (long long)e.position[1]) * engine->g.nzp +
                  (long long)e.position[2]);
    R.dir.push_back((int)e.direction);
    R.v_vv.push_back((float)v_vv);
    R.v_il.push_back((float)v_il);
  }
  const size_t k = R.q.size();
  if (k == 0) return OEMS_OK;
  OEMS_CUDA(R.d_q.ensure(k));
  OEMS_CUDA(R.d_dir.ensure(k));
  OEMS_CUDA(R.d_vv.ensure(k));
  OEMS_CUDA(R.d_vil.ensure(k));
  OEMS_CUDA(R.d_int.ensure(k));
  OEMS_CUDA(cudaMemcpyAsync(R.d_q.p, R.q.data(), k * sizeof(long long), cudaMemcpyHostToDevice, engine->stream));
  OEMS_CUDA(cudaMemcpyAsync(R.d_dir.p, R.dir.data(), k * sizeof(int), cudaMemcpyHostToDevice, engine->stream));
  OEMS_CUDA(cudaMemcpyAsync(R.d_vv.p, R.v_vv.data(), k * sizeof(float), cudaMemcpyHostToDevice, engine->stream));
  OEMS_CUDA(cudaMemcpyAsync(R.d_vil.p, R.v_il.data(), k * sizeof(float), cudaMemcpyHostToDevice, engine->stream));
  OEMS_CUDA(cudaMemsetAsync(R.d_int.p, 0, k * sizeof(float), engine->stream));
  engine->graph_epoch++;
  return OEMS_OK;
}

oems_status oems_engine_add_field_dft(oems_engine* engine, const oems_field_dft_desc* d, const double* freqs,
                                      uint32_t nfreq, int32_t* dump_id) {
  if (!engine || !d || (!freqs && nfreq)) return fail(OEMS_ERR_INVALID_ARGUMENT, "NULL argument");
  if (engine->storage) return fail(OEMS_ERR_CONFIG, "field DFT dumps need float field storage");
  if (nfreq == 0) return fail(OEMS_ERR_CONFIG, "a field DFT needs at least one frequency");
  if ((d->components & 0x3Fu) == 0 || (d->components & ~0x3Fu))
    return fail(OEMS_ERR_CONFIG, "field DFT components must be a non-empty mask of bits 0..5");
  EngineScope guard(engine);
  FieldDftHost h;
  FieldDftArgs& A = h.args;
  const long long ext[3] = {engine->nx, engine->ny, engine->nz};
  long long r[6], ss[3], n[3];
  A.npts = 1;
  for (int a = 0; a < 3; ++a) {
    r[2 * a] = (long long)std::min<uint64_t>(d->region[2 * a], (uint64_t)ext[a]);
    r[2 * a + 1] = (long long)std::min<uint64_t>(d->region[2 * a + 1], (uint64_t)ext[a]);
    ss[a] = std::max<uint32_t>(d->sub_sample[a], 1u);
    const long long len = std::max(r[2 * a + 1] - r[2 * a], 0LL);
    n[a] = (len + ss[a] - 1) / ss[a];
    A.npts *= n[a];
  }
  if (A.npts == 0) return fail(OEMS_ERR_CONFIG, "field DFT region is empty");
  for (int c = 0; c < 6; ++c)
    if (d->components >> c & 1u) {
      A.f[h.comps.size()] = c < 3 ? engine->E(c) : engine->H(c - 3);
      if (c >= 3) A.hmask |= 1u << h.comps.size();
      h.comps.push_back(c);
    }
  A.ncomp = (int)h.comps.size();
  A.nf = (int)nfreq;
  A.n1 = n[1];
  A.n2 = n[2];
  A.r0 = r[0];
  A.r1 = r[2];
  A.r2 = r[4];
  A.s0 = ss[0];
  A.s1 = ss[1];
  A.s2 = ss[2];
  A.ny = engine->ny;
  A.nzp = engine->g.nzp;
  h.freqs.assign(freqs, freqs + nfreq);
  h.interval = std::max<uint32_t>(d->interval, 1u);
  const size_t nacc = 2 * (size_t)nfreq * A.ncomp * (size_t)A.npts;
  OEMS_CUDA(h.acc->ensure(nacc));
  OEMS_CUDA(cudaMemsetAsync(h.acc->p, 0, nacc * sizeof(double), engine->stream));
  A.acc = reinterpret_cast<double2*>(h.acc->p);
  if (!engine->d_base.p) OEMS_CUDA(engine->d_base.ensure(1));
  engine->fdumps.push_back(std::move(h));
  engine->graph_epoch++;
  if (dump_id) *dump_id = (int32_t)engine->fdumps.size() - 1;
  return OEMS_OK;
}

oems_status oems_engine_read_field_dft(oems_engine* engine, int32_t id, uint32_t f, uint32_t component,
                                       double* out, uint64_t npoints) {
  if (!engine || !out) return fail(OEMS_ERR_INVALID_ARGUMENT, "NULL argument");
  if (id < 0 || id >= (int32_t)engine->fdumps.size()) return fail(OEMS_ERR_CONFIG, "unknown field DFT id");
  const FieldDftHost& h = engine->fdumps[id];
  if (f >= h.freqs.size()) return fail(OEMS_ERR_CONFIG, "frequency index out of range");
  const auto it = std::find(h.comps.begin(), h.comps.end(), (int)component);
  if (it == h.comps.end()) return fail(OEMS_ERR_CONFIG, "component not recorded by this field DFT");
  if (npoints < (uint64_t)h.args.npts) return fail(OEMS_ERR_INVALID_ARGUMENT, "output buffer too small");
  EngineScope guard(engine);
  const size_t slot = it - h.comps.begin();
  const size_t off = 2 * ((size_t)f * h.comps.size() + slot) * (size_t)h.args.npts;
  OEMS_CUDA(cudaStreamSynchronize(engine->stream));
  OEMS_CUDA(cudaMemcpyAsync(out, h.acc->p + off, 2 * (size_t)h.args.npts * sizeof(double), cudaMemcpyDeviceToHost,
                            engine->stream));
  OEMS_CUDA(cudaStreamSynchronize(engine->stream));
  return OEMS_OK;
}

oems_status oems_engine_add_nf2ff_box(oems_engine* engine, const oems_nf2ff_box_desc* d, const double* freqs,
                                      uint32_t nfreq, int32_t* box_id) {
  if (!engine || !d || (!freqs && nfreq)) return fail(OEMS_ERR_INVALID_ARGUMENT, "NULL argument");
  if (engine->storage) return fail(OEMS_ERR_CONFIG, "NF2FF boxes need float field storage");
  if (nfreq == 0) return fail(OEMS_ERR_CONFIG, "an NF2FF box needs at least one frequency");
  const long long ext[3] = {engine->nx, engine->ny, engine->nz};
  for (int a = 0; a < 3; ++a)
    if (d->start[a] < 1 || d->stop[a] <= d->start[a] || d->stop[a] > (uint64_t)ext[a] - 1)
      return fail(OEMS_ERR_CONFIG, "NF2FF box must satisfy 1 <= start < stop <= n - 1 on every axis");
  EngineScope guard(engine);
  Nf2ffHost h;
  Nf2ffAccArgs& A = h.args;
  for (int a = 0; a < 3; ++a) {
    h.lo[a] = (long long)d->start[a];
    h.hi[a] = (long long)d->stop[a];
  }
  size_t total = 0;
  A.off[0] = 0;
  for (int f = 0; f < 6; ++f) {
    if (!d->directions[f]) continue;
    Nf2ffFace& F = A.face[A.nfaces];
    F.a = f / 2;
    F.b = (F.a + 1) % 3;
    F.c = (F.a + 2) % 3;
    F.p = (f & 1) ? h.hi[F.a] : h.lo[F.a];
    F.lo_b = h.lo[F.b];
    F.lo_c = h.lo[F.c];
    F.nb = h.hi[F.b] - h.lo[F.b] + 1;
    F.nc = h.hi[F.c] - h.lo[F.c] + 1;
    F.np = F.nb * F.nc;
    h.sign[A.nfaces] = (f & 1) ? 1 : -1;
    total += (size_t)F.np;
    A.nfaces++;
    A.off[A.nfaces] = (long long)total;
  }
  if (A.nfaces == 0) return fail(OEMS_ERR_CONFIG, "NF2FF box has no face enabled");
  const size_t nacc = 8 * (size_t)nfreq * total;  // 4 complex values per point and frequency
  OEMS_CUDA(h.acc->ensure(nacc));
  OEMS_CUDA(cudaMemsetAsync(h.acc->p, 0, nacc * sizeof(double), engine->stream));
  size_t off = 0;
  for (int i = 0; i < A.nfaces; ++i) {
    A.face[i].acc = reinterpret_cast<double2*>(h.acc->p + off);
    off += 8 * (size_t)nfreq * (size_t)A.face[i].np;
  }
  for (int c = 0; c < 3; ++c) {
    A.e[c] = engine->E(c);
    A.h[c] = engine->H(c);
  }
  A.ny = engine->ny;
  A.nzp = engine->g.nzp;
  A.nf = (int)nfreq;
  h.freqs.assign(freqs, freqs + nfreq);
  h.interval = std::max<uint32_t>(d->interval, 1u);
  if (!engine->d_base.p) OEMS_CUDA(engine->d_base.ensure(1));
  engine->boxes.push_back(std::move(h));
  engine->graph_epoch++;
  if (box_id) *box_id = (int32_t)engine->boxes.size() - 1;
  return OEMS_OK;
}

oems_status oems_engine_read_nf2ff_face(oems_engine* engine, int32_t id, uint32_t face, uint32_t f, double* out,
                                        uint64_t cap_doubles, uint64_t* npoints) {
  if (!engine) return fail(OEMS_ERR_INVALID_ARGUMENT, "NULL engine");
  if (id < 0 || id >= (int32_t)engine->boxes.size()) return fail(OEMS_ERR_CONFIG, "unknown NF2FF box id");
  const Nf2ffHost& h = engine->boxes[id];
  if (f >= h.freqs.size() || face > 5) return fail(OEMS_ERR_CONFIG, "face or frequency index out of range");
  for (int i = 0; i < h.args.nfaces; ++i) {
    const Nf2ffFace& F = h.args.face[i];
    if (2 * F.a + (h.sign[i] > 0 ? 1 : 0) != (int)face) continue;
    if (npoints) *npoints = (uint64_t)F.np;
    if (!out) return OEMS_OK;
    if (cap_doubles < 8 * (uint64_t)F.np) return fail(OEMS_ERR_INVALID_ARGUMENT, "output buffer too small");
    EngineScope guard(engine);
    OEMS_CUDA(cudaStreamSynchronize(engine->stream));
    OEMS_CUDA(cudaMemcpyAsync(out, F.acc + (size_t)f * 4 * F.np, 8 * (size_t)F.np * sizeof(double),
                              cudaMemcpyDeviceToHost, engine->stream));
    OEMS_CUDA(cudaStreamSynchronize(engine->stream));
    return OEMS_OK;
  }
  return fail(OEMS_ERR_CONFIG, "face not recorded by this NF2FF box");
}

// Far field of a device point list on `stream`: directions over the theta x
// phi grid, radiation vectors on the GPU, then E_theta / E_phi, P_rad, Prad
// and Dmax on the host (python/openEMS/nf2ff.py:178-220 result fields).
static oems_status far_field(cudaStream_t stream, const double* d_pts, long long npts, double freq,
                             const oems_nf2ff_request* q, oems_nf2ff_result* res) {
  const long long nt = (long long)q->ntheta, np = (long long)q->nphi, ndir = nt * np;
  if (ndir > (1LL << 24)) return fail(OEMS_ERR_CONFIG, "too many far-field directions");
  std::vector<double> dirs(3 * ndir);
  for (long long i = 0; i < nt; ++i)
    for (long long j = 0; j < np; ++j) {
      const double th = q->theta[i], ph = q->phi[j];
      double* r = dirs.data() + 3 * (i * np + j);
      r[0] = std::sin(th) * std::cos(ph);
      r[1] = std::sin(th) * std::sin(ph);
      r[2] = std::cos(th);
    }
  const int dir_blocks = (int)((ndir + kFarThreads - 1) / kFarThreads);
  long long nchunks = std::max<long long>(1, (4 * 148 + dir_blocks - 1) / dir_blocks);
  nchunks = std::min<long long>(nchunks, std::max<long long>(1, (npts + kFarTile - 1) / kFarTile));
  nchunks = std::min<long long>(nchunks, 65535);
  long long chunk = (npts + nchunks - 1) / nchunks;
  chunk = (chunk + kFarTile - 1) / kFarTile * kFarTile;
  nchunks = (npts + chunk - 1) / chunk;
  DevBuf<double> d_dirs, d_partial, d_nl;
  OEMS_CUDA(d_dirs.ensure(3 * ndir));
  OEMS_CUDA(d_partial.ensure((size_t)nchunks * ndir * 12));
  OEMS_CUDA(d_nl.ensure((size_t)ndir * 12));
  OEMS_CUDA(cudaMemcpyAsync(d_dirs.p, dirs.data(), dirs.size() * sizeof(double), cudaMemcpyHostToDevice, stream));
  const double k = 2.0 * 3.14159265358979323846 * freq / 299792458.0;
  Nf2ffFarArgs a{};
  a.pts = d_pts;
  a.npts = npts;
  a.chunk = chunk;
  a.dirs = d_dirs.p;
  a.ndir = (int)ndir;
  a.k = k;
  a.cx = q->center[0];
  a.cy = q->center[1];
  a.cz = q->center[2];
  a.partial = d_partial.p;
  k_nf2ff_far<<<dim3(dir_blocks, (unsigned)nchunks), kFarThreads, 0, stream>>>(a);
  OEMS_CUDA(cudaGetLastError());
  k_nf2ff_reduce<<<(int)((ndir * 12 + 255) / 256), 256, 0, stream>>>(d_partial.p, (int)nchunks, (int)ndir, d_nl.p);
  OEMS_CUDA(cudaGetLastError());
  std::vector<double> nl((size_t)ndir * 12);
  OEMS_CUDA(cudaMemcpyAsync(nl.data(), d_nl.p, nl.size() * sizeof(double), cudaMemcpyDeviceToHost, stream));
  OEMS_CUDA(cudaStreamSynchronize(stream));
  const double eta = 376.730313668, R = q->radius, pi = 3.14159265358979323846;
  // fac = j k exp(-j k R) / (4 pi R)
  const double g = k / (4.0 * pi * R);
  const double fr = g * std::sin(k * R), fi = g * std::cos(k * R);
  double pmax = 0.0, prad = 0.0;
  auto trap = [](const double* x, long long n, long long i) {
    if (n < 2) return 0.0;
    if (i == 0) return 0.5 * (x[1] - x[0]);
    if (i == n - 1) return 0.5 * (x[n - 1] - x[n - 2]);
    return 0.5 * (x[i + 1] - x[i - 1]);
  };
  for (long long i = 0; i < nt; ++i)
    for (long long j = 0; j < np; ++j) {
      const long long dI = i * np + j;
      const double th = q->theta[i], ph = q->phi[j];
      const double tv[3] = {std::cos(th) * std::cos(ph), std::cos(th) * std::sin(ph), -std::sin(th)};
      const double pv[3] = {-std::sin(ph), std::cos(ph), 0.0};
      const double* v = nl.data() + 12 * dI;
      double Nt[2] = {0, 0}, Np[2] = {0, 0}, Lt[2] = {0, 0}, Lp[2] = {0, 0};
      for (int c = 0; c < 3; ++c) {
        Nt[0] += v[2 * c] * tv[c];
        Nt[1] += v[2 * c + 1] * tv[c];
        Np[0] += v[2 * c] * pv[c];
        Np[1] += v[2 * c + 1] * pv[c];
        Lt[0] += v[6 + 2 * c] * tv[c];
        Lt[1] += v[7 + 2 * c] * tv[c];
        Lp[0] += v[6 + 2 * c] * pv[c];
        Lp[1] += v[7 + 2 * c] * pv[c];
      }
      // E_theta = -fac (L_phi + eta N_theta); E_phi = fac (L_theta - eta N_phi)
      const double ar = Lp[0] + eta * Nt[0], ai = Lp[1] + eta * Nt[1];
      const double br = Lt[0] - eta * Np[0], bi = Lt[1] - eta * Np[1];
      const double etr = -(fr * ar - fi * ai), eti = -(fr * ai + fi * ar);
      const double epr = fr * br - fi * bi, epi = fr * bi + fi * br;
      if (res->e_theta) {
        res->e_theta[2 * dI] = etr;
        res->e_theta[2 * dI + 1] = eti;
      }
      if (res->e_phi) {
        res->e_phi[2 * dI] = epr;
        res->e_phi[2 * dI + 1] = epi;
      }
      const double p = (etr * etr + eti * eti + epr * epr + epi * epi) / (2.0 * eta);
      if (res->p_rad) res->p_rad[dI] = p;
      pmax = std::max(pmax, p);
      prad += p * R * R * std::sin(th) * trap(q->theta, nt, i) * trap(q->phi, np, j);
    }
  res->prad = prad;
  res->dmax = prad > 0.0 ? 4.0 * pi * R * R * pmax / prad : 0.0;
  return OEMS_OK;
}

static oems_status check_request(const oems_nf2ff_request* q, double freq) {
  if (!q || !q->theta || !q->phi) return fail(OEMS_ERR_INVALID_ARGUMENT, "NULL far-field request");
  if (q->ntheta == 0 || q->nphi == 0) return fail(OEMS_ERR_CONFIG, "empty theta or phi grid");
  if (!(q->radius > 0.0)) return fail(OEMS_ERR_CONFIG, "far-field radius must be positive");
  if (!(freq > 0.0)) return fail(OEMS_ERR_CONFIG, "frequency must be positive");
  return OEMS_OK;
}

oems_status oems_engine_nf2ff(oems_engine* engine, int32_t id, uint32_t f, const oems_nf2ff_request* q,
                              oems_nf2ff_result* res) {
  if (!engine || !res) return fail(OEMS_ERR_INVALID_ARGUMENT, "NULL argument");
  if (id < 0 || id >= (int32_t)engine->boxes.size()) return fail(OEMS_ERR_CONFIG, "unknown NF2FF box id");
  const Nf2ffHost& h = engine->boxes[id];
  if (f >= h.freqs.size()) return fail(OEMS_ERR_CONFIG, "frequency index out of range");
  OEMS_TRY(check_request(q, h.freqs[f]));
  EngineScope guard(engine);
  const long long ext[3] = {engine->nx, engine->ny, engine->nz};
  DevBuf<double> d_lines[3];
  Nf2ffPointsArgs P{};
  for (int a = 0; a < 3; ++a) {
    std::vector<double> l(ext[a] + 1);
    for (long long i = 0; i <= ext[a]; ++i) l[i] = q->lines[a] ? q->lines[a][i] : (double)i * engine->delta[a];
    OEMS_CUDA(d_lines[a].ensure(l.size()));
    OEMS_CUDA(cudaMemcpyAsync(d_lines[a].p, l.data(), l.size() * sizeof(double), cudaMemcpyHostToDevice,
                              engine->stream));
    P.lines[a] = d_lines[a].p;
  }
  P.nfaces = h.args.nfaces;
  P.off[0] = 0;
  for (int i = 0; i < P.nfaces; ++i) {
    P.face[i] = h.args.face[i];
    P.sign[i] = h.sign[i];
    const Nf2ffFace& F = P.face[i];
    P.off[i + 1] = P.off[i] + F.nb * (F.nc - 1) + (F.nb - 1) * F.nc;
  }
  P.f = (int)f;
  const long long npts = P.off[P.nfaces];
  DevBuf<double> pts;
  OEMS_CUDA(pts.ensure((size_t)npts * 16));
  P.pts = pts.p;
  k_nf2ff_points<<<(int)((npts + 255) / 256), 256, 0, engine->stream>>>(P);
  OEMS_CUDA(cudaGetLastError());
  return far_field(engine->stream, pts.p, npts, h.freqs[f], q, res);
}

oems_status oems_nf2ff_surface(int32_t device, const double* points, uint64_t npoints, double freq,
                               const oems_nf2ff_request* q, oems_nf2ff_result* res) {
  if (!points || !res) return fail(OEMS_ERR_INVALID_ARGUMENT, "NULL argument");
  if (npoints == 0) return fail(OEMS_ERR_CONFIG, "empty point list");
  OEMS_TRY(check_request(q, freq));
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) return fail(OEMS_ERR_NO_DEVICE, "no CUDA device");
  int dev = device;
  if (dev < 0) OEMS_CUDA(cudaGetDevice(&dev));
  DeviceGuard guard(dev);
  cudaStream_t stream = nullptr;
  OEMS_CUDA(cudaStreamCreateWithFlags(&stream, cudaStreamNonBlocking));
  oems_status st = OEMS_OK;
  {
    DevBuf<double> pts;
    cudaError_t e = pts.ensure((size_t)npoints * 16);
    if (e == cudaSuccess)
      e = cudaMemcpy(pts.p, points, (size_t)npoints * 16 * sizeof(double), cudaMemcpyHostToDevice);
    st = e == cudaSuccess ? far_field(stream, pts.p, (long long)npoints, freq, q, res)
                          : fail(OEMS_ERR_CUDA, cudaGetErrorString(e));
  }
  cudaStreamDestroy(stream);
  return st;
}

// Upml::calculate_kappa (src/extensions/pml.rs:370-420): conductivity at a
// node depth into the layer; the current grading is shifted by half a cell,
// -1/2 for the component along the PML direction, +1/2 otherwise.
static void upml_kappa(int comp, int dir, const long long pos[3], bool is_min, long long layers, double width,
                       double smax, double m, const long long n[3], const double delta[3], double* kv, double* ki) {
  const double d = delta[dir];
  double depth = 0.0;
  if (is_min) {
    if (pos[dir] <= layers) depth = (double)(layers - pos[dir]) * d;
  } else {
    const long long bs = n[dir] - layers - 1;
    if (pos[dir] >= bs) depth = (double)(pos[dir] - bs) * d;
  }
  if (depth <= 0.0) {
    *kv = *ki = 0.0;
    return;
  }
  *kv = smax * std::pow(depth / width, m);
  const double di = depth + (comp == dir ? -0.5 : 0.5) * d;
  const double ni = std::min(std::max(di / width, 0.0), 1.0);
  *ki = smax * std::pow(ni, m);
}

// Conductivity of the corrected UPML along axis `dir` at index i, at the node
// (half = false) or half a cell above it, over both faces of that axis (a
// position lies in at most one slab): sigma_max (depth / width)^m with the
// depth from the region's inner node, L at a min face and n - L - 1 at a max
// face (the nodes the reference grades from, pml.rs:370-420), taken at the
// Yee position of the component.
static double upml_sigma_axis(const long long L[6], int dir, long long i, bool half, double m, double R0,
                              const long long n[3], const double delta[3]) {
  const double z0 = 376.730313668;
  double sg = 0.0;
  for (int side = 0; side < 2; ++side) {
    const long long l = L[2 * dir + side];
    if (l <= 0 || l >= n[dir]) continue;
    const double smax = -(m + 1.0) * std::log(R0) / (2.0 * z0 * (double)l * delta[dir]);
    const double x = (double)i + (half ? 0.5 : 0.0);
    double depth = side == 0 ? (double)l - x : x - (double)(n[dir] - l - 1);
    depth = std::min(std::max(depth, 0.0), (double)l);
    sg = std::max(sg, smax * std::pow(depth / (double)l, m));
  }
  return sg;
}

oems_status oems_engine_add_upml(oems_engine* engine, const oems_upml_desc* desc) {
  if (!engine || !desc) return fail(OEMS_ERR_INVALID_ARGUMENT, "NULL argument");
  if (engine->storage) return fail(OEMS_ERR_CONFIG, "UPML needs float field storage");
  if (desc->kind != 0 && desc->kind != 1) return fail(OEMS_ERR_CONFIG, "UPML kind must be 0 or 1");
  if (desc->kind == 1 && engine->id_bytes != 0)
    return fail(OEMS_ERR_CONFIG, "the corrected UPML rewrites coefficients: needs full coefficient arrays");
  if (engine->upml.on) return fail(OEMS_ERR_CONFIG, "UPML already attached");
  if (!(desc->reflection_coeff > 0.0 && desc->reflection_coeff < 1.0))
    return fail(OEMS_ERR_CONFIG, "UPML reflection coefficient must be in (0, 1)");
  EngineScope guard(engine);
  const long long n[3] = {engine->nx, engine->ny, engine->nz};
  const long long* L = nullptr;
  long long lay[6];
  for (int f = 0; f < 6; ++f) lay[f] = (long long)desc->layers[f];
  L = lay;
  // Upml::build_regions (pml.rs:222-296): x slabs over the full y-z plane,
  // y slabs without the x corners, z slabs without x and y edges.
  struct Reg {
    long long start[3], size[3];
    int dir;
    bool is_min;
  };
  std::vector<Reg> regs;
  if (L[0] > 0 && L[0] < n[0]) regs.push_back({{0, 0, 0}, {L[0] + 1, n[1], n[2]}, 0, true});
  if (L[1] > 0 && L[1] < n[0]) regs.push_back({{n[0] - L[1] - 1, 0, 0}, {L[1] + 1, n[1], n[2]}, 0, false});
  const long long xs = L[0] > 0 ? L[0] + 1 : 0, xe = L[1] > 0 ? n[0] - L[1] - 1 : n[0];
  if (L[2] > 0 && L[2] < n[1] && xs < xe) regs.push_back({{xs, 0, 0}, {xe - xs, L[2] + 1, n[2]}, 1, true});
  if (L[3] > 0 && L[3] < n[1] && xs < xe)
    regs.push_back({{xs, n[1] - L[3] - 1, 0}, {xe - xs, L[3] + 1, n[2]}, 1, false});
  const long long ys = L[2] > 0 ? L[2] + 1 : 0, ye = L[3] > 0 ? n[1] - L[3] - 1 : n[1];
  if (L[4] > 0 && L[4] < n[2] && xs < xe && ys < ye)
    regs.push_back({{xs, ys, 0}, {xe - xs, ye - ys, L[4] + 1}, 2, true});
  if (L[5] > 0 && L[5] < n[2] && xs < xe && ys < ye)
    regs.push_back({{xs, ys, n[2] - L[5] - 1}, {xe - xs, ye - ys, L[5] + 1}, 2, false});
  if (regs.empty()) return fail(OEMS_ERR_CONFIG, "UPML has no active region");
  long long total = 0;
  for (const Reg& r : regs) total += r.size[0] * r.size[1] * r.size[2];
  // Upml::init_region_coefficients (pml.rs:299-367)
  std::vector<float> ce(9 * (size_t)total), ch(9 * (size_t)total);
  const double dt = engine->dt, m = desc->grading_order, eps0 = 8.854187817e-12, z0 = 376.730313668;
  // kind 1 rewrites the region cells' main coefficients: work on a host copy
  // of the 12 arrays (padded layout), uploaded again below
  const size_t ncoef = (size_t)engine->ncells_padded;
  std::vector<float> coef;
  if (desc->kind == 1) {
    coef.resize(12 * ncoef);
    for (int a = 0; a < 12; ++a)
      OEMS_CUDA(cudaMemcpyAsync(coef.data() + a * ncoef, engine->C(a), ncoef * sizeof(float),
                                cudaMemcpyDeviceToHost, engine->stream));
    OEMS_CUDA(cudaStreamSynchronize(engine->stream));
  }
  long long base = 0;
  for (const Reg& r : regs) {
    const long long layers = L[2 * r.dir + (r.is_min ? 0 : 1)];
    const double width = (double)layers * engine->delta[r.dir];
    const double smax = -(m + 1.0) * std::log(desc->reflection_coeff) / (2.0 * z0 * width);
    long long t = 0;
    for (long long li = 0; li < r.size[0]; ++li)
      for (long long lj = 0; lj < r.size[1]; ++lj)
        for (long long lk = 0; lk < r.size[2]; ++lk, ++t) {
          const long long pos[3] = {r.start[0] + li, r.start[1] + lj, r.start[2] + lk};
          if (desc->kind == 1) {
            // Taflove & Hagness 7.8 for component c (cp, cpp the next axes):
            // D_c advances with sigma_cp in the main update, E_c follows
            // from D_c through the hooks with sigma_cpp and sigma_c; H likewise
            const size_t qc = (size_t)((pos[0] * engine->ny + pos[1]) * engine->g.nzp + pos[2]);
            const size_t q = (size_t)(base + t);
            for (int c = 0; c < 3; ++c) {
              double sv[3], si[3];
              for (int dd = 0; dd < 3; ++dd) {
                sv[dd] = upml_sigma_axis(L, dd, pos[dd], c == dd, m, desc->reflection_coeff, n, engine->delta);
                si[dd] = upml_sigma_axis(L, dd, pos[dd], c != dd, m, desc->reflection_coeff, n, engine->delta);
              }
              const int np = (c + 1) % 3, npp = (c + 2) % 3;
              const double dv = 2.0 * eps0 + sv[npp] * dt, di = 2.0 * eps0 + si[npp] * dt;
              ce[(0 * 3 + c) * total + q] = (float)((2.0 * eps0 - sv[npp] * dt) / dv);
              ce[(1 * 3 + c) * total + q] = (float)((2.0 * eps0 - sv[c] * dt) / dv);
              ce[(2 * 3 + c) * total + q] = (float)((2.0 * eps0 + sv[c] * dt) / dv);
              ch[(0 * 3 + c) * total + q] = (float)((2.0 * eps0 - si[npp] * dt) / di);
              ch[(1 * 3 + c) * total + q] = (float)((2.0 * eps0 - si[c] * dt) / di);
              ch[(2 * 3 + c) * total + q] = (float)((2.0 * eps0 + si[c] * dt) / di);
              float* ca = coef.data() + (size_t)c * ncoef;
              float* cb = coef.data() + (size_t)(3 + c) * ncoef;
              float* da = coef.data() + (size_t)(6 + c) * ncoef;
              float* db = coef.data() + (size_t)(9 + c) * ncoef;
              if (ca[qc] != 0.0f || cb[qc] != 0.0f) {
                ca[qc] = (float)((2.0 * eps0 - sv[np] * dt) / (2.0 * eps0 + sv[np] * dt));
                cb[qc] = (float)((double)cb[qc] * (2.0 * eps0 / (2.0 * eps0 + sv[np] * dt)));
              }
              if (da[qc] != 0.0f || db[qc] != 0.0f) {
                da[qc] = (float)((2.0 * eps0 - si[np] * dt) / (2.0 * eps0 + si[np] * dt));
                db[qc] = (float)((double)db[qc] * (2.0 * eps0 / (2.0 * eps0 + si[np] * dt)));
              }
            }
            continue;
          }
          double kv[3], ki[3];
          for (int c = 0; c < 3; ++c)
            upml_kappa(c, r.dir, pos, r.is_min, layers, width, smax, m, n, engine->delta, &kv[c], &ki[c]);
          for (int c = 0; c < 3; ++c) {
            const int npp = (c + 2) % 3;
            const size_t q = (size_t)(base + t);
            float* v[3] = {&ce[(0 * 3 + c) * total + q], &ce[(1 * 3 + c) * total + q], &ce[(2 * 3 + c) * total + q]};
            float* w[3] = {&ch[(0 * 3 + c) * total + q], &ch[(1 * 3 + c) * total + q], &ch[(2 * 3 + c) * total + q]};
            if (kv[0] + kv[1] + kv[2] > 0.0) {
              const double den = 2.0 * eps0 + kv[npp] * dt;
              *v[0] = (float)((2.0 * eps0 - kv[npp] * dt) / den);
              *v[1] = (float)((2.0 * eps0 - kv[c] * dt) / den);
              *v[2] = (float)((2.0 * eps0 + kv[c] * dt) / den);
            } else {
              *v[0] = 1.0f;
              *v[1] = 0.0f;
              *v[2] = 1.0f;
            }
            if (ki[0] + ki[1] + ki[2] > 0.0) {
              const double den = 2.0 * eps0 + ki[npp] * dt;
              *w[0] = (float)((2.0 * eps0 - ki[npp] * dt) / den);
              *w[1] = (float)((2.0 * eps0 - ki[c] * dt) / den);
              *w[2] = (float)((2.0 * eps0 + ki[c] * dt) / den);
            } else {
              *w[0] = 1.0f;
              *w[1] = 0.0f;
              *w[2] = 1.0f;
            }
          }
        }
    base += t;
  }
  if (desc->kind == 1)
    for (int a = 0; a < 12; ++a)
      OEMS_CUDA(cudaMemcpyAsync(engine->C(a), coef.data() + a * ncoef, ncoef * sizeof(float),
                                cudaMemcpyHostToDevice, engine->stream));
  UpmlHost& U = engine->upml;
  OEMS_CUDA(U.coef.ensure(18 * (size_t)total));
  OEMS_CUDA(U.flux.ensure(6 * (size_t)total));
  OEMS_CUDA(cudaMemcpyAsync(U.coef.p, ce.data(), ce.size() * sizeof(float), cudaMemcpyHostToDevice, engine->stream));
  OEMS_CUDA(cudaMemcpyAsync(U.coef.p + 9 * total, ch.data(), ch.size() * sizeof(float), cudaMemcpyHostToDevice,
                            engine->stream));
  OEMS_CUDA(cudaMemsetAsync(U.flux.p, 0, 6 * (size_t)total * sizeof(float), engine->stream));
  for (UpmlArgs* a : {&U.e, &U.h}) {
    *a = UpmlArgs{};
    a->nreg = (int)regs.size();
    a->off[0] = 0;
    for (size_t i = 0; i < regs.size(); ++i) {
      for (int k = 0; k < 3; ++k) {
        a->start[i][k] = regs[i].start[k];
        a->size[i][k] = regs[i].size[k];
      }
      a->off[i + 1] = a->off[i] + regs[i].size[0] * regs[i].size[1] * regs[i].size[2];
    }
    for (size_t i = regs.size(); i < 6; ++i) a->off[i + 1] = a->off[regs.size()];
    a->total = total;
    a->ny = engine->ny;
    a->nzp = engine->g.nzp;
  }
  U.e.coef = U.coef.p;
  U.h.coef = U.coef.p + 9 * total;
  U.e.flux = U.flux.p;
  U.h.flux = U.flux.p + 3 * total;
  for (int c = 0; c < 3; ++c) {
    U.e.f[c] = engine->E(c);
    U.h.f[c] = engine->H(c);
  }
  U.on = true;
  engine->graph_epoch++;
  return OEMS_OK;
}

oems_status oems_engine_add_tfsf(oems_engine* engine, const oems_tfsf_desc* d) {
  if (!engine || !d) return fail(OEMS_ERR_INVALID_ARGUMENT, "NULL argument");
  if (engine->storage) return fail(OEMS_ERR_CONFIG, "TF/SF needs float field storage");
  if (engine->tfsf.on) return fail(OEMS_ERR_CONFIG, "TF/SF already attached");
  if (d->direction < 0 || d->direction > 5) return fail(OEMS_ERR_CONFIG, "TF/SF direction must be 0..5");
  if (d->polarization < 0 || d->polarization > 1) return fail(OEMS_ERR_CONFIG, "TF/SF polarization must be 0 or 1");
  if (!std::isfinite(d->frequency) || !std::isfinite(d->amplitude))
    return fail(OEMS_ERR_CONFIG, "TF/SF frequency and amplitude must be finite");
  TfsfHost& T = engine->tfsf;
  const int prop = d->direction / 2;
  const int n[3] = {engine->nx, engine->ny, engine->nz};
  if (d->boundary_layer >= (uint64_t)n[prop]) return fail(OEMS_ERR_CONFIG, "TF/SF boundary layer outside the grid");
  if (d->kind < 0 || d->kind > 1) return fail(OEMS_ERR_CONFIG, "TF/SF kind must be 0 or 1");
  if (d->kind == 1 && (d->boundary_layer < 1 || d->direction % 2 != 0))
    return fail(OEMS_ERR_CONFIG, "the corrected TF/SF needs a positive direction and boundary_layer >= 1");
  T.kind = d->kind;
  T.prop = prop;
  T.e_axis = d->polarization == 0 ? (prop + 1) % 3 : (prop + 2) % 3;
  T.h_axis = d->polarization == 0 ? (prop + 2) % 3 : (prop + 1) % 3;
  T.pos = (long long)d->boundary_layer;
  T.freq = d->frequency;
  T.amp = d->amplitude;
  T.v = d->phase_velocity > 0.0 ? d->phase_velocity : 299792458.0;
  T.e1d.assign(n[prop] + 1, 0.0f);
  T.h1d.assign(n[prop] + 1, 0.0f);
  T.t = 0;
  T.on = true;
  engine->graph_epoch++;
  return OEMS_OK;
}

oems_status oems_engine_add_mur(oems_engine* engine, const oems_mur_desc* desc) {
  if (!engine) return fail(OEMS_ERR_INVALID_ARGUMENT, "NULL engine");
  return add_mur(engine, desc);
}

oems_status oems_engine_add_probe(oems_engine* engine, const oems_probe_term* terms, uint64_t nterms, int32_t mode,
                                  int32_t* probe_id) {
  // no terms is valid: the probe reads 0 (a VoltageProbe with an invalid
  // direction, src/processing/probes.rs:125)
  if (!engine || (!terms && nterms)) return fail(OEMS_ERR_INVALID_ARGUMENT, "NULL argument");
  if (mode != OEMS_PROBE_SUM_F32 && mode != OEMS_PROBE_SUM_F64) return fail(OEMS_ERR_CONFIG, "unknown probe mode");
  if (engine->term_idx.size() + nterms > (size_t)INT32_MAX) return fail(OEMS_ERR_CONFIG, "too many probe terms");
  bool all_h = nterms > 0;
  for (uint64_t t = 0; t < nterms; ++t) {
    const oems_probe_term& q = terms[t];
    if (q.component < 0 || q.component > 5) return fail(OEMS_ERR_CONFIG, "probe component must be 0..5");
    if (q.position[0] >= (uint64_t)engine->nx || q.position[1] >= (uint64_t)engine->ny ||
        q.position[2] >= (uint64_t)engine->nz)
      return fail(OEMS_ERR_CONFIG, "probe position outside the grid");
    if (!std::isfinite(q.weight)) return fail(OEMS_ERR_CONFIG, "probe weight must be finite");
    all_h = all_h && q.component >= 3;
  }
  EngineScope guard(engine);
  for (uint64_t t = 0; t < nterms; ++t) {
    const oems_probe_term& q = terms[t];
    engine->term_idx.push_back(((long long)q.position[0] * engine->ny + (long long)q.position[1]) * engine->g.nzp +
                               (long long)q.position[2]);
    engine->term_comp.push_back(q.component);
    engine->term_w.push_back(q.weight);
  }
  engine->probe_off.push_back((int)engine->term_idx.size());
  engine->probe_mode.push_back(mode);
  engine->probe_half.push_back(all_h ? 0.5 : 0.0);
  const size_t np = engine->probe_mode.size(), nt = engine->term_idx.size();
  OEMS_CUDA(engine->d_probe_off.ensure(np + 1));
  OEMS_CUDA(engine->d_probe_mode.ensure(np));
  OEMS_CUDA(engine->d_term_idx.ensure(nt));
  OEMS_CUDA(engine->d_term_comp.ensure(nt));
  OEMS_CUDA(engine->d_term_w.ensure(nt));
  OEMS_CUDA(cudaMemcpyAsync(engine->d_probe_off.p, engine->probe_off.data(), (np + 1) * sizeof(int), cudaMemcpyHostToDevice, engine->stream));
  OEMS_CUDA(cudaMemcpyAsync(engine->d_probe_mode.p, engine->probe_mode.data(), np * sizeof(int), cudaMemcpyHostToDevice, engine->stream));
  OEMS_CUDA(cudaMemcpyAsync(engine->d_term_idx.p, engine->term_idx.data(), nt * sizeof(long long), cudaMemcpyHostToDevice, engine->stream));
  OEMS_CUDA(cudaMemcpyAsync(engine->d_term_comp.p, engine->term_comp.data(), nt * sizeof(int), cudaMemcpyHostToDevice, engine->stream));
  OEMS_CUDA(cudaMemcpyAsync(engine->d_term_w.p, engine->term_w.data(), nt * sizeof(double), cudaMemcpyHostToDevice, engine->stream));
  engine->d_traces.ensure(0);
  engine->traces_steps = 0;
  engine->graph_epoch++;  // device table pointers and the probe count are baked into graphs
  if (probe_id) *probe_id = (int32_t)(np - 1);
  return OEMS_OK;
}

oems_status oems_engine_add_point_probe(oems_engine* engine, int32_t component, const uint64_t position[3],
                                        int32_t* probe_id) {
  if (!position) return fail(OEMS_ERR_INVALID_ARGUMENT, "NULL argument");
  oems_probe_term t{};
  t.component = component;
  for (int a = 0; a < 3; ++a) t.position[a] = position[a];
  t.weight = 1.0;
  return oems_engine_add_probe(engine, &t, 1, OEMS_PROBE_SUM_F32, probe_id);
}

oems_status oems_engine_read_probe_traces(oems_engine* engine, double* out, uint64_t max_steps, uint64_t* steps_out) {
  if (!engine) return fail(OEMS_ERR_INVALID_ARGUMENT, "NULL engine");
  const uint64_t steps = std::min<uint64_t>(engine->traces_steps, max_steps);
  if (steps_out) *steps_out = engine->traces_steps;
  const size_t np = engine->nprobe();
  if (steps == 0 || np == 0) return OEMS_OK;
  if (!out) return fail(OEMS_ERR_INVALID_ARGUMENT, "NULL output buffer");
  EngineScope guard(engine);
  OEMS_CUDA(cudaMemcpyAsync(out, engine->d_traces.p, steps * np * sizeof(double), cudaMemcpyDeviceToHost,
                            engine->stream));
  OEMS_CUDA(cudaStreamSynchronize(engine->stream));
  return OEMS_OK;
}

oems_status oems_engine_add_probe_dft(oems_engine* engine, int32_t probe_id, const double* freqs, uint64_t nfreq,
                                      int32_t* dft_id) {
  if (!engine || (!freqs && nfreq)) return fail(OEMS_ERR_INVALID_ARGUMENT, "NULL argument");
  if (probe_id < 0 || probe_id >= engine->nprobe()) return fail(OEMS_ERR_CONFIG, "unknown probe");
  if (nfreq == 0) return fail(OEMS_ERR_CONFIG, "a DFT needs at least one frequency");
  EngineScope guard(engine);
  engine->dft_first.push_back((int)engine->entry_probe.size());
  engine->dft_count.push_back((int)nfreq);
  for (uint64_t f = 0; f < nfreq; ++f) {
    engine->entry_probe.push_back(probe_id);
    engine->entry_freq.push_back(freqs[f]);
    engine->entry_half.push_back(engine->probe_half[probe_id]);
  }
  const size_t ne = engine->entry_probe.size();
  // keep the accumulated values of existing DFTs
  std::vector<double> acc(2 * ne, 0.0);
  const size_t old = ne - nfreq;
  cudaStream_t s = engine->stream;
  if (old) {
    OEMS_CUDA(cudaMemcpyAsync(acc.data(), engine->d_dft_acc.p, 2 * old * sizeof(double), cudaMemcpyDeviceToHost, s));
    OEMS_CUDA(cudaStreamSynchronize(s));
  }
  OEMS_CUDA(engine->d_entry_probe.ensure(ne));
  OEMS_CUDA(engine->d_entry_freq.ensure(ne));
  OEMS_CUDA(engine->d_entry_half.ensure(ne));
  OEMS_CUDA(engine->d_dft_acc.ensure(2 * ne));
  OEMS_CUDA(cudaMemcpyAsync(engine->d_entry_probe.p, engine->entry_probe.data(), ne * sizeof(int),
                            cudaMemcpyHostToDevice, s));
  OEMS_CUDA(cudaMemcpyAsync(engine->d_entry_freq.p, engine->entry_freq.data(), ne * sizeof(double),
                            cudaMemcpyHostToDevice, s));
  OEMS_CUDA(cudaMemcpyAsync(engine->d_entry_half.p, engine->entry_half.data(), ne * sizeof(double),
                            cudaMemcpyHostToDevice, s));
  OEMS_CUDA(cudaMemcpyAsync(engine->d_dft_acc.p, acc.data(), 2 * ne * sizeof(double), cudaMemcpyHostToDevice, s));
  OEMS_CUDA(cudaStreamSynchronize(s));
  if (dft_id) *dft_id = (int32_t)engine->dft_first.size() - 1;
  return OEMS_OK;
}

oems_status oems_engine_read_probe_dft(oems_engine* engine, int32_t dft_id, double* out) {
  if (!engine || !out) return fail(OEMS_ERR_INVALID_ARGUMENT, "NULL argument");
  if (dft_id < 0 || dft_id >= (int32_t)engine->dft_first.size()) return fail(OEMS_ERR_CONFIG, "unknown DFT");
  EngineScope guard(engine);
  OEMS_CUDA(cudaMemcpyAsync(out, engine->d_dft_acc.p + 2 * engine->dft_first[dft_id],
                            2 * engine->dft_count[dft_id] * sizeof(double), cudaMemcpyDeviceToHost, engine->stream));
  OEMS_CUDA(cudaStreamSynchronize(engine->stream));
  return OEMS_OK;
}


oems_status oems_engine_energy(oems_engine* engine, double* e_energy, double* h_energy) {
  if (!engine) return fail(OEMS_ERR_INVALID_ARGUMENT, "NULL engine");
  EngineScope guard(engine);
  OEMS_CUDA(engine->d_energy.ensure(2));
  OEMS_TRY(launch_energy(engine, engine->d_energy.p));
  double out[2];
  OEMS_CUDA(cudaMemcpyAsync(out, engine->d_energy.p, sizeof(out), cudaMemcpyDeviceToHost, engine->stream));
  OEMS_CUDA(cudaStreamSynchronize(engine->stream));
  if (e_energy) *e_energy = out[0];
  if (h_energy) *h_energy = out[1];
  return OEMS_OK;
}

// ---------------------------------------------------------------------------
// engine interface (src/fdtd/engine_interface.rs:27-595)
// ---------------------------------------------------------------------------


// Checks a sample descriptor's grid against the engine; *words = the lines' count.
static oems_status check_sample_grid(const oems_engine* en, const oems_sample_desc* d, uint64_t* words) {
  if (!std::isfinite(d->unit) || d->unit == 0.0) return fail(OEMS_ERR_CONFIG, "grid unit must be finite and non-zero");
  const int ext[3] = {en->nx, en->ny, en->nz};
  *words = 0;
  for (int ax = 0; ax < 3; ++ax) {
    const uint64_t nl = d->nlines[ax];
    if (!d->lines[ax] || nl == 0) return fail(OEMS_ERR_INVALID_ARGUMENT, "mesh lines missing");
    if (std::max<uint64_t>(nl, 2) - 1 != (uint64_t)ext[ax])
      return fail(OEMS_ERR_CONFIG, "mesh lines do not match the engine's grid");
    *words += nl;
  }
  return OEMS_OK;
}

// The grid part of SampleArgs, with the lines copied to words base[0..).
static oems_status upload_sample_grid(oems_engine* en, const oems_sample_desc* d, unsigned long long* base,
                                      SampleArgs* a) {
  for (int c = 0; c < 6; ++c) a->f[c] = c < 3 ? en->E(c) : en->H(c - 3);
  a->nx = en->nx;
  a->ny = en->ny;
  a->nz = en->nz;
  a->nzp = en->g.nzp;
  uint64_t off = 0;
  for (int ax = 0; ax < 3; ++ax) {
    a->lines[ax] = reinterpret_cast<const double*>(base + off);
    a->nl[ax] = (int)d->nlines[ax];
    a->sorted[ax] = std::is_sorted(d->lines[ax], d->lines[ax] + d->nlines[ax]) ? 1 : 0;
    OEMS_CUDA(cudaMemcpyAsync(base + off, d->lines[ax], d->nlines[ax] * 8, cudaMemcpyHostToDevice, en->stream));
    off += d->nlines[ax];
  }
  a->unit = d->unit;
  a->h_inv = 1.0f / en->h_scale;
  return OEMS_OK;
}

oems_status oems_engine_sample(oems_engine* engine, const oems_sample_desc* desc, const double* positions,
                               const uint64_t* cells, uint64_t count, double* values, uint64_t* snapped) {
  if (!engine || !desc) return fail(OEMS_ERR_INVALID_ARGUMENT, "NULL engine or descriptor");
  if (count == 0) return OEMS_OK;
  if (!values) return fail(OEMS_ERR_INVALID_ARGUMENT, "NULL values");
  if ((positions != nullptr) == (cells != nullptr))
    return fail(OEMS_ERR_INVALID_ARGUMENT, "give either positions or cells");
  if (desc->quantity < OEMS_SAMPLE_E || desc->quantity > OEMS_SAMPLE_CURL_H)
    return fail(OEMS_ERR_CONFIG, "sample quantity must be E, H or curl H");
  if (desc->interpolation < OEMS_INTERP_NONE || desc->interpolation > OEMS_INTERP_CELL)
    return fail(OEMS_ERR_CONFIG, "unknown interpolation");
  if (count > (uint64_t)1 << 31) return fail(OEMS_ERR_CONFIG, "at most 2^31 queries per call");
  uint64_t nl_total = 0;
  OEMS_TRY(check_sample_grid(engine, desc, &nl_total));
  if (cells)
    for (uint64_t q = 0; q < count; ++q)
      if (cells[3 * q] >= (uint64_t)engine->nx || cells[3 * q + 1] >= (uint64_t)engine->ny ||
          cells[3 * q + 2] >= (uint64_t)engine->nz)
        return fail(OEMS_ERR_CONFIG, "cell outside the grid");
  EngineScope guard(engine);
  // words: lines | queries (3 per) | values (3 per) | snapped cells (3 per)
  const uint64_t w_q = nl_total, w_v = w_q + 3 * count, w_c = w_v + 3 * count, words = w_c + 3 * count;
  OEMS_CUDA(engine->d_iface.ensure(words));
  unsigned long long* base = engine->d_iface.p;
  SampleArgs a{};
  OEMS_TRY(upload_sample_grid(engine, desc, base, &a));
  if (positions) {
    a.pos = reinterpret_cast<const double*>(base + w_q);
    OEMS_CUDA(cudaMemcpyAsync(base + w_q, positions, 3 * count * 8, cudaMemcpyHostToDevice, engine->stream));
  } else {
    a.cells_in = base + w_q;
    OEMS_CUDA(cudaMemcpyAsync(base + w_q, cells, 3 * count * 8, cudaMemcpyHostToDevice, engine->stream));
  }
  a.count = (long long)count;
  a.quantity = desc->quantity;
  a.interp = desc->interpolation;
  a.out = reinterpret_cast<double*>(base + w_v);
  a.cells_out = base + w_c;
  launch_storage<KSample>(engine, a, (int)((count + 127) / 128), 128);
  OEMS_CUDA(cudaGetLastError());
  OEMS_CUDA(cudaMemcpyAsync(values, a.out, 3 * count * 8, cudaMemcpyDeviceToHost, engine->stream));
  if (snapped)
    OEMS_CUDA(cudaMemcpyAsync(snapped, a.cells_out, 3 * count * 8, cudaMemcpyDeviceToHost, engine->stream));
  OEMS_CUDA(cudaStreamSynchronize(engine->stream));
  return OEMS_OK;
}

oems_status oems_engine_integral(oems_engine* engine, const oems_sample_desc* desc, int32_t kind,
                                 const double start[3], const double stop[3], int32_t normal_dir, double* value) {
  if (!engine || !desc || !start || !stop || !value) return fail(OEMS_ERR_INVALID_ARGUMENT, "NULL argument");
  if (kind != 0 && kind != 1) return fail(OEMS_ERR_CONFIG, "integral kind must be 0 (voltage) or 1 (current)");
  if (normal_dir < 0) return fail(OEMS_ERR_CONFIG, "normal direction must be >= 0");
  uint64_t nl_total = 0;
  OEMS_TRY(check_sample_grid(engine, desc, &nl_total));
  EngineScope guard(engine);
  OEMS_CUDA(engine->d_iface.ensure(nl_total + 1));
  unsigned long long* base = engine->d_iface.p;
  IntegralArgs a{};
  OEMS_TRY(upload_sample_grid(engine, desc, base, &a.s));
  for (int ax = 0; ax < 3; ++ax) {
    a.start[ax] = start[ax];
    a.stop[ax] = stop[ax];
  }
  a.kind = kind;
  a.normal = normal_dir;
  a.out = reinterpret_cast<double*>(base + nl_total);
  launch_storage<KIntegral>(engine, a, 1, 32);
  OEMS_CUDA(cudaGetLastError());
  OEMS_CUDA(cudaMemcpyAsync(value, a.out, 8, cudaMemcpyDeviceToHost, engine->stream));
  OEMS_CUDA(cudaStreamSynchronize(engine->stream));
  return OEMS_OK;
}

oems_status oems_engine_eval_terms(oems_engine* engine, const oems_probe_term* terms, uint64_t nterms, int32_t mode,
                                   double* value) {
  if (!engine || !value || (!terms && nterms)) return fail(OEMS_ERR_INVALID_ARGUMENT, "NULL argument");
  if (mode != OEMS_PROBE_SUM_F32 && mode != OEMS_PROBE_SUM_F64) return fail(OEMS_ERR_CONFIG, "unknown probe mode");
  if (nterms > (uint64_t)INT32_MAX) return fail(OEMS_ERR_CONFIG, "too many terms");
  std::vector<long long> idx(nterms);
  std::vector<double> w(nterms);
  std::vector<int> comp(nterms);
  for (uint64_t t = 0; t < nterms; ++t) {
    const oems_probe_term& q = terms[t];
    if (q.component < 0 || q.component > 5) return fail(OEMS_ERR_CONFIG, "term component must be 0..5");
    if (q.position[0] >= (uint64_t)engine->nx || q.position[1] >= (uint64_t)engine->ny ||
        q.position[2] >= (uint64_t)engine->nz)
      return fail(OEMS_ERR_CONFIG, "term position outside the grid");
    if (!std::isfinite(q.weight)) return fail(OEMS_ERR_CONFIG, "term weight must be finite");
    idx[t] = ((long long)q.position[0] * engine->ny + (long long)q.position[1]) * engine->g.nzp +
             (long long)q.position[2];
    w[t] = q.weight;
    comp[t] = q.component;
  }
  EngineScope guard(engine);
  // words: idx | w | comp (two per word) | result
  const uint64_t w_w = nterms, w_c = 2 * nterms, w_o = w_c + (nterms + 1) / 2;
  OEMS_CUDA(engine->d_iface.ensure(w_o + 1));
  unsigned long long* base = engine->d_iface.p;
  TermArgs a{};
  for (int c = 0; c < 6; ++c) a.f[c] = c < 3 ? engine->E(c) : engine->H(c - 3);
  a.idx = reinterpret_cast<const long long*>(base);
  a.w = reinterpret_cast<const double*>(base + w_w);
  a.comp = reinterpret_cast<const int*>(base + w_c);
  a.n = (long long)nterms;
  a.mode = mode;
  a.h_inv = 1.0f / engine->h_scale;
  a.out = reinterpret_cast<double*>(base + w_o);
  if (nterms) {
    OEMS_CUDA(cudaMemcpyAsync(base, idx.data(), nterms * 8, cudaMemcpyHostToDevice, engine->stream));
    OEMS_CUDA(cudaMemcpyAsync(base + w_w, w.data(), nterms * 8, cudaMemcpyHostToDevice, engine->stream));
    OEMS_CUDA(cudaMemcpyAsync(base + w_c, comp.data(), nterms * 4, cudaMemcpyHostToDevice, engine->stream));
  }
  launch_storage<KTerms>(engine, a, 1, 32);
  OEMS_CUDA(cudaGetLastError());
  OEMS_CUDA(cudaMemcpyAsync(value, a.out, 8, cudaMemcpyDeviceToHost, engine->stream));
  OEMS_CUDA(cudaStreamSynchronize(engine->stream));
  return OEMS_OK;
}

oems_status oems_engine_set_cells(oems_engine* engine, int32_t field, const uint64_t* cells, const float* values,
                                  uint64_t count, int32_t add) {
  if (!engine) return fail(OEMS_ERR_INVALID_ARGUMENT, "NULL engine");
  if (count == 0) return OEMS_OK;
  if (!cells || !values) return fail(OEMS_ERR_INVALID_ARGUMENT, "NULL cells or values");
  if (field != 0 && field != 1) return fail(OEMS_ERR_CONFIG, "field must be 0 (E) or 1 (H)");
  if (count > (uint64_t)1 << 31) return fail(OEMS_ERR_CONFIG, "at most 2^31 writes per call");
  std::vector<long long> idx(count);
  for (uint64_t q = 0; q < count; ++q) {
    const uint64_t* c = cells + 3 * q;
    if (c[0] >= (uint64_t)engine->nx || c[1] >= (uint64_t)engine->ny || c[2] >= (uint64_t)engine->nz)
      return fail(OEMS_ERR_CONFIG, "cell outside the grid");
    idx[q] = ((long long)c[0] * engine->ny + (long long)c[1]) * engine->g.nzp + (long long)c[2];
  }
  EngineScope guard(engine);
  // words: idx | values (3 floats per write)
  const uint64_t w_v = count, words = w_v + (3 * count + 1) / 2;
  OEMS_CUDA(engine->d_iface.ensure(words));
  unsigned long long* base = engine->d_iface.p;
  SetArgs a{};
  for (int c = 0; c < 3; ++c) a.f[c] = field == 0 ? engine->E(c) : engine->H(c);
  a.idx = reinterpret_cast<const long long*>(base);
  a.v = reinterpret_cast<const float*>(base + w_v);
  a.n = (long long)count;
  a.add = add != 0;
  a.scale = field == 1 ? engine->h_scale : 1.0f;
  OEMS_CUDA(cudaMemcpyAsync(base, idx.data(), count * 8, cudaMemcpyHostToDevice, engine->stream));
  OEMS_CUDA(cudaMemcpyAsync(base + w_v, values, 3 * count * 4, cudaMemcpyHostToDevice, engine->stream));
  launch_storage<KSet>(engine, a, 1, 32);
  OEMS_CUDA(cudaGetLastError());
  OEMS_CUDA(cudaStreamSynchronize(engine->stream));
  return OEMS_OK;
}

oems_status oems_engine_set_kernel_profiling(oems_engine* engine, int32_t enable) {
  if (!engine) return fail(OEMS_ERR_INVALID_ARGUMENT, "NULL engine");
  engine->profiling = enable != 0;
  engine->prof_h_s = engine->prof_e_s = 0.0;
  engine->prof_h_n = engine->prof_e_n = 0;
  return OEMS_OK;
}

oems_status oems_engine_launch_info(const oems_engine* engine, int32_t* staged, int32_t* threads, int32_t* ichunk,
                                    int32_t* rows_per_tile, int32_t* stages, int32_t* grid) {
  if (!engine) return fail(OEMS_ERR_INVALID_ARGUMENT, "NULL engine");
  const LaunchShape& s = engine->shape;
  if (staged) *staged = shape_kind(s);
  if (threads) *threads = s.tma ? s.nconsumer + 32 : s.block;
  if (ichunk) *ichunk = s.ichunk;
  if (rows_per_tile) *rows_per_tile = s.tma ? s.tg.TJ : 0;
  if (stages) *stages = s.tma ? s.tg.NS : s.pipe ? s.pipe_ns : s.pf;
  if (grid) *grid = s.grid_h;
  return OEMS_OK;
}

oems_status oems_engine_tune_report(const oems_engine* engine, oems_tune_entry* out, uint64_t capacity,
                                    uint64_t* count) {
  if (!engine || !count) return fail(OEMS_ERR_INVALID_ARGUMENT, "NULL engine or count");
  *count = engine->tune_report.size();
  if (out)
    for (uint64_t i = 0; i < std::min<uint64_t>(capacity, engine->tune_report.size()); ++i)
      out[i] = engine->tune_report[i];
  return OEMS_OK;
}

oems_status oems_engine_kernel_profile(const oems_engine* engine, double* h_seconds, uint64_t* h_launches,
                                       double* e_seconds, uint64_t* e_launches) {
  if (!engine) return fail(OEMS_ERR_INVALID_ARGUMENT, "NULL engine");
  if (h_seconds) *h_seconds = engine->prof_h_s;
  if (h_launches) *h_launches = engine->prof_h_n;
  if (e_seconds) *e_seconds = engine->prof_e_s;
  if (e_launches) *e_launches = engine->prof_e_n;
  return OEMS_OK;
}

const char* oems_status_string(oems_status st) {
  switch (st) {
    case OEMS_OK: return "ok";
    case OEMS_ERR_CONFIG: return "configuration error";
    case OEMS_ERR_IO: return "I/O error";
    case OEMS_ERR_GRID: return "grid error";
    case OEMS_ERR_MATERIAL: return "material error";
    case OEMS_ERR_NUMERICAL: return "numerical error";
    case OEMS_ERR_XML: return "XML error";
    case OEMS_ERR_CUDA: return "CUDA error";
    case OEMS_ERR_NO_DEVICE: return "no CUDA device";
    case OEMS_ERR_TIMEOUT: return "device wait timed out";
    case OEMS_ERR_INVALID_ARGUMENT: return "invalid argument";
  }
  return "unknown status";
}

const char* oems_last_error_message(void) { return g_last_error.c_str(); }

int32_t oems_abi_version(void) { return OEMS_ABI_VERSION; }

oems_status oems_engine_last_batch_stats(const oems_engine* engine, uint64_t* kernel_launches, double* device_seconds) {
  if (!engine) return fail(OEMS_ERR_INVALID_ARGUMENT, "NULL engine");
  if (kernel_launches) *kernel_launches = engine->last_launches;
  if (device_seconds) *device_seconds = engine->last_device_seconds;
  return OEMS_OK;
}

oems_status oems_release_cached_memory(int32_t device) {
  int dev = device;
  if (dev < 0) OEMS_CUDA(cudaGetDevice(&dev));
  cudaMemPool_t pool = nullptr;
  OEMS_CUDA(device_pool(dev, false, &pool));
  if (pool) {
    DeviceGuard guard(dev);
    OEMS_CUDA(cudaDeviceSynchronize());  // frees still pending on engine streams complete first
    OEMS_CUDA(cudaMemPoolTrimTo(pool, 0));
  }
  std::multimap<size_t, void*> bufs;
  {
    PinnedCache& pc = pinned_cache();
    std::lock_guard<std::mutex> lk(pc.mu);
    bufs.swap(pc.free);
  }
  for (auto& kv : bufs) OEMS_CUDA(cudaFreeHost(kv.second));
  return OEMS_OK;
}

}  // extern "C"

// ---------------------------------------------------------------------------
// packs: several engines stepped by shared launches
// ---------------------------------------------------------------------------
// A sweep's instances are small independent grids.  Run one by one, each
// half-step of each grid is a launch too small to fill the GPU, and every
// grid keeps its own graphs and host round trips.  A pack steps a set of
// engines together: per half-step one launch of the plain update kernels over
// the CPML-free boxes of every grid and one of the CPML kernels over all
// their slab cells (work items of all grids in one list, each grid's
// arguments in a device table), then one post-step launch with a CTA per
// grid; energies of all grids in two launches; CUDA graphs per span length.
// Each grid is one part of the launch of its kind (plain or CPML).
// Every grid's cells, sources, probes, energies, DFTs and termination are
// computed by the same code in the same order as oems_engine_run_batch, so
// each engine ends with the bits it would have on its own.
struct oems_pack {
  int device = 0;
  int storage = 0;
  cudaStream_t stream = nullptr;
  cudaEvent_t ev0 = nullptr, ev1 = nullptr;
  std::vector<oems_engine*> en;
  // layout of the active engines: plain parts first, then CPML parts
  std::vector<int> active;
  int n_plain = 0, n_cpml = 0;
  int grid_hp = 1, grid_hc = 1, grid_ep = 1, grid_ec = 1;
  oems::DevBuf<oems::HArgs> h_args;
  oems::DevBuf<oems::EArgs> e_args;
  oems::DevBuf<int> off;  // [n_plain + 1] then [n_cpml + 1]
  oems::DevBuf<oems::PostArgs> post;
  oems::DevBuf<oems::EnergyArgs> energy;
  oems::DevBuf<long long> d_base;
  oems::DevBuf<double> d_energy;  // [active][2]
  double* h_energy = nullptr;     // pinned mirror
  size_t h_energy_cap = 0;
  std::map<int, cudaGraphExec_t> graphs;
  // launch shape of the update kernels: CTA size and x-planes per work item,
  // chosen by pack_tune on the first batch unless set explicitly
  int threads = 256, ichunk = 8;
  // split: a CPML grid enters as two parts, its CPML-free box (plain
  // kernels) and its slab cells (CPML kernels), as the engine's z-split
  bool split = false;
  // fork (split only): each half-step's CPML launch runs on a second stream
  // beside the plain one, whose grid is cut by `cut` CTAs per SM to leave
  // room for it (the bandwidth-bound interiors overlap the latency-bound
  // slabs)
  bool fork = false;
  int cut = 0;
  cudaStream_t side = nullptr;
  cudaEvent_t fork_ev = nullptr, join_ev = nullptr;
  bool tuned = false;
  bool shape_set = false;  // chosen by oems_pack_set_shape: never re-tuned
  double tuned_cells = 0;  // cells of the engines the shape was tuned on
};

namespace oems {

static void pack_drop_graphs(oems_pack* p) {
  for (auto& kv : p->graphs) cudaGraphExecDestroy(kv.second);
  p->graphs.clear();
}


template <typename T>
static oems_status pack_grids(oems_pack* p) {
  int sms = 0, o = 0;
  OEMS_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, p->device));
  const int cut = p->fork ? p->cut : 0;
  OEMS_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&o, (const void*)k_update_h_pack<false, T>, p->threads, 0));
  p->grid_hp = std::max(1, o - cut) * sms;
  OEMS_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&o, (const void*)k_update_h_pack<true, T>, p->threads, 0));
  p->grid_hc = std::max(1, o) * sms;
  OEMS_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&o, (const void*)k_update_e_pack<false, T>, p->threads, 0));
  p->grid_ep = std::max(1, o - cut) * sms;
  OEMS_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&o, (const void*)k_update_e_pack<true, T>, p->threads, 0));
  p->grid_ec = std::max(1, o) * sms;
  return OEMS_OK;
}

// Device tables of the active engines (uploaded on the pack's stream); the
// graphs bake the part counts and the post / energy grid sizes, so they are
// dropped whenever the active set changes.
static oems_status pack_layout(oems_pack* p, const std::vector<int>& active) {
  std::vector<HArgs> hp, hc;
  std::vector<EArgs> ep, ec;
  std::vector<int> op{0}, oc{0};
  std::vector<PostArgs> post;
  std::vector<EnergyArgs> energy;
  for (int i : active) {
    oems_engine* en = p->en[i];
    HArgs a = h_args(en);
    EArgs b = e_args(en);
    auto add = [&](const Geom& g, bool cpml) {
      if (g.work <= 0) return;
      a.g = g;
      b.g = g;
      a.g.pf = b.g.pf = 0;
      if (cpml) {
        hc.push_back(a);
        ec.push_back(b);
        oc.push_back(oc.back() + g.work);
      } else {
        hp.push_back(a);
        ep.push_back(b);
        op.push_back(op.back() + g.work);
      }
    };
    // a CPML grid as one part, or (split) as its CPML-free box for the
    // plain kernels plus its slab cells for the CPML kernels; the tuner
    // times both
    if (p->split && can_zsplit(en)) {
      add(make_interior_geom(en, p->threads, p->ichunk), false);
      add(make_shell_geom(en, p->threads, p->ichunk, true), true);
    } else {
      add(make_geom(en, p->threads, p->ichunk), en->cpml.on);
    }
    PostArgs q{};
    for (int c = 0; c < 3; ++c) {
      q.e[c] = en->E(c);
      q.h[c] = en->H(c);
    }
    q.nexc = en->nexc;
    q.exc_idx = en->d_exc_idx.p;
    q.exc_meta = en->d_exc_meta.p;
    q.exc_off = en->d_exc_off.p;
    q.exc_count = en->d_exc_count.p;
    q.exc_samples = en->d_exc_samples.p;
    q.nprobe = en->nprobe();
    q.probe_off = en->d_probe_off.p;
    q.probe_mode = en->d_probe_mode.p;
    q.term_idx = en->d_term_idx.p;
    q.term_comp = en->d_term_comp.p;
    q.term_w = en->d_term_w.p;
    q.traces = en->d_traces.p;
    q.d_base = p->d_base.p;
    q.h_inv = 1.0f / en->h_scale;
    post.push_back(q);
    EnergyArgs ea{};
    for (int c = 0; c < 6; ++c) ea.arr[c] = en->at((size_t)c);
    ea.n4 = en->ncells_padded / 4;
    ea.partials = en->d_partials.p;
    energy.push_back(ea);
  }
  const size_t na = std::max<size_t>(active.size(), 1);
  OEMS_CUDA(p->h_args.ensure(std::max<size_t>(hp.size() + hc.size(), 1)));
  OEMS_CUDA(p->e_args.ensure(std::max<size_t>(ep.size() + ec.size(), 1)));
  OEMS_CUDA(p->off.ensure(op.size() + oc.size()));
  OEMS_CUDA(p->post.ensure(na));
  OEMS_CUDA(p->energy.ensure(na));
  OEMS_CUDA(p->d_energy.ensure(2 * na));
  std::vector<HArgs> hall(hp);
  hall.insert(hall.end(), hc.begin(), hc.end());
  std::vector<EArgs> eall(ep);
  eall.insert(eall.end(), ec.begin(), ec.end());
  std::vector<int> oall(op);
  oall.insert(oall.end(), oc.begin(), oc.end());
  if (!hall.empty()) {
    OEMS_CUDA(cudaMemcpyAsync(p->h_args.p, hall.data(), hall.size() * sizeof(HArgs), cudaMemcpyHostToDevice, p->stream));
    OEMS_CUDA(cudaMemcpyAsync(p->e_args.p, eall.data(), eall.size() * sizeof(EArgs), cudaMemcpyHostToDevice, p->stream));
  }
  OEMS_CUDA(cudaMemcpyAsync(p->off.p, oall.data(), oall.size() * sizeof(int), cudaMemcpyHostToDevice, p->stream));
  if (!post.empty()) {
    OEMS_CUDA(cudaMemcpyAsync(p->post.p, post.data(), post.size() * sizeof(PostArgs), cudaMemcpyHostToDevice, p->stream));
    OEMS_CUDA(cudaMemcpyAsync(p->energy.p, energy.data(), energy.size() * sizeof(EnergyArgs), cudaMemcpyHostToDevice,
                              p->stream));
  }
  // the host vectors are released on return
  OEMS_CUDA(cudaStreamSynchronize(p->stream));
  p->n_plain = (int)hp.size();
  p->n_cpml = (int)hc.size();
  p->active = active;
  pack_drop_graphs(p);
  return OEMS_OK;
}

template <typename T>
static cudaError_t pack_launch_steps(oems_pack* p, int steps, bool post = true) {
  const int na = (int)p->active.size();
  const PackH hp{p->n_plain, p->off.p, p->h_args.p};
  const PackH hc{p->n_cpml, p->off.p + p->n_plain + 1, p->h_args.p + p->n_plain};
  const PackE ep{p->n_plain, p->off.p, p->e_args.p};
  const PackE ec{p->n_cpml, p->off.p + p->n_plain + 1, p->e_args.p + p->n_plain};
  const bool fork = p->fork && p->side && p->n_plain && p->n_cpml;
  cudaStream_t cs = fork ? p->side : p->stream;
  for (int s = 0; s < steps; ++s) {
    if (fork) {
      cudaEventRecord(p->fork_ev, p->stream);
      cudaStreamWaitEvent(cs, p->fork_ev, 0);
    }
    if (p->n_plain) k_update_h_pack<false, T><<<p->grid_hp, p->threads, 0, p->stream>>>(hp);
    if (p->n_cpml) k_update_h_pack<true, T><<<p->grid_hc, p->threads, 0, cs>>>(hc);
    if (fork) {
      cudaEventRecord(p->join_ev, cs);
      cudaStreamWaitEvent(p->stream, p->join_ev, 0);
      cudaEventRecord(p->fork_ev, p->stream);
      cudaStreamWaitEvent(cs, p->fork_ev, 0);
    }
    if (p->n_plain) k_update_e_pack<false, T><<<p->grid_ep, p->threads, 0, p->stream>>>(ep);
    if (p->n_cpml) k_update_e_pack<true, T><<<p->grid_ec, p->threads, 0, cs>>>(ec);
    if (fork) {
      cudaEventRecord(p->join_ev, cs);
      cudaStreamWaitEvent(p->stream, p->join_ev, 0);
    }
    if (post) k_post_step_pack<T><<<na, 128, 0, p->stream>>>(p->post.p, p->d_base.p, s);
  }
  return cudaGetLastError();
}

static cudaError_t pack_launch_steps_any(oems_pack* p, int steps, bool post = true) {
  if (p->storage == 1) return pack_launch_steps<__half>(p, steps, post);
  if (p->storage == 2) return pack_launch_steps<__nv_bfloat16>(p, steps, post);
  return pack_launch_steps<float>(p, steps, post);
}

static oems_status pack_grids_any(oems_pack* p) {
  if (p->storage == 1) return pack_grids<__half>(p);
  if (p->storage == 2) return pack_grids<__nv_bfloat16>(p);
  return pack_grids<float>(p);
}

// Times the update kernels of the active engines at each candidate shape
// (CTA size x x-planes per work item) on saved copies of their fields and
// CPML psi, restores the state and keeps the fastest.  Sweeps pack small
// grids, most of whose cells lie in the CPML slabs, so the single-grid
// tuner's choice does not carry over.
static oems_status pack_tune(oems_pack* p) {
  p->tuned = true;
  const std::vector<int> act = p->active;
  if (act.empty()) return OEMS_OK;
  p->tuned_cells = 0;
  for (int i : act) p->tuned_cells += (double)p->en[i]->nx * p->en[i]->ny * p->en[i]->nz;
  std::vector<void*> saved(act.size(), nullptr);
  long long cells = 0;
  oems_status st = OEMS_OK;
  for (size_t k = 0; k < act.size() && st == OEMS_OK; ++k) {
    oems_engine* en = p->en[act[k]];
    const size_t fb = en->field_bytes(), pb = en->cpml.on ? en->cpml.psi.n * sizeof(float) : 0;
    cells += (long long)en->nx * en->ny * en->nz;
    if (pool_alloc(&saved[k], fb + pb, p->stream) != cudaSuccess ||
        cudaMemcpyAsync(saved[k], en->fields, fb, cudaMemcpyDeviceToDevice, p->stream) != cudaSuccess ||
        (pb && cudaMemcpyAsync((char*)saved[k] + fb, en->cpml.psi.p, pb, cudaMemcpyDeviceToDevice, p->stream) !=
                   cudaSuccess))
      st = fail(OEMS_ERR_CUDA, "pack tuning: saving the state failed");
  }
  const int reps = (int)std::max<long long>(4, std::min<long long>(20, 400000000LL / std::max(1LL, cells)));
  int best_t = p->threads, best_c = p->ichunk, best_cut = p->cut;
  bool best_split = p->split, best_fork = p->fork;
  float best_ms = 1e30f;
  // modes: 0 whole grids, 1 split, 2 / 3 split with the CPML launch forked
  // beside the plain one (interior grid cut by 0 / 1 CTA per SM)
  for (int mode = 0; mode < (p->side ? 4 : 2); ++mode)
  for (int t : {128, 256, 512})
    for (int c : {2, 4, 8, 16}) {
      if (st != OEMS_OK) break;
      if (mode >= 2 && (t == 512 || c == 16)) continue;
      p->split = mode >= 1;
      p->fork = mode >= 2;
      p->cut = mode == 3 ? 1 : 0;
      p->threads = t;
      p->ichunk = c;
      if ((st = pack_grids_any(p)) != OEMS_OK || (st = pack_layout(p, act)) != OEMS_OK) break;
      cudaError_t e = pack_launch_steps_any(p, 1, false);
      if (e == cudaSuccess) e = cudaEventRecord(p->ev0, p->stream);
      if (e == cudaSuccess) e = pack_launch_steps_any(p, reps, false);
      if (e == cudaSuccess) e = cudaEventRecord(p->ev1, p->stream);
      if (e == cudaSuccess) e = cudaEventSynchronize(p->ev1);
      float ms = 0.f;
      if (e == cudaSuccess) e = cudaEventElapsedTime(&ms, p->ev0, p->ev1);
      if (e != cudaSuccess) {
        st = fail(OEMS_ERR_CUDA, std::string("pack tuning: ") + cudaGetErrorString(e));
        break;
      }
      if (ms < best_ms) {
        best_ms = ms;
        best_t = t;
        best_c = c;
        best_split = p->split;
        best_fork = p->fork;
        best_cut = p->cut;
      }
    }
  for (size_t k = 0; k < act.size(); ++k) {
    if (!saved[k]) continue;
    oems_engine* en = p->en[act[k]];
    const size_t fb = en->field_bytes(), pb = en->cpml.on ? en->cpml.psi.n * sizeof(float) : 0;
    cudaMemcpyAsync(en->fields, saved[k], fb, cudaMemcpyDeviceToDevice, p->stream);
    if (pb) cudaMemcpyAsync(en->cpml.psi.p, (char*)saved[k] + fb, pb, cudaMemcpyDeviceToDevice, p->stream);
    cudaFreeAsync(saved[k], p->stream);
  }
  if (cudaStreamSynchronize(p->stream) != cudaSuccess && st == OEMS_OK)
    st = fail(OEMS_ERR_CUDA, "pack tuning: restoring the state failed");
  if (st != OEMS_OK) return st;
  p->threads = best_t;
  p->ichunk = best_c;
  p->split = best_split;
  p->fork = best_fork;
  p->cut = best_cut;
  OEMS_TRY(pack_grids_any(p));
  return pack_layout(p, act);
}

static oems_status pack_run_span(oems_pack* p, long long base, int steps) {
  k_set_i64<<<1, 1, 0, p->stream>>>(p->d_base.p, base);
  OEMS_CUDA(cudaGetLastError());
  auto it = p->graphs.find(steps);
  if (it == p->graphs.end()) {
    if (p->graphs.size() >= 8) pack_drop_graphs(p);
    cudaGraph_t graph = nullptr;
    OEMS_CUDA(cudaStreamBeginCapture(p->stream, cudaStreamCaptureModeThreadLocal));
    const cudaError_t le = pack_launch_steps_any(p, steps);
    const cudaError_t ce = cudaStreamEndCapture(p->stream, &graph);
    if (le != cudaSuccess || ce != cudaSuccess) {
      if (graph) cudaGraphDestroy(graph);
      return fail(OEMS_ERR_CUDA, std::string("pack graph capture: ") +
                                     cudaGetErrorString(le != cudaSuccess ? le : ce));
    }
    cudaGraphExec_t exec = nullptr;
    const cudaError_t ie = cudaGraphInstantiate(&exec, graph, 0);
    cudaGraphDestroy(graph);
    if (ie != cudaSuccess) return fail(OEMS_ERR_CUDA, std::string("pack graph instantiate: ") + cudaGetErrorString(ie));
    it = p->graphs.emplace(steps, exec).first;
  }
  OEMS_CUDA(cudaGraphLaunch(it->second, p->stream));
  return OEMS_OK;
}

// Energies of the active engines into p->h_energy[2 k], [2 k + 1].
static oems_status pack_energy(oems_pack* p) {
  const int na = (int)p->active.size();
  const dim3 grid(kEnergyBlocks, 6, na);
  if (p->storage == 1)
    k_energy_partial_pack<__half><<<grid, kEnergyThreads, 0, p->stream>>>(p->energy.p);
  else if (p->storage == 2)
    k_energy_partial_pack<__nv_bfloat16><<<grid, kEnergyThreads, 0, p->stream>>>(p->energy.p);
  else
    k_energy_partial_pack<float><<<grid, kEnergyThreads, 0, p->stream>>>(p->energy.p);
  OEMS_CUDA(cudaGetLastError());
  const float hs = p->en[p->active[0]]->h_scale;
  k_energy_final_pack<<<na, 32, 0, p->stream>>>(p->energy.p, p->d_energy.p, 1.0 / ((double)hs * hs));
  OEMS_CUDA(cudaGetLastError());
  if (p->h_energy_cap < (size_t)na) {
    pinned_put(p->h_energy, p->h_energy_cap * 2 * sizeof(double));
    p->h_energy = nullptr;
    p->h_energy_cap = 0;
    void* q = nullptr;
    OEMS_CUDA(pinned_get(&q, (size_t)na * 2 * sizeof(double)));
    p->h_energy = static_cast<double*>(q);
    p->h_energy_cap = na;
  }
  OEMS_CUDA(cudaMemcpyAsync(p->h_energy, p->d_energy.p, (size_t)na * 2 * sizeof(double), cudaMemcpyDeviceToHost,
                            p->stream));
  OEMS_CUDA(cudaStreamSynchronize(p->stream));
  return OEMS_OK;
}

// Per-engine state of one pack batch (the locals of run_batch).
struct PackRun {
  const oems_batch* b = nullptr;
  uint64_t t0 = 0, executed = 0;
  int reason = OEMS_TERMINATION_STEPS_COMPLETED;
  double final_db = 0.0, peak = 0.0;
  bool numerical = false, running = false;
  std::vector<oems_energy_sample> samples;
  size_t peaked = 0;
};

static oems_status pack_run_batch(oems_pack* p, const oems_batch* const* batches, oems_batch_result* results,
                                  oems_status* statuses) {
  const auto t_start = std::chrono::steady_clock::now();
  const size_t n = p->en.size();
  std::vector<PackRun> R(n);
  std::vector<int> part;
  const oems_batch* b0 = nullptr;
  for (size_t i = 0; i < n; ++i) {
    statuses[i] = OEMS_OK;
    if (!batches[i]) continue;
    const oems_batch* b = batches[i];
    if (!b0) b0 = b;
    if (b->num_steps != b0->num_steps || b->sample_interval != b0->sample_interval ||
        b->check_interval != b0->check_interval || b->has_energy_decay_db != b0->has_energy_decay_db ||
        p->en[i]->timestep != p->en[part.empty() ? i : part[0]]->timestep)
      return fail(OEMS_ERR_CONFIG, "the batches of a pack must share step count, intervals and start step");
    part.push_back((int)i);
  }
  if (part.empty()) return OEMS_OK;
  const uint64_t steps = b0->num_steps;
  for (int i : part) {
    oems_engine* en = p->en[i];
    EngineScope guard(en);
    PackRun& r = R[i];
    r.b = batches[i];
    r.t0 = en->timestep;
    r.peak = r.b->initial_peak_energy;
    r.running = true;
    OEMS_TRY(upload_excitations(en, r.b));
    const int np = en->nprobe();
    if (np > 0) OEMS_CUDA(en->d_traces.ensure((size_t)std::max<uint64_t>(steps, 1) * np));
    OEMS_CUDA(cudaStreamSynchronize(en->stream));
  }
  DeviceGuard dg(p->device);
  OEMS_TRY(pack_layout(p, part));
  // tuned on the first batch, and again when the engines in the batch hold
  // under half the cells the shape was tuned on (a sweep's pack shrinks as
  // its instances end)
  double cells = 0;
  for (int i : part) cells += (double)p->en[i]->nx * p->en[i]->ny * p->en[i]->nz;
  if (!p->shape_set && (!p->tuned || cells < 0.5 * p->tuned_cells)) OEMS_TRY(pack_tune(p));
  const uint64_t si = b0->sample_interval, ci = b0->check_interval;
  const bool has_decay = b0->has_energy_decay_db != 0;
  const uint64_t t0 = R[part[0]].t0;
  OEMS_CUDA(cudaEventRecord(p->ev0, p->stream));
  uint64_t s = 0;
  while (s < steps && !p->active.empty()) {
    const uint64_t cur = t0 + s;
    uint64_t ev = UINT64_MAX;
    if (si > 0) ev = std::min(ev, (cur + si - 1) / si * si);
    if (has_decay && ci > 0) {
      uint64_t c = (cur + ci - 1) / ci * ci;
      if (c == 0) c = ci;
      ev = std::min(ev, c);
    }
    uint64_t span = steps - s;
    if (ev != UINT64_MAX && ev - cur + 1 < span) span = ev - cur + 1;
    span = std::min<uint64_t>(span, 1u << 20);
    OEMS_TRY(pack_run_span(p, (long long)s, (int)span));
    s += span;
    const uint64_t last = t0 + s - 1;
    const bool do_sample = si > 0 && last % si == 0;
    const bool do_check = has_decay && ci > 0 && last > 0 && last % ci == 0;
    if (!do_sample && !do_check) continue;
    OEMS_TRY(pack_energy(p));
    std::vector<int> still;
    for (size_t k = 0; k < p->active.size(); ++k) {
      const int i = p->active[k];
      PackRun& r = R[i];
      const double e = p->h_energy[2 * k], h = p->h_energy[2 * k + 1];
      if (do_sample) r.samples.push_back({last, e, h, e + h});
      bool stop = false;
      if (do_check) {
        // run_batch's check: fold the samples since the last check into
        // the peak, then compare this energy with it
        for (; r.peaked < r.samples.size(); ++r.peaked) {
          const double tot = r.samples[r.peaked].total_energy;
          if (!std::isfinite(tot)) r.numerical = true;
          if (r.b->track_peak) r.peak = std::max(r.peak, tot);
        }
        const double tot = e + h;
        if (!std::isfinite(tot)) r.numerical = true;
        if (r.numerical) {
          stop = true;
        } else if (r.peak > 0.0 && tot > 0.0) {
          const double d = 10.0 * std::log10(tot / r.peak);
          if (d < -std::fabs(r.b->energy_decay_db)) {
            r.reason = OEMS_TERMINATION_ENERGY_DECAY;
            r.final_db = d;
            stop = true;
          }
        }
      }
      if (stop) {
        r.executed = s;
        r.running = false;
      } else {
        still.push_back(i);
      }
    }
    if (still.size() != p->active.size()) {
      if (still.empty())
        p->active.clear();
      else
        OEMS_TRY(pack_layout(p, still));
    }
  }
  for (int i : p->active) R[i].executed = s;
  // probe DFTs of each engine's executed steps
  for (int i : part) {
    oems_engine* en = p->en[i];
    if (en->entry_probe.empty() || R[i].executed == 0) continue;
    DftArgs da{};
    da.nentries = (int)en->entry_probe.size();
    da.entry_probe = en->d_entry_probe.p;
    da.entry_freq = en->d_entry_freq.p;
    da.entry_half = en->d_entry_half.p;
    da.acc = en->d_dft_acc.p;
    da.traces = en->d_traces.p;
    da.nprobe = en->nprobe();
    da.steps = (long long)R[i].executed;
    da.t0 = (long long)R[i].t0;
    da.dt = en->dt;
    k_probe_dft<<<(da.nentries + 127) / 128, 128, 0, p->stream>>>(da);
    OEMS_CUDA(cudaGetLastError());
  }
  OEMS_CUDA(cudaEventRecord(p->ev1, p->stream));
  OEMS_CUDA(cudaStreamSynchronize(p->stream));
  float ms = 0.f;
  cudaEventElapsedTime(&ms, p->ev0, p->ev1);
  double cell_steps = 0.0;
  for (int i : part) cell_steps += (double)p->en[i]->nx * p->en[i]->ny * p->en[i]->nz * (double)R[i].executed;
  const double elapsed = std::chrono::duration<double>(std::chrono::steady_clock::now() - t_start).count();
  for (int i : part) {
    oems_engine* en = p->en[i];
    PackRun& r = R[i];
    for (; r.peaked < r.samples.size(); ++r.peaked) {
      const double tot = r.samples[r.peaked].total_energy;
      if (!std::isfinite(tot)) r.numerical = true;
      if (r.b->track_peak) r.peak = std::max(r.peak, tot);
    }
    en->timestep = r.t0 + r.executed;
    en->traces_steps = r.executed;
    const double share = cell_steps > 0.0 ? (double)en->nx * en->ny * en->nz * (double)r.executed / cell_steps : 0.0;
    en->last_device_seconds = ms * 1e-3 * share;
    en->last_launches = 0;
    oems_batch_result& out = results[i];
    out.timesteps_executed = r.executed;
    out.termination_reason = r.reason;
    out.reserved0 = 0;
    out.final_decay_db = r.final_db;
    out.num_energy_samples = r.samples.size();
    out.peak_energy = r.peak;
    for (size_t q = 0; q < r.samples.size() && out.energy_samples && q < out.energy_capacity; ++q)
      out.energy_samples[q] = r.samples[q];
    out.elapsed_seconds = elapsed;
    if (r.numerical) statuses[i] = OEMS_ERR_NUMERICAL;
  }
  return OEMS_OK;
}

}  // namespace oems

extern "C" {

oems_status oems_pack_create(oems_engine* const* engines, uint64_t count, oems_pack** out) {
  if (!out || (!engines && count)) return fail(OEMS_ERR_INVALID_ARGUMENT, "NULL argument");
  if (count == 0) return fail(OEMS_ERR_CONFIG, "a pack needs at least one engine");
  for (uint64_t i = 0; i < count; ++i) {
    const oems_engine* en = engines[i];
    if (!en) return fail(OEMS_ERR_INVALID_ARGUMENT, "NULL engine in the pack");
    if (en->device != engines[0]->device) return fail(OEMS_ERR_CONFIG, "the engines of a pack share one device");
    if (en->storage != engines[0]->storage) return fail(OEMS_ERR_CONFIG, "the engines of a pack share one field storage");
    if (en->id_bytes != 0) return fail(OEMS_ERR_CONFIG, "a pack needs full coefficient arrays");
    if (en->mur.on || en->upml.on || en->tfsf.on || !en->disp.empty() || !en->rlc.q.empty() || !en->fdumps.empty() ||
        !en->boxes.empty())
      return fail(OEMS_ERR_CONFIG, "a pack runs CPML, sources, probes and probe DFTs only");
    for (uint64_t j = 0; j < i; ++j)
      if (engines[j] == en) return fail(OEMS_ERR_CONFIG, "an engine appears twice in the pack");
  }
  auto p = std::make_unique<oems_pack>();
  p->device = engines[0]->device;
  p->storage = engines[0]->storage;
  p->en.assign(engines, engines + count);
  DeviceGuard dg(p->device);
  OEMS_CUDA(cudaStreamCreateWithFlags(&p->stream, cudaStreamNonBlocking));
  OEMS_CUDA(cudaEventCreate(&p->ev0));
  OEMS_CUDA(cudaEventCreate(&p->ev1));
  // the fork's stream and events: a failure leaves the pack unforked
  if (cudaStreamCreateWithFlags(&p->side, cudaStreamNonBlocking) != cudaSuccess ||
      cudaEventCreateWithFlags(&p->fork_ev, cudaEventDisableTiming) != cudaSuccess ||
      cudaEventCreateWithFlags(&p->join_ev, cudaEventDisableTiming) != cudaSuccess) {
    cudaGetLastError();
    if (p->side) cudaStreamDestroy(p->side);
    if (p->fork_ev) cudaEventDestroy(p->fork_ev);
    if (p->join_ev) cudaEventDestroy(p->join_ev);
    p->side = nullptr;
    p->fork_ev = p->join_ev = nullptr;
  }
  OEMS_CUDA(p->d_base.ensure(1));
  const oems_status st = pack_grids_any(p.get());
  if (st != OEMS_OK) {
    oems_pack_destroy(p.release());
    return st;
  }
  *out = p.release();
  return OEMS_OK;
}

void oems_pack_destroy(oems_pack* pack) {
  if (!pack) return;
  DeviceGuard dg(pack->device);
  if (pack->stream) cudaStreamSynchronize(pack->stream);
  oems::pack_drop_graphs(pack);
  pack->h_args.release();
  pack->e_args.release();
  pack->off.release();
  pack->post.release();
  pack->energy.release();
  pack->d_base.release();
  pack->d_energy.release();
  oems::pinned_put(pack->h_energy, pack->h_energy_cap * 2 * sizeof(double));
  if (pack->ev0) cudaEventDestroy(pack->ev0);
  if (pack->ev1) cudaEventDestroy(pack->ev1);
  if (pack->side) {
    cudaStreamSynchronize(pack->side);
    cudaStreamDestroy(pack->side);
  }
  if (pack->fork_ev) cudaEventDestroy(pack->fork_ev);
  if (pack->join_ev) cudaEventDestroy(pack->join_ev);
  if (pack->stream) cudaStreamDestroy(pack->stream);
  delete pack;
}

oems_status oems_pack_set_shape(oems_pack* pack, int32_t threads, int32_t ichunk, int32_t split) {
  if (!pack) return fail(OEMS_ERR_INVALID_ARGUMENT, "NULL pack");
  if (threads < 32 || threads > 512 || threads % 32 || ichunk < 1)
    return fail(OEMS_ERR_CONFIG, "pack shape: threads a multiple of 32 in [32, 512], ichunk >= 1");
  DeviceGuard dg(pack->device);
  if (split < 0 || split > 3 || (split >= 2 && !pack->side))
    return fail(OEMS_ERR_CONFIG, "pack shape: split 0 (whole), 1 (split), 2 / 3 (split, forked, cut 0 / 1)");
  pack->threads = threads;
  pack->ichunk = ichunk;
  pack->split = split != 0;
  pack->fork = split >= 2;
  pack->cut = split == 3 ? 1 : 0;
  pack->tuned = true;
  pack->shape_set = true;
  OEMS_TRY(oems::pack_grids_any(pack));
  if (!pack->active.empty()) OEMS_TRY(oems::pack_layout(pack, pack->active));
  return OEMS_OK;
}

oems_status oems_pack_shape(const oems_pack* pack, int32_t* threads, int32_t* ichunk, int32_t* split) {
  if (!pack) return fail(OEMS_ERR_INVALID_ARGUMENT, "NULL pack");
  if (threads) *threads = pack->threads;
  if (ichunk) *ichunk = pack->ichunk;
  if (split) *split = !pack->split ? 0 : !pack->fork ? 1 : 2 + pack->cut;
  return OEMS_OK;
}

oems_status oems_pack_run_batch(oems_pack* pack, const oems_batch* const* batches, oems_batch_result* results,
                                oems_status* statuses) {
  if (!pack || !batches || !results || !statuses) return fail(OEMS_ERR_INVALID_ARGUMENT, "NULL argument");
  return oems::pack_run_batch(pack, batches, results, statuses);
}

}  // extern "C"
