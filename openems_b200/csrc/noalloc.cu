// noalloc.cu -- field energy without any device allocation.
//
// Some callers cannot let this library call cudaMalloc: a co-simulation or
// plugin host that owns every byte of device memory and hands the solver
// fixed buffers, or a tight control loop that must not pay the implicit
// device-wide synchronisation an allocation can cause.  For them,
// oems_field_energy_noalloc computes the same unweighted energies as
// oems_engine_energy (sum of E^2 and sum of H^2 in f64) from six caller-owned
// device arrays, keeping its per-block partial sums in a fixed, file-scope
// device array instead of an allocation.
//
// The scratch array is shared by every call on a device and keeps the last
// call's contents; its completion counter is cleared before every launch.
// Calls that overlap on the GPU (concurrent streams) race on it.  Every call
// looks up the array's device address with the device current (a host-side
// lookup, no allocation): an address kept from an earlier call would dangle
// after cudaDeviceReset or a re-created context, which reload the module.
// The first call on each device loads the module; make it before any stream
// capture.
#include <cuda_runtime.h>

#include <mutex>
#include <string>

#include "../../include/oems.h"

namespace oems {
extern thread_local std::string g_last_error;
}

namespace {

constexpr int kNaThreads = 256;
constexpr int kNaPerThread = 16;    // float4 loads per thread and array
constexpr int kNaMaxBlocks = 4096;  // blocks per array the scratch can hold
constexpr unsigned long long kNaMaxCount =
    (unsigned long long)kNaMaxBlocks * kNaThreads * kNaPerThread * 4;  // 67,108,864 floats per array
constexpr int kNaMaxDevices = 64;

// [6][kNaMaxBlocks] partial sums, then one slot whose first word is the
// completion counter: 196,616 bytes per device.
static __device__ __align__(256) double g_energy_scratch[6 * kNaMaxBlocks + 1];

struct NaArgs {
  const float* arr[6];
  unsigned long long count;  // floats per array
  int blocks;                // blocks per array
  double* out;               // out[0] = sum E^2, out[1] = sum H^2
};

// Each block sums x^2 over a contiguous slice of one array (blockIdx.y); the
// last block to finish adds all partials in a fixed order.
__global__ void __launch_bounds__(kNaThreads) k_energy_noalloc(const NaArgs a, double* scratch) {
  const float* p = a.arr[blockIdx.y];
  const unsigned long long n4 = a.count / 4;
  const unsigned long long base = (unsigned long long)blockIdx.x * kNaThreads * kNaPerThread;
  double s = 0.0;
#pragma unroll 4
  for (int r = 0; r < kNaPerThread; ++r) {
    const unsigned long long q = base + (unsigned long long)r * kNaThreads + threadIdx.x;
    if (q < n4) {
      const float4 v = __ldcs(reinterpret_cast<const float4*>(p) + q);
      s += (double)v.x * (double)v.x + (double)v.y * (double)v.y + (double)v.z * (double)v.z +
           (double)v.w * (double)v.w;
    }
  }
  // the tail (count not a multiple of 4) belongs to the last block
  if (blockIdx.x == (unsigned)(a.blocks - 1)) {
    for (unsigned long long q = n4 * 4 + threadIdx.x; q < a.count; q += kNaThreads) {
      const double v = (double)p[q];
      s += v * v;
    }
  }
  __shared__ double red[kNaThreads];
  red[threadIdx.x] = s;
  __syncthreads();
  for (int w = kNaThreads / 2; w > 0; w >>= 1) {
    if ((int)threadIdx.x < w) red[threadIdx.x] += red[threadIdx.x + w];
    __syncthreads();
  }
  __shared__ bool last;
  if (threadIdx.x == 0) {
    scratch[blockIdx.y * kNaMaxBlocks + blockIdx.x] = red[0];
    __threadfence();
    unsigned int* counter = reinterpret_cast<unsigned int*>(scratch + 6 * kNaMaxBlocks);
    const unsigned int ticket = atomicAdd(counter, 1u);
    last = ticket == (unsigned int)(6 * a.blocks - 1);
  }
  __syncthreads();
  if (!last) return;
  // final sum by the whole last block, in a fixed order for a fixed count
  __threadfence();
  __shared__ double comp[6];
  for (int c = 0; c < 6; ++c) {
    double t = 0.0;
    for (int b = threadIdx.x; b < a.blocks; b += kNaThreads)
      t += ((volatile double*)scratch)[c * kNaMaxBlocks + b];
    red[threadIdx.x] = t;
    __syncthreads();
    for (int w = kNaThreads / 2; w > 0; w >>= 1) {
      if ((int)threadIdx.x < w) red[threadIdx.x] += red[threadIdx.x + w];
      __syncthreads();
    }
    if (threadIdx.x == 0) comp[c] = red[0];
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    a.out[0] = comp[0] + comp[1] + comp[2];
    a.out[1] = comp[3] + comp[4] + comp[5];
  }
}

std::mutex g_na_mutex;

oems_status na_fail(oems_status st, const char* msg) {
  oems::g_last_error = msg;
  return st;
}

// Device address of the scratch array in the current device's context,
// looked up on every call (see the file comment: a cached one can go stale).
oems_status na_scratch(double** out) {
  std::lock_guard<std::mutex> lock(g_na_mutex);
  double* ptr = nullptr;
  const cudaError_t e = cudaGetSymbolAddress((void**)&ptr, g_energy_scratch);
  if (e != cudaSuccess || !ptr) {
    oems::g_last_error = std::string("cudaGetSymbolAddress: ") + cudaGetErrorString(e);
    return OEMS_ERR_CUDA;
  }
  *out = ptr;
  return OEMS_OK;
}

}  // namespace

extern "C" oems_status oems_field_energy_noalloc(const float* const fields[6], uint64_t count,
                                                 double* energies, void* stream) {
  oems::g_last_error.clear();
  if (!fields || !energies) return na_fail(OEMS_ERR_INVALID_ARGUMENT, "NULL argument");
  if (count == 0) return na_fail(OEMS_ERR_INVALID_ARGUMENT, "count must be positive");
  if (count > kNaMaxCount)
    return na_fail(OEMS_ERR_INVALID_ARGUMENT,
                   "count exceeds the no-allocation maximum of 67108864 floats per array");
  for (int c = 0; c < 6; ++c) {
    if (!fields[c]) return na_fail(OEMS_ERR_INVALID_ARGUMENT, "NULL field array");
    if (reinterpret_cast<uintptr_t>(fields[c]) % 16 != 0)
      return na_fail(OEMS_ERR_INVALID_ARGUMENT, "field arrays must be 16-byte aligned");
  }
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) {
    cudaGetLastError();
    return na_fail(OEMS_ERR_NO_DEVICE, cudaGetErrorString(e));
  }
  if (dev < 0 || dev >= kNaMaxDevices) return na_fail(OEMS_ERR_NO_DEVICE, "device ordinal out of range");
  double* scratch = nullptr;
  const oems_status st = na_scratch(&scratch);
  if (st != OEMS_OK) return st;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  // the completion counter must start at zero; the partials are overwritten
  e = cudaMemsetAsync(scratch + 6 * kNaMaxBlocks, 0, sizeof(double), s);
  if (e != cudaSuccess) return na_fail(OEMS_ERR_CUDA, cudaGetErrorString(e));
  NaArgs a{};
  for (int c = 0; c < 6; ++c) a.arr[c] = fields[c];
  a.count = count;
  const unsigned long long per_block = (unsigned long long)kNaThreads * kNaPerThread * 4;
  a.blocks = (int)((count + per_block - 1) / per_block);
  a.out = energies;
  k_energy_noalloc<<<dim3(a.blocks, 6), kNaThreads, 0, s>>>(a, scratch);
  e = cudaGetLastError();
  if (e != cudaSuccess) return na_fail(OEMS_ERR_CUDA, cudaGetErrorString(e));
  return OEMS_OK;
}
