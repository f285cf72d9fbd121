// predictor_kernels.cu -- kernels of the early-termination network.
//
// The network (a strided temporal convolution stack and an MLP, see
// openems_b200/predictor_net.py) runs forward and backward on these kernels:
// every matrix product goes through the tcgen05 BF16 GEMM (gemm_tc.cuh) with
// f32 accumulation; activations are kept as f32 (B, T, C) row-major with bf16
// copies for the GEMM operands; weights are f32 masters with bf16 copies.
// All entry points take device pointers and a CUDA stream (NULL = default)
// and return an oems_status; nothing here allocates except the error word
// (once per device, on first use).

#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include <stdint.h>

#include <algorithm>
#include <mutex>
#include <string>

#include "../../include/oems.h"
#include "../../include/oems_predictor.h"
#include "gemm_tc.cuh"

namespace oems {
extern thread_local std::string g_last_error;
}

namespace {

oems_status pfail(oems_status st, const std::string& m) {
  oems::g_last_error = m;
  return st;
}

#define PK_CUDA(x)                                                              \
  do {                                                                          \
    cudaError_t e_ = (x);                                                       \
    if (e_ != cudaSuccess) return pfail(OEMS_ERR_CUDA, cudaGetErrorString(e_)); \
  } while (0)

int* g_err[64] = {nullptr};

oems_status err_word(int** out) {
  int dev = 0;
  PK_CUDA(cudaGetDevice(&dev));
  if (dev < 0 || dev >= 64) return pfail(OEMS_ERR_CUDA, "device index out of range");
  if (!g_err[dev]) {
    PK_CUDA(cudaMalloc(&g_err[dev], sizeof(int)));
    PK_CUDA(cudaMemset(g_err[dev], 0, sizeof(int)));
  }
  *out = g_err[dev];
  return OEMS_OK;
}

inline cudaStream_t S(void* s) { return reinterpret_cast<cudaStream_t>(s); }

// cuTensorMapEncodeTiled through the runtime's driver entry point (no link
// against the driver library)
typedef CUresult (*EncodeTiled)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*,
                                const cuuint64_t*, const cuuint32_t*, const cuuint32_t*, CUtensorMapInterleave,
                                CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

oems_status encode_fn(EncodeTiled* out) {
  static EncodeTiled fn = nullptr;
  static std::once_flag once;
  std::call_once(once, [] {
    void* f = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &f, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = reinterpret_cast<EncodeTiled>(f);
  });
  if (!fn) return pfail(OEMS_ERR_CUDA, "cuTensorMapEncodeTiled is not available from the driver");
  *out = fn;
  return OEMS_OK;
}

// Tensor map of a row-major bf16 matrix [rows, k] with row pitch ld
// elements: boxes of 64 K-elements (128 bytes, the swizzle span) x box_rows
// rows, 128-byte swizzle, zero fill outside the matrix.
oems_status bf16_map(EncodeTiled enc, CUtensorMap* m, const void* ptr, int ld, int k, int rows, int box_rows) {
  const cuuint64_t dims[2] = {(cuuint64_t)k, (cuuint64_t)rows};
  const cuuint64_t strides[1] = {(cuuint64_t)ld * 2};
  const cuuint32_t box[2] = {64, (cuuint32_t)box_rows};
  const cuuint32_t estr[2] = {1, 1};
  const CUresult r = enc(m, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 2, const_cast<void*>(ptr), dims, strides, box, estr,
                         CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                         CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  if (r != CUDA_SUCCESS) return pfail(OEMS_ERR_CUDA, "GEMM: cuTensorMapEncodeTiled failed (" + std::to_string((int)r) + ")");
  return OEMS_OK;
}

template <int BN>
cudaError_t launch_gemm(const CUtensorMap& ta, const CUtensorMap& tb, const oems::GemmArgs& p, int grid, void* stream) {
  const size_t smem = oems::GemmCfg<BN>::smem;
  cudaError_t e = cudaFuncSetAttribute(oems::k_gemm_tc<BN>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return e;
  oems::k_gemm_tc<BN><<<grid, 192, smem, S(stream)>>>(ta, tb, p);
  return cudaGetLastError();
}
inline int blocks(long long n, int t) { return (int)((n + t - 1) / t); }
inline int grid_for(long long n, int cap) { return std::max(1, std::min(blocks(n, 256), cap)); }

__global__ void k_f32_to_bf16(const float* x, __nv_bfloat16* y, long long n) {
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
    y[i] = __float2bfloat16_rn(x[i]);
}

// y[c * ldy + r] = x[r * ldx + c] for r < R, c < C (bf16), through a 32 x 32 tile
__global__ void k_transpose_bf16(const __nv_bfloat16* x, int ldx, __nv_bfloat16* y, int ldy, int R, int C) {
  __shared__ __nv_bfloat16 t[32][33];
  const int r0 = blockIdx.y * 32, c0 = blockIdx.x * 32;
  for (int i = threadIdx.y; i < 32; i += blockDim.y) {
    const int r = r0 + i, c = c0 + threadIdx.x;
    if (r < R && c < C) t[i][threadIdx.x] = x[(size_t)r * ldx + c];
  }
  __syncthreads();
  for (int i = threadIdx.y; i < 32; i += blockDim.y) {
    const int c = c0 + i, r = r0 + threadIdx.x;
    if (r < R && c < C) y[(size_t)c * ldy + r] = t[threadIdx.x][i];
  }
}

// cols[(b, t), k * C + c] = x[b, t * s + k, c]  (bf16, row pitch ldc)
__global__ void k_im2col(const float* x, __nv_bfloat16* cols, int B, int T, int C, int ks, int s, int Tout,
                         int ldc) {
  const long long n = (long long)B * Tout * ks * C;
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    const int c = (int)(i % C);
    long long r = i / C;
    const int k = (int)(r % ks);
    r /= ks;
    const int t = (int)(r % Tout);
    const int b = (int)(r / Tout);
    cols[((long long)b * Tout + t) * ldc + (long long)k * C + c] =
        __float2bfloat16_rn(x[((long long)b * T + (long long)t * s + k) * C + c]);
  }
}

// dx[b, tau, c] = sum over (t, k) with t * s + k = tau of dcols[(b, t), k * C + c]
__global__ void k_col2im(const float* dcols, int ldc, float* dx, int B, int T, int C, int ks, int s, int Tout) {
  const long long n = (long long)B * T * C;
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    const int c = (int)(i % C);
    const long long r = i / C;
    const int tau = (int)(r % T);
    const int b = (int)(r / T);
    float acc = 0.f;
    for (int k = 0; k < ks; ++k) {
      const int u = tau - k;
      if (u < 0 || u % s) continue;
      const int t = u / s;
      if (t >= Tout) continue;
      acc += dcols[((long long)b * Tout + t) * ldc + (long long)k * C + c];
    }
    dx[i] = acc;
  }
}

// Causal dilated im2col: output length T; row (b, t) holds, at k C + c,
// x[b, t - (ks - 1 - k) dil, c] (0 before the start), so tap ks - 1 is the
// current step and the others reach back by multiples of the dilation.
__global__ void k_im2col_causal(const float* x, __nv_bfloat16* cols, int B, int T, int C, int ks, int dil, int ldc) {
  const long long n = (long long)B * T * ks * C;
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    const int c = (int)(i % C);
    long long r = i / C;
    const int k = (int)(r % ks);
    r /= ks;
    const int t = (int)(r % T);
    const int b = (int)(r / T);
    const int u = t - (ks - 1 - k) * dil;
    const float v = u >= 0 ? x[((long long)b * T + u) * C + c] : 0.0f;
    cols[((long long)b * T + t) * ldc + (long long)k * C + c] = __float2bfloat16_rn(v);
  }
}

// Adjoint: dx[b, tau, c] = sum over k of dcols[(b, tau + (ks - 1 - k) dil), k C + c]
// (terms past the end dropped), summed in k order.
__global__ void k_col2im_causal(const float* dcols, int ldc, float* dx, int B, int T, int C, int ks, int dil) {
  const long long n = (long long)B * T * C;
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    const int c = (int)(i % C);
    const long long r = i / C;
    const int tau = (int)(r % T);
    const int b = (int)(r / T);
    float acc = 0.f;
    for (int k = 0; k < ks; ++k) {
      const int t = tau + (ks - 1 - k) * dil;
      if (t >= T) continue;
      acc += dcols[((long long)b * T + t) * ldc + (long long)k * C + c];
    }
    dx[i] = acc;
  }
}

// y = max(x, 0) in place, with a bf16 copy of y (pitch ldb, rows of width w)
__global__ void k_relu(float* x, __nv_bfloat16* xb, long long rows, int w, int ldb) {
  const long long n = rows * w;
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    const float v = fmaxf(x[i], 0.f);
    x[i] = v;
    if (xb) xb[(i / w) * ldb + i % w] = __float2bfloat16_rn(v);
  }
}

// dy *= (y > 0)
__global__ void k_relu_bwd(float* dy, const float* y, long long n) {
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
    if (!(y[i] > 0.f)) dy[i] = 0.f;
}

// db[c] = sum_r dy[r, c]: one block per column, fixed order
__global__ void k_colsum(const float* dy, long long rows, int w, float* db) {
  const int c = blockIdx.x;
  __shared__ float part[256];
  float acc = 0.f;
  for (long long r = threadIdx.x; r < rows; r += blockDim.x) acc += dy[r * w + c];
  part[threadIdx.x] = acc;
  __syncthreads();
  for (int st = blockDim.x / 2; st > 0; st >>= 1) {
    if (threadIdx.x < st) part[threadIdx.x] += part[threadIdx.x + st];
    __syncthreads();
  }
  if (threadIdx.x == 0) db[c] = part[0];
}

// g = 2 (p - t) w_row / n ; loss partials per block (sum of w_row (p - t)^2)
__global__ void k_mse(const float* p, const float* t, const float* wrow, float* g, long long rows, int w,
                      double* partial) {
  __shared__ double part[256];
  const long long n = rows * w;
  double acc = 0.0;
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    const float d = p[i] - t[i];
    const float wr = wrow ? wrow[i / w] : 1.f;
    g[i] = 2.f * d * wr / (float)n;
    acc += (double)wr * d * d;
  }
  part[threadIdx.x] = acc;
  __syncthreads();
  for (int st = blockDim.x / 2; st > 0; st >>= 1) {
    if (threadIdx.x < st) part[threadIdx.x] += part[threadIdx.x + st];
    __syncthreads();
  }
  if (threadIdx.x == 0) partial[blockIdx.x] = part[0];
}

// Adam (Kingma & Ba) with decoupled weight decay, f32 masters, bf16 copy
__global__ void k_adam(float* w, __nv_bfloat16* wb, const float* g, float* m, float* v, long long n, float lr,
                       float b1, float b2, float eps, float wd, float c1, float c2) {
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    const float gi = g[i];
    const float mi = b1 * m[i] + (1.f - b1) * gi;
    const float vi = b2 * v[i] + (1.f - b2) * gi * gi;
    m[i] = mi;
    v[i] = vi;
    const float wi = w[i] * (1.f - lr * wd) - lr * (mi / c1) / (sqrtf(vi / c2) + eps);
    w[i] = wi;
    if (wb) wb[i] = __float2bfloat16_rn(wi);
  }
}

}  // namespace

extern "C" {

oems_status oems_tc_gemm_bf16(const void* a, int lda, const void* b, int ldb, float* c, int ldc, int M, int N, int K,
                              float beta, const float* bias, void* stream) {
  if (!a || !b || !c) return pfail(OEMS_ERR_INVALID_ARGUMENT, "NULL operand");
  if (M <= 0 || N <= 0 || K <= 0) return pfail(OEMS_ERR_CONFIG, "GEMM sizes must be positive");
  if (K % 8 || lda % 8 || ldb % 8 || lda < K || ldb < K || ldc < N)
    return pfail(OEMS_ERR_CONFIG, "GEMM: K and the A / B row pitches must be multiples of 8 elements");
  if ((reinterpret_cast<uintptr_t>(a) | reinterpret_cast<uintptr_t>(b)) & 15)
    return pfail(OEMS_ERR_CONFIG, "GEMM: A and B must be 16-byte aligned");
  int* err = nullptr;
  oems_status st = err_word(&err);
  if (st != OEMS_OK) return st;
  oems::GemmArgs p{};
  p.c = c;
  p.bias = bias;
  p.ldc = ldc;
  p.M = M;
  p.N = N;
  p.K = K;
  p.beta = beta;
  p.err = err;
  EncodeTiled enc = nullptr;
  st = encode_fn(&enc);
  if (st != OEMS_OK) return st;
  int dev = 0, sms = 0;
  PK_CUDA(cudaGetDevice(&dev));
  PK_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
  // tile width: one CTA per SM (the stage ring takes ~192 KB of shared
  // memory), so the estimate is waves x a tile's cost, taken as its MMA
  // columns plus a fixed 64 for loading A and draining the accumulator
  const long long tm = (M + 127) / 128;
  int BN = 64;
  long long best = -1;
  for (int cand : {256, 128, 64}) {
    const long long waves = (tm * ((N + cand - 1) / cand) + sms - 1) / sms;
    const long long cost = waves * (cand + 64);
    if (best < 0 || cost < best) best = cost, BN = cand;
  }
  CUtensorMap ta, tb;
  st = bf16_map(enc, &ta, a, lda, K, M, 128);
  if (st == OEMS_OK) st = bf16_map(enc, &tb, b, ldb, K, N, BN);
  if (st != OEMS_OK) return st;
  const long long tiles = tm * ((N + BN - 1) / BN);
  const int grid = (int)std::min<long long>(tiles, sms);
  if (BN == 256) {
    PK_CUDA(launch_gemm<256>(ta, tb, p, grid, stream));
  } else if (BN == 128) {
    PK_CUDA(launch_gemm<128>(ta, tb, p, grid, stream));
  } else {
    PK_CUDA(launch_gemm<64>(ta, tb, p, grid, stream));
  }
  PK_CUDA(cudaGetLastError());
  return OEMS_OK;
}

oems_status oems_tc_wait_probe(void* stream) {
  int* err = nullptr;
  oems_status st = err_word(&err);
  if (st != OEMS_OK) return st;
  oems::k_tc_wait_probe<<<1, 32, 0, S(stream)>>>(err);
  PK_CUDA(cudaGetLastError());
  return OEMS_OK;
}

oems_status oems_tc_check(void* stream) {
  int* err = nullptr;
  oems_status st = err_word(&err);
  if (st != OEMS_OK) return st;
  int h = 0;
  PK_CUDA(cudaMemcpyAsync(&h, err, sizeof(int), cudaMemcpyDeviceToHost, S(stream)));
  PK_CUDA(cudaStreamSynchronize(S(stream)));
  if (h) {
    PK_CUDA(cudaMemset(err, 0, sizeof(int)));
    return pfail(OEMS_ERR_TIMEOUT, "a tensor-core GEMM gave up waiting for its MMAs");
  }
  return OEMS_OK;
}

oems_status oems_pk_f32_to_bf16(const float* x, void* y, int64_t n, void* stream) {
  k_f32_to_bf16<<<grid_for(n, 4096), 256, 0, S(stream)>>>(x, static_cast<__nv_bfloat16*>(y), n);
  PK_CUDA(cudaGetLastError());
  return OEMS_OK;
}

oems_status oems_pk_transpose_bf16(const void* x, int ldx, void* y, int ldy, int R, int C, void* stream) {
  const dim3 grid((C + 31) / 32, (R + 31) / 32);
  k_transpose_bf16<<<grid, dim3(32, 8), 0, S(stream)>>>(static_cast<const __nv_bfloat16*>(x), ldx,
                                                       static_cast<__nv_bfloat16*>(y), ldy, R, C);
  PK_CUDA(cudaGetLastError());
  return OEMS_OK;
}

oems_status oems_pk_im2col(const float* x, void* cols, int B, int T, int C, int ks, int s, int ldc, void* stream) {
  if (T < ks) return pfail(OEMS_ERR_CONFIG, "im2col: sequence shorter than the kernel");
  const int Tout = (T - ks) / s + 1;
  const long long n = (long long)B * Tout * ks * C;
  k_im2col<<<grid_for(n, 8192), 256, 0, S(stream)>>>(x, static_cast<__nv_bfloat16*>(cols), B, T, C, ks, s, Tout,
                                                     ldc);
  PK_CUDA(cudaGetLastError());
  return OEMS_OK;
}

oems_status oems_pk_col2im(const float* dcols, int ldc, float* dx, int B, int T, int C, int ks, int s, void* stream) {
  const int Tout = (T - ks) / s + 1;
  const long long n = (long long)B * T * C;
  k_col2im<<<grid_for(n, 8192), 256, 0, S(stream)>>>(dcols, ldc, dx, B, T, C, ks, s, Tout);
  PK_CUDA(cudaGetLastError());
  return OEMS_OK;
}

oems_status oems_pk_im2col_causal(const float* x, void* cols, int B, int T, int C, int ks, int dil, int ldc,
                                  void* stream) {
  if (ks < 1 || dil < 1 || ldc < ks * C) return pfail(OEMS_ERR_CONFIG, "im2col_causal: bad kernel, dilation or pitch");
  const long long n = (long long)B * T * ks * C;
  k_im2col_causal<<<grid_for(n, 8192), 256, 0, S(stream)>>>(x, static_cast<__nv_bfloat16*>(cols), B, T, C, ks, dil,
                                                            ldc);
  PK_CUDA(cudaGetLastError());
  return OEMS_OK;
}

oems_status oems_pk_col2im_causal(const float* dcols, int ldc, float* dx, int B, int T, int C, int ks, int dil,
                                  void* stream) {
  if (ks < 1 || dil < 1 || ldc < ks * C) return pfail(OEMS_ERR_CONFIG, "col2im_causal: bad kernel, dilation or pitch");
  const long long n = (long long)B * T * C;
  k_col2im_causal<<<grid_for(n, 8192), 256, 0, S(stream)>>>(dcols, ldc, dx, B, T, C, ks, dil);
  PK_CUDA(cudaGetLastError());
  return OEMS_OK;
}

oems_status oems_pk_relu(float* x, void* xb, int64_t rows, int w, int ldb, void* stream) {
  const long long n = rows * w;
  k_relu<<<grid_for(n, 8192), 256, 0, S(stream)>>>(x, static_cast<__nv_bfloat16*>(xb), rows, w, ldb);
  PK_CUDA(cudaGetLastError());
  return OEMS_OK;
}

oems_status oems_pk_relu_bwd(float* dy, const float* y, int64_t n, void* stream) {
  k_relu_bwd<<<grid_for(n, 8192), 256, 0, S(stream)>>>(dy, y, n);
  PK_CUDA(cudaGetLastError());
  return OEMS_OK;
}

oems_status oems_pk_colsum(const float* dy, int64_t rows, int w, float* db, void* stream) {
  k_colsum<<<w, 256, 0, S(stream)>>>(dy, rows, w, db);
  PK_CUDA(cudaGetLastError());
  return OEMS_OK;
}

oems_status oems_pk_mse(const float* p, const float* t, const float* wrow, float* g, int64_t rows, int w,
                        double* partial, int nblocks, void* stream) {
  if (nblocks < 1 || nblocks > 4096) return pfail(OEMS_ERR_CONFIG, "mse: 1..4096 blocks");
  k_mse<<<nblocks, 256, 0, S(stream)>>>(p, t, wrow, g, rows, w, partial);
  PK_CUDA(cudaGetLastError());
  return OEMS_OK;
}

oems_status oems_pk_adam(float* w, void* wb, const float* g, float* m, float* v, int64_t n, float lr, float b1,
                         float b2, float eps, float wd, int step, void* stream) {
  const float c1 = 1.f - powf(b1, (float)step), c2 = 1.f - powf(b2, (float)step);
  k_adam<<<grid_for(n, 4096), 256, 0, S(stream)>>>(w, static_cast<__nv_bfloat16*>(wb), g, m, v, n, lr, b1, b2, eps,
                                                   wd, c1, c2);
  PK_CUDA(cudaGetLastError());
  return OEMS_OK;
}

}  // extern "C"
