/*
 * oems_predictor.h -- kernels of the learned early-termination network
 * (liboems_b200.so; no counterpart in the reference).
 *
 * All pointers are device pointers; stream NULL = the default stream.  bf16
 * buffers hold raw 16-bit values.  The GEMM runs on the tcgen05 tensor cores
 * with f32 accumulation.
 */
#ifndef OEMS_PREDICTOR_H
#define OEMS_PREDICTOR_H

#include <stdint.h>

#include "oems.h"

#ifdef __cplusplus
extern "C" {
#endif

/* C[M, N] = A[M, K] B[N, K]^T (+ beta C) (+ bias[N]): A, B bf16 K-major with
 * row pitches lda, ldb (multiples of 8 elements, 16-byte aligned bases), K a
 * multiple of 8; C f32 with row pitch ldc; bias may be NULL. */
OEMS_API oems_status oems_tc_gemm_bf16(const void* a, int lda, const void* b, int ldb, float* c, int ldc, int M,
                                       int N, int K, float beta, const float* bias, void* stream);
/* Synchronises the stream and reports (then clears) a GEMM whose bounded
 * wait for its MMAs gave up: OEMS_ERR_TIMEOUT. */
OEMS_API oems_status oems_tc_check(void* stream);
/* Launches one CTA whose bounded mbarrier wait (the GEMM's own, about one
 * second) runs out on a barrier nothing arrives at; the next oems_tc_check
 * on the stream reports OEMS_ERR_TIMEOUT.  For tests of the timeout path. */
OEMS_API oems_status oems_tc_wait_probe(void* stream);
OEMS_API oems_status oems_pk_f32_to_bf16(const float* x, void* y, int64_t n, void* stream);
/* y[c * ldy + r] = x[r * ldx + c], r < R, c < C (bf16). */
OEMS_API oems_status oems_pk_transpose_bf16(const void* x, int ldx, void* y, int ldy, int R, int C, void* stream);
/* Strided valid 1-D convolution as a GEMM, activations (B, T, C) f32:
 * cols[(b, t), k C + c] = x[b, t s + k, c] (bf16, row pitch ldc), t < (T - ks) / s + 1. */
OEMS_API oems_status oems_pk_im2col(const float* x, void* cols, int B, int T, int C, int ks, int s, int ldc,
                                    void* stream);
/* Adjoint of im2col: dx[b, tau, c] = sum of the dcols entries that read x[b, tau, c]. */
OEMS_API oems_status oems_pk_col2im(const float* dcols, int ldc, float* dx, int B, int T, int C, int ks, int s,
                                    void* stream);
/* Causal dilated conv1d as im2col over (B, T, C) f32: cols (B T rows, pitch
 * ldc >= ks C, bf16) row (b, t) holds x[b, t - (ks - 1 - k) dil, c] at
 * column k C + c, 0 before the start; the output keeps the length T. */
OEMS_API oems_status oems_pk_im2col_causal(const float* x, void* cols, int B, int T, int C, int ks, int dil,
                                           int ldc, void* stream);
/* Adjoint of the causal im2col: dx[b, tau, c] sums the dcols entries that read x[b, tau, c]. */
OEMS_API oems_status oems_pk_col2im_causal(const float* dcols, int ldc, float* dx, int B, int T, int C, int ks,
                                           int dil, void* stream);
/* x = max(x, 0) for rows x w values; xb (may be NULL) receives a bf16 copy with row pitch ldb. */
OEMS_API oems_status oems_pk_relu(float* x, void* xb, int64_t rows, int w, int ldb, void* stream);
OEMS_API oems_status oems_pk_relu_bwd(float* dy, const float* y, int64_t n, void* stream);
/* db[c] = sum over rows of dy[r, c] (fixed order). */
OEMS_API oems_status oems_pk_colsum(const float* dy, int64_t rows, int w, float* db, void* stream);
/* g = 2 (p - t) wrow[r] / (rows w); partial[block] = sum wrow (p - t)^2 over the block's share. */
OEMS_API oems_status oems_pk_mse(const float* p, const float* t, const float* wrow, float* g, int64_t rows, int w,
                                 double* partial, int nblocks, void* stream);
/* Adam with decoupled weight decay; step counts from 1; wb (may be NULL)
 * receives the bf16 copy of the updated weights. */
OEMS_API oems_status oems_pk_adam(float* w, void* wb, const float* g, float* m, float* v, int64_t n, float lr,
                                  float b1, float b2, float eps, float wd, int step, void* stream);

#ifdef __cplusplus
}
#endif
#endif /* OEMS_PREDICTOR_H */
