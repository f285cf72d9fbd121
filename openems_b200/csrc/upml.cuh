// upml.cuh -- the reference's uniaxial PML (src/extensions/pml.rs:194-855).
//
// Flux form around each field update, per region cell and component n:
//   pre  (pml.rs:505-549, 586-620): f = vv V - vvfo flux; V <- flux; flux <- f
//   (the main update then advances V, which now holds the flux)
//   post (pml.rs:554-581, 625-655): f = flux; flux <- V; V <- f + vvfn V
// with (vv, vvfo, vvfn) for E and (ii, iifo, iifn) for H.  The regions do not
// overlap (pml.rs:222-296), so every cell is handled by one thread.  Products
// and sums are rounded separately in the reference's order.  The reference's
// coefficients make the scheme grow without bound (its cross-engine tests
// are disabled for this reason); the update is reproduced as it is.
#pragma once

#include <cuda_runtime.h>

namespace oems {

struct UpmlArgs {
  int nreg;
  long long start[6][3];
  long long size[6][3];
  long long off[7];    // prefix sums of region cell counts
  long long total;     // region cells
  long long ny, nzp;   // padded field layout
  const float* coef;   // [3 coefficients][3 components][total]: v(i)v, v(i)vfo, v(i)vfn
  float* flux;         // [3 components][total]
  float* f[3];         // E or H components
};

__device__ __forceinline__ void upml_cell(const UpmlArgs& a, long long m, long long* q) {
  int r = 0;
  while (m >= a.off[r + 1]) ++r;
  const long long l = m - a.off[r];
  const long long sz1 = a.size[r][1], sz2 = a.size[r][2];
  const long long lk = l % sz2, t = l / sz2;
  const long long lj = t % sz1, li = t / sz1;
  *q = ((a.start[r][0] + li) * a.ny + (a.start[r][1] + lj)) * a.nzp + a.start[r][2] + lk;
}

__global__ void k_upml_pre(const UpmlArgs a) {
  const long long m = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (m >= a.total) return;
  long long q;
  upml_cell(a, m, &q);
#pragma unroll
  for (int n = 0; n < 3; ++n) {
    const float v_old = a.f[n][q];
    float* fl = a.flux + (long long)n * a.total + m;
    const float flux_old = *fl;
    const float vv = a.coef[(0 * 3 + n) * a.total + m];
    const float vvfo = a.coef[(1 * 3 + n) * a.total + m];
    const float f_help = __fsub_rn(__fmul_rn(vv, v_old), __fmul_rn(vvfo, flux_old));
    a.f[n][q] = flux_old;
    *fl = f_help;
  }
}

__global__ void k_upml_post(const UpmlArgs a) {
  const long long m = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (m >= a.total) return;
  long long q;
  upml_cell(a, m, &q);
#pragma unroll
  for (int n = 0; n < 3; ++n) {
    float* fl = a.flux + (long long)n * a.total + m;
    const float f_help = *fl;
    const float flux_new = a.f[n][q];
    *fl = flux_new;
    const float vvfn = a.coef[(2 * 3 + n) * a.total + m];
    a.f[n][q] = __fadd_rn(f_help, __fmul_rn(vvfn, flux_new));
  }
}

}  // namespace oems
