// mur.cuh -- Mur absorbing boundary kernels (face cells only).
//
// First order restates src/extensions/mur_abc.rs:88-324:
//   pre  (before the E update): v = E_shift - c * E_bnd
//   post (after the E update):  v = v + c * E_shift
//   apply:                      E_bnd = v, faces in order (a later face wins
//                               on a shared edge)
// Second order (Mur 1981) on the interior of a face, first order on its two
// outermost rows and columns; at a min face the boundary sits on line 1
// because plane 0 is never updated by the E update.  Every product and sum is
// rounded separately, in the same order as the oracle.
#pragma once

#include <cuda_runtime.h>

namespace oems {

struct MurFaceDev {
  int ny, nyp, nypp;  // normal axis and the two tangential axes
  int line, shift;    // boundary line and its neighbour along the normal
  int size0, size1;   // face extent along nyp, nypp
  int lo0, lo1;       // first live row / column (second order)
  float coeff, c2, c3p, c3q;
  long long off;      // offset of the face's cells in the state arrays
};

struct MurArgs {
  int nfaces, order;
  MurFaceDev f[6];
  long long total;  // face cells over all faces
  float* v;         // [2][total] pending boundary values
  float* ob;        // [2][total] boundary line at n-1 (second order)
  float* os;        // [2][total] shift line at n-1 (second order)
  float* e[3];
  int ny, nzp;      // grid (row pitch)
};

__device__ __forceinline__ long long mur_cell(const MurArgs& a, const MurFaceDev& F, int line, int p, int q) {
  int pos[3];
  pos[F.ny] = line;
  pos[F.nyp] = p;
  pos[F.nypp] = q;
  return ((long long)pos[0] * a.ny + pos[1]) * a.nzp + pos[2];
}

// face index and (p, q) of global face cell t; false if t is past the end
__device__ __forceinline__ bool mur_locate(const MurArgs& a, long long t, int& fi, int& p, int& q) {
  if (t >= a.total) return false;
  fi = 0;
  while (fi + 1 < a.nfaces && t >= a.f[fi + 1].off) ++fi;
  const long long m = t - a.f[fi].off;
  p = (int)(m / a.f[fi].size1);
  q = (int)(m - (long long)p * a.f[fi].size1);
  return true;
}

__device__ __forceinline__ float mur_lap(const MurArgs& a, const float* W, const MurFaceDev& F, int line, int p, int q,
                                         bool along_p) {
  const long long i1 = along_p ? mur_cell(a, F, line, p + 1, q) : mur_cell(a, F, line, p, q + 1);
  const long long i2 = along_p ? mur_cell(a, F, line, p - 1, q) : mur_cell(a, F, line, p, q - 1);
  const float s1 = __fadd_rn(W[i1], W[i2]);
  const float s2 = __fmul_rn(2.0f, W[mur_cell(a, F, line, p, q)]);
  return __fsub_rn(s1, s2);
}

__global__ void k_mur_pre(const MurArgs a) {
  int fi, p, q;
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (!mur_locate(a, t, fi, p, q)) return;
  const MurFaceDev& F = a.f[fi];
  if (p < F.lo0 || q < F.lo1) return;
  const bool interior = a.order == 2 && p > F.lo0 + 1 && p + 2 < F.size0 && q > F.lo1 + 1 && q + 2 < F.size1;
  const int comp[2] = {F.nyp, F.nypp};
  for (int c = 0; c < 2; ++c) {
    const float* W = a.e[comp[c]];
    const float wb = W[mur_cell(a, F, F.line, p, q)];
    const float ws = W[mur_cell(a, F, F.shift, p, q)];
    const long long m = (long long)c * a.total + t;
    if (!interior) {
      a.v[m] = __fsub_rn(ws, __fmul_rn(F.coeff, wb));
    } else {
      float acc = __fsub_rn(__fmul_rn(F.coeff, a.ob[m]), a.os[m]);
      acc = __fadd_rn(acc, __fmul_rn(F.c2, __fadd_rn(wb, ws)));
      const float lp = __fadd_rn(mur_lap(a, W, F, F.line, p, q, true), mur_lap(a, W, F, F.shift, p, q, true));
      acc = __fadd_rn(acc, __fmul_rn(F.c3p, lp));
      const float lq = __fadd_rn(mur_lap(a, W, F, F.line, p, q, false), mur_lap(a, W, F, F.shift, p, q, false));
      acc = __fadd_rn(acc, __fmul_rn(F.c3q, lq));
      a.v[m] = acc;
    }
    if (a.order == 2) {
      a.ob[m] = wb;
      a.os[m] = ws;
    }
  }
}

__global__ void k_mur_post(const MurArgs a) {
  int fi, p, q;
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (!mur_locate(a, t, fi, p, q)) return;
  const MurFaceDev& F = a.f[fi];
  if (p < F.lo0 || q < F.lo1) return;
  const int comp[2] = {F.nyp, F.nypp};
  for (int c = 0; c < 2; ++c) {
    const long long m = (long long)c * a.total + t;
    a.v[m] = __fadd_rn(a.v[m], __fmul_rn(F.coeff, a.e[comp[c]][mur_cell(a, F, F.shift, p, q)]));
  }
}

// A component at a cell is written by the last enabled face that owns it.
__global__ void k_mur_apply(const MurArgs a) {
  int fi, p, q;
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (!mur_locate(a, t, fi, p, q)) return;
  const MurFaceDev& F = a.f[fi];
  if (p < F.lo0 || q < F.lo1) return;
  int pos[3];
  pos[F.ny] = F.line;
  pos[F.nyp] = p;
  pos[F.nypp] = q;
  const int comp[2] = {F.nyp, F.nypp};
  for (int c = 0; c < 2; ++c) {
    bool later = false;
    for (int g = fi + 1; g < a.nfaces; ++g) {
      const MurFaceDev& G = a.f[g];
      if (comp[c] == G.ny || pos[G.ny] != G.line) continue;
      if (pos[G.nyp] < G.lo0 || pos[G.nypp] < G.lo1) continue;
      later = true;
    }
    if (!later) a.e[comp[c]][mur_cell(a, F, F.line, p, q)] = a.v[(long long)c * a.total + t];
  }
}

}  // namespace oems
