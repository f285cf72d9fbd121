// lumped_ade.cuh -- per-cell extension kernels applied after the E update:
// dispersive ADE point lists and the reference's lumped RLC elements.
//
// Dispersive (src/extensions/dispersive.rs), all three components per cell:
//   Drude   (:510-535)  j = a j + b e;  e = e - c j
//   Lorentz (:171-196)  j = a j + c e;  e = e - b j        (as the reference)
//   Debye   (:604-630)  p' = a p + b e; e = e - c (p' - p) / dt
//   second order (no counterpart: the reference's Lorentz drops P^{n-1} and
//   diverges): p' = (a p + b p_prev) + c e_n; e = e - c2 (p' - p), with e_n
//   the field before the E update (k_dispersive_pre), as the standard
//   explicit Lorentz ADE; kind 3 Lorentz, kind 4 Drude (omega_0 = 0)
// LumpedRlc (src/extensions/lumped_rlc.rs:263-286): e' = v_vv e + v_il int;
//   int = int + e dt.
// Arithmetic order and rounding match the f32 reference (no FMA).
#pragma once

#include <cuda_runtime.h>

namespace oems {

struct DispArgs {
  int kind;
  float a, b, c, c2, dtf;
  long long n;
  const long long* q;  // cell (padded linear index)
  float* st;           // [3][n] J or P
  float* pp;           // [3][n] P at n-1 (second-order kinds)
  float* ep;           // [3][n] E^n (second-order kinds)
  float* e[3];
};

// E^n of the second-order kinds, copied before the E update.
__global__ void k_dispersive_pre(const DispArgs a) {
  const long long m = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (m >= a.n) return;
  const long long q = a.q[m];
#pragma unroll
  for (int c = 0; c < 3; ++c) a.ep[(long long)c * a.n + m] = a.e[c][q];
}

__global__ void k_dispersive(const DispArgs a) {
  const long long m = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (m >= a.n) return;
  const long long q = a.q[m];
#pragma unroll
  for (int c = 0; c < 3; ++c) {
    float* ef = a.e[c] + q;
    const float e = *ef;
    float* sp = a.st + (long long)c * a.n + m;
    const float old = *sp;
    if (a.kind == 0) {
      const float jn = __fadd_rn(__fmul_rn(a.a, old), __fmul_rn(a.b, e));
      *sp = jn;
      *ef = __fsub_rn(e, __fmul_rn(a.c, jn));
    } else if (a.kind == 1) {
      const float jn = __fadd_rn(__fmul_rn(a.a, old), __fmul_rn(a.c, e));
      *sp = jn;
      *ef = __fsub_rn(e, __fmul_rn(a.b, jn));
    } else if (a.kind == 2) {
      const float pn = __fadd_rn(__fmul_rn(a.a, old), __fmul_rn(a.b, e));
      *sp = pn;
      const float dpdt = __fdiv_rn(__fsub_rn(pn, old), a.dtf);
      *ef = __fsub_rn(e, __fmul_rn(a.c, dpdt));
    } else {
      float* ppp = a.pp + (long long)c * a.n + m;
      const float en = a.ep[(long long)c * a.n + m];
      const float pn = __fadd_rn(__fadd_rn(__fmul_rn(a.a, old), __fmul_rn(a.b, *ppp)), __fmul_rn(a.c, en));
      *ppp = old;
      *sp = pn;
      *ef = __fsub_rn(e, __fmul_rn(a.c2, __fsub_rn(pn, old)));
    }
  }
}

struct RlcArgs {
  int n;
  const long long* q;
  const int* dir;
  const float* v_vv;
  const float* v_il;
  float* i_int;
  float dtf;
  float* e[3];
};

// Elements in list order (one thread), so elements on the same edge compose
// like the reference's sequential loop.
__global__ void k_lumped_rlc(const RlcArgs a) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  for (int m = 0; m < a.n; ++m) {
    float* ef = a.e[a.dir[m]] + a.q[m];
    const float e = *ef;
    const float en = __fadd_rn(__fmul_rn(a.v_vv[m], e), __fmul_rn(a.v_il[m], a.i_int[m]));
    a.i_int[m] = __fadd_rn(a.i_int[m], __fmul_rn(e, a.dtf));
    *ef = en;
  }
}

}  // namespace oems
