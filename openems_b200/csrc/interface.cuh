// Field reads and writes of the engine interface: EngineInterface and
// EngineInterfaceMut (src/fdtd/engine_interface.rs:27-595), run on the
// resident fields.
//
// A query is a physical position (metres) or, for the raw reads, a cell.  A
// position snaps to its cell like EngineInterface::snap_to_grid (:327-333):
// per axis the first cell whose two mesh lines bracket the coordinate
// (Grid::find_cell_x, src/geometry/mod.rs:334-342; the coordinate is divided
// by the grid unit first), the last cell (lines - 2) when none does, then
// clamped to cells - 1.  The reference scans the lines; on non-decreasing
// lines the same cell is the first line pair whose upper line is >= the
// coordinate, found here by bisection, and an axis whose lines are not sorted
// falls back to the scan.
//
// Node interpolation (:380-437) is the trilinear blend of the eight values
// around the snapped cell, the upper neighbour clamped to the last cell, with
// the fractions (pos - line) / delta clamped to [0, 1]; cell interpolation
// (:482-504) moves the position by half of the snapped cell's deltas and
// interpolates to the node there.  curl H (:336-377) takes each difference in
// f32, widens it and divides by the delta in f64, 0 at the upper edge.  Every
// f64 product and sum is rounded on its own (__dmul_rn / __dadd_rn /
// __dsub_rn / __ddiv_rn), in the reference's order, so the results are the
// bits of the reference's arithmetic.
#pragma once

#include <cuda_runtime.h>

namespace oems {

struct SampleArgs {
  const float* f[6];                      // Ex Ey Ez Hx Hy Hz, padded layout
  int nx, ny, nz, nzp;
  const double* lines[3];                 // mesh lines per axis (grid units)
  int nl[3];                              // lines per axis
  int sorted[3];                          // 1: lines non-decreasing (bisection)
  double unit;                            // metres per grid unit
  const double* pos;                      // [count][3] metres, or null
  const unsigned long long* cells_in;     // [count][3] cells (raw reads), or null
  long long count;
  int quantity;                           // 0 E, 1 H, 2 curl H
  int interp;                             // 0 none, 1 node, 2 cell
  double* out;                            // [count][3]
  unsigned long long* cells_out;          // [count][3] snapped cells, or null
  float h_inv;                            // 2-byte storage: 1 / the H scale
};

// Grid::find_cell_x on lines l[0..n).
__device__ __forceinline__ int iface_find_cell(const double* l, int n, int sorted, double x) {
  if (n < 2) return 0;
  if (sorted) {
    // first pair index i in [0, n-2] with x <= l[i+1]
    int lo = 0, hi = n - 1;  // answer in [lo, hi]; hi = n-1 means none
    while (lo < hi) {
      const int mid = (lo + hi) >> 1;
      if (x <= l[mid + 1])
        hi = mid;
      else
        lo = mid + 1;
    }
    if (lo < n - 1 && x >= l[lo]) return lo;
    return n - 2;
  }
  for (int i = 0; i + 1 < n; ++i)
    if (x >= l[i] && x <= l[i + 1]) return i;
  return n - 2;
}

// Grid::x_line (src/geometry/mod.rs:317-319).
__device__ __forceinline__ double iface_line(const SampleArgs& a, int ax, int i) {
  return __dmul_rn(i < a.nl[ax] ? a.lines[ax][i] : 0.0, a.unit);
}

// Grid::delta_x (src/geometry/mod.rs:281-289).
__device__ __forceinline__ double iface_delta(const SampleArgs& a, int ax, int i) {
  const double* l = a.lines[ax];
  if (i + 1 < a.nl[ax]) return __dmul_rn(__dsub_rn(l[i + 1], l[i]), a.unit);
  if (i > 0) return __dmul_rn(__dsub_rn(l[i], l[i - 1]), a.unit);
  return a.unit;
}

__device__ __forceinline__ void iface_snap(const SampleArgs& a, const double p[3], int c[3]) {
  const int n[3] = {a.nx, a.ny, a.nz};
  for (int ax = 0; ax < 3; ++ax) {
    const int i = iface_find_cell(a.lines[ax], a.nl[ax], a.sorted[ax], __ddiv_rn(p[ax], a.unit));
    c[ax] = i < n[ax] - 1 ? i : n[ax] - 1;
  }
}

template <typename T>
__device__ __forceinline__ float iface_value(const SampleArgs& a, int comp, int i, int j, int k) {
  const long long q = ((long long)i * a.ny + j) * a.nzp + k;
  if constexpr (std::is_same<T, float>::value) {
    return a.f[comp][q];
  } else {
    const float v = FieldIO<T>::ld1(a.f[comp], q);
    return comp < 3 ? v : v * a.h_inv;
  }
}

// c0 * (1 - f) + c1 * f
__device__ __forceinline__ double iface_lerp(double c0, double c1, double f) {
  return __dadd_rn(__dmul_rn(c0, __dsub_rn(1.0, f)), __dmul_rn(c1, f));
}

__device__ __forceinline__ double iface_clamp01(double f) { return f < 0.0 ? 0.0 : (f > 1.0 ? 1.0 : f); }

// interpolate_{e,h}_field_to_node (:380-479) of the three components base..base+2.
template <typename T>
__device__ void iface_node(const SampleArgs& a, int base, const double p[3], double out[3]) {
  int c[3];
  iface_snap(a, p, c);
  double fr[3];
  for (int ax = 0; ax < 3; ++ax)
    fr[ax] = iface_clamp01(__ddiv_rn(__dsub_rn(p[ax], iface_line(a, ax, c[ax])), iface_delta(a, ax, c[ax])));
  const int i = c[0], j = c[1], k = c[2];
  const int i1 = i + 1 < a.nx - 1 ? i + 1 : a.nx - 1;
  const int j1 = j + 1 < a.ny - 1 ? j + 1 : a.ny - 1;
  const int k1 = k + 1 < a.nz - 1 ? k + 1 : a.nz - 1;
  for (int d = 0; d < 3; ++d) {
    const int m = base + d;
    const double c000 = iface_value<T>(a, m, i, j, k), c100 = iface_value<T>(a, m, i1, j, k);
    const double c010 = iface_value<T>(a, m, i, j1, k), c110 = iface_value<T>(a, m, i1, j1, k);
    const double c001 = iface_value<T>(a, m, i, j, k1), c101 = iface_value<T>(a, m, i1, j, k1);
    const double c011 = iface_value<T>(a, m, i, j1, k1), c111 = iface_value<T>(a, m, i1, j1, k1);
    const double c00 = iface_lerp(c000, c100, fr[0]), c01 = iface_lerp(c001, c101, fr[0]);
    const double c10 = iface_lerp(c010, c110, fr[0]), c11 = iface_lerp(c011, c111, fr[0]);
    const double c0 = iface_lerp(c00, c10, fr[1]), c1 = iface_lerp(c01, c11, fr[1]);
    out[d] = iface_lerp(c0, c1, fr[2]);
  }
}

// (h[hi] - h[lo]) in f32, widened, / delta; 0 when hi is outside the grid
template <typename T>
__device__ __forceinline__ double iface_diff(const SampleArgs& a, int comp, int ax, int i, int j, int k) {
  const int n[3] = {a.nx, a.ny, a.nz};
  int c[3] = {i, j, k};
  if (c[ax] + 1 >= n[ax]) return 0.0;
  const float lo = iface_value<T>(a, comp, i, j, k);
  c[ax] += 1;
  const float hi = iface_value<T>(a, comp, c[0], c[1], c[2]);
  return __ddiv_rn((double)__fsub_rn(hi, lo), iface_delta(a, ax, ax == 0 ? i : ax == 1 ? j : k));
}

// calc_curl_h (:336-377)
template <typename T>
__device__ void iface_curl_h(const SampleArgs& a, int i, int j, int k, double out[3]) {
  out[0] = __dsub_rn(iface_diff<T>(a, 5, 1, i, j, k), iface_diff<T>(a, 4, 2, i, j, k));
  out[1] = __dsub_rn(iface_diff<T>(a, 3, 2, i, j, k), iface_diff<T>(a, 5, 0, i, j, k));
  out[2] = __dsub_rn(iface_diff<T>(a, 4, 0, i, j, k), iface_diff<T>(a, 3, 1, i, j, k));
}

// One query per thread.
template <typename T>
__global__ void k_iface_sample(const SampleArgs a) {
  const long long q = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= a.count) return;
  int c[3];
  double p[3] = {0.0, 0.0, 0.0};
  if (a.cells_in) {
    for (int ax = 0; ax < 3; ++ax) c[ax] = (int)a.cells_in[3 * q + ax];
  } else {
    for (int ax = 0; ax < 3; ++ax) p[ax] = a.pos[3 * q + ax];
    iface_snap(a, p, c);
  }
  double v[3];
  const int base = a.quantity == 1 ? 3 : 0;
  if (a.quantity == 2) {
    iface_curl_h<T>(a, c[0], c[1], c[2], v);
  } else if (a.cells_in || a.interp == 0) {
    for (int d = 0; d < 3; ++d) v[d] = iface_value<T>(a, base + d, c[0], c[1], c[2]);
  } else if (a.interp == 1) {
    iface_node<T>(a, base, p, v);
  } else {
    double s[3];
    for (int ax = 0; ax < 3; ++ax) s[ax] = __dadd_rn(p[ax], __dmul_rn(iface_delta(a, ax, c[ax]), 0.5));
    iface_node<T>(a, base, s, v);
  }
  for (int d = 0; d < 3; ++d) a.out[3 * q + d] = v[d];
  if (a.cells_out)
    for (int ax = 0; ax < 3; ++ax) a.cells_out[3 * q + ax] = (unsigned long long)c[ax];
}

// calc_voltage_integral (kind 0, :208-247) and calc_current_integral (kind 1,
// :251-305) between two positions, on one thread in the reference's loop
// order: V -= E * d per edge; I += (H_a * d_b - H_b * d_a) per face cell, the
// pair's difference rounded before it is added.
struct IntegralArgs {
  SampleArgs s;  // grid, lines and fields (no queries)
  double start[3], stop[3];
  int kind, normal;
  double* out;
};

template <typename T>
__global__ void k_iface_integral(const IntegralArgs a) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  const SampleArgs& g = a.s;
  int s[3], t[3];
  iface_snap(g, a.start, s);
  iface_snap(g, a.stop, t);
  const int n[3] = {g.nx, g.ny, g.nz};
  int lo[3], hi[3];
  for (int ax = 0; ax < 3; ++ax) {
    lo[ax] = s[ax] < t[ax] ? s[ax] : t[ax];
    hi[ax] = s[ax] < t[ax] ? t[ax] : s[ax];
  }
  auto cl = [&](int ax, int v) { return v < n[ax] - 1 ? v : n[ax] - 1; };
  double acc = 0.0;
  if (a.kind == 0) {
    for (int i = lo[0]; i < hi[0]; ++i) {
      const int c = cl(0, i);
      acc = __dsub_rn(acc, __dmul_rn((double)iface_value<T>(g, 0, c, s[1], s[2]), iface_delta(g, 0, c)));
    }
    for (int j = lo[1]; j < hi[1]; ++j) {
      const int c = cl(1, j);
      acc = __dsub_rn(acc, __dmul_rn((double)iface_value<T>(g, 1, t[0], c, s[2]), iface_delta(g, 1, c)));
    }
    for (int k = lo[2]; k < hi[2]; ++k) {
      const int c = cl(2, k);
      acc = __dsub_rn(acc, __dmul_rn((double)iface_value<T>(g, 2, t[0], t[1], c), iface_delta(g, 2, c)));
    }
  } else {
    // normal 0: Hy dz - Hz dy over (j, k) at i_start; 1: Hz dx - Hx dz over
    // (i, k) at j_start; else: Hx dy - Hy dx over (i, j) at k_start
    const int nd = a.normal == 0 ? 0 : a.normal == 1 ? 1 : 2;
    const int u = nd == 0 ? 1 : 0, v = nd == 2 ? 1 : 2;  // the two in-plane axes, u < v
    // component multiplied by d_v, and the one multiplied by d_u (subtracted)
    const int cp = nd == 0 ? 4 : nd == 1 ? 5 : 3;
    const int cm = nd == 0 ? 5 : nd == 1 ? 3 : 4;
    // in the reference's sums the term added carries the delta of axis
    // (nd 0: z, nd 1: x, nd 2: y) and the term subtracted the other one
    const int ap = nd == 0 ? 2 : nd == 1 ? 0 : 1;
    const int am = nd == 0 ? 1 : nd == 1 ? 2 : 0;
    for (int p = lo[u]; p < hi[u]; ++p)
      for (int q = lo[v]; q < hi[v]; ++q) {
        int c[3];
        c[nd] = s[nd];
        c[u] = cl(u, p);
        c[v] = cl(v, q);
        const double hp = iface_value<T>(g, cp, c[0], c[1], c[2]);
        const double hm = iface_value<T>(g, cm, c[0], c[1], c[2]);
        const double dp = iface_delta(g, ap, c[ap]), dm = iface_delta(g, am, c[am]);
        acc = __dadd_rn(acc, __dsub_rn(__dmul_rn(hp, dp), __dmul_rn(hm, dm)));
      }
  }
  *a.out = acc;
}

// A probe term list evaluated once on the current fields, with the probes'
// arithmetic: mode 0 the f32 ordered sum with weights +-1, mode 1 the f64 sum
// of weight * value.  One thread: the sum order is the list order.
struct TermArgs {
  const float* f[6];
  const long long* idx;
  const int* comp;
  const double* w;
  long long n;
  int mode;
  float h_inv;
  double* out;
};

template <typename T>
__device__ __forceinline__ float term_value(const TermArgs& a, int c, long long q) {
  if constexpr (std::is_same<T, float>::value) {
    return a.f[c][q];
  } else {
    const float v = FieldIO<T>::ld1(a.f[c], q);
    return c < 3 ? v : v * a.h_inv;
  }
}

template <typename T>
__global__ void k_iface_terms(const TermArgs a) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  double val;
  if (a.mode == 0) {
    float acc = 0.0f;
    for (long long t = 0; t < a.n; ++t) {
      const float v = term_value<T>(a, a.comp[t], a.idx[t]);
      acc = a.w[t] >= 0.0 ? __fadd_rn(acc, v) : __fsub_rn(acc, v);
    }
    val = (double)acc;
  } else {
    double acc = 0.0;
    for (long long t = 0; t < a.n; ++t)
      acc = __dadd_rn(acc, __dmul_rn(a.w[t], (double)term_value<T>(a, a.comp[t], a.idx[t])));
    val = acc;
  }
  *a.out = val;
}

// EngineInterfaceMut::set_e_field / set_h_field / add_e_field (:542-561):
// the writes in list order (one thread), so a cell named twice ends as the
// sequential loop leaves it.  2-byte storage: H is stored times h_scale,
// rounded to nearest like a field upload.
struct SetArgs {
  float* f[3];          // the three components of E or of H
  const long long* idx; // padded linear index per write
  const float* v;       // [n][3]
  long long n;
  int add;
  float scale;          // h_scale for H in 2-byte storage, else 1
};

template <typename T>
__global__ void k_iface_set(const SetArgs a) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  for (long long t = 0; t < a.n; ++t)
    for (int d = 0; d < 3; ++d) {
      const float v = a.v[3 * t + d];
      if constexpr (std::is_same<T, float>::value) {
        float* p = a.f[d] + a.idx[t];
        *p = a.add ? __fadd_rn(*p, v) : v;
      } else {
        const float cur = FieldIO<T>::ld1(a.f[d], a.idx[t]) / a.scale;
        FieldIO<T>::st1(a.f[d], a.idx[t], __fmul_rn(a.add ? __fadd_rn(cur, v) : v, a.scale));
      }
    }
}

}  // namespace oems
