// fd_nf2ff.cuh -- frequency-domain accumulation and the near-field to
// far-field transform.
//
// Field DFT dumps (src/processing/fields_fd.rs:149-217): X += x w with the
// twiddle w = exp(-j 2 pi f t) 2 dt interval taken from a per-batch table the
// host fills with the same libm cos / sin as the reference formula; E samples
// at t = n dt, H at (n - 1/2) dt.  Products and sums are rounded separately
// (__dmul_rn / __dadd_rn), so the accumulators are bit-identical to a scalar
// f64 loop.
//
// NF2FF box faces: tangential E on the face's node plane p and tangential H
// averaged over the planes p-1 and p (the H half-cells on either side), which
// puts Ec with Hb at (b node, c mid-cell) and Eb with Hc at (b mid-cell, c
// node); b = a+1, c = a+2 (mod 3) for normal axis a.
//
// The far-field transform (the radiation vectors the reference's
// Nf2ff::integrate_surfaces, src/nf2ff/mod.rs:172-188, leaves at zero):
//   N = sum J w exp(+j k r.r'),  L = sum M w exp(+j k r.r')
// over a point list (x y z w, J re/im x 3, M re/im x 3).  One thread per
// observation direction, points staged through shared memory in tiles that
// every thread of the block reuses; the point list is split over blockIdx.y
// and the partial sums are reduced in a fixed order.
#pragma once

#include <cuda_runtime.h>

namespace oems {

struct FieldDftArgs {
  const float* f[6];        // field array per recorded component, in slot order
  unsigned hmask;           // bit ci: slot ci is an H component
  int ncomp, nf;
  long long npts, n1, n2;   // points; points along the 2nd and 3rd axes
  long long r0, r1, r2;     // region start (i, j, k)
  long long s0, s1, s2;     // sub-sampling
  long long ny, nzp;        // padded layout
  const double* tw;         // [batch step][nf][4]: E re, E im, H re, H im
  const int* sampled;       // [batch step]
  const long long* d_base;  // batch step of local step 0
  int local;
  double2* acc;             // [nf][ncomp][npts]
};

__global__ void k_field_dft(const FieldDftArgs a) {
  const long long s = *a.d_base + a.local;
  if (!a.sampled[s]) return;
  const long long p = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= a.npts) return;
  const long long pc = p % a.n2, t = p / a.n2;
  const long long pb = t % a.n1, pa = t / a.n1;
  const long long q = ((a.r0 + pa * a.s0) * a.ny + (a.r1 + pb * a.s1)) * a.nzp + a.r2 + pc * a.s2;
  const double* tw = a.tw + s * (long long)a.nf * 4;
  for (int ci = 0; ci < a.ncomp; ++ci) {
    const double x = (double)a.f[ci][q];
    const int h = (a.hmask >> ci) & 1 ? 2 : 0;
    for (int f = 0; f < a.nf; ++f) {
      double2* z = a.acc + ((long long)f * a.ncomp + ci) * a.npts + p;
      double2 v = *z;
      v.x = __dadd_rn(v.x, __dmul_rn(x, tw[4 * f + h]));
      v.y = __dadd_rn(v.y, __dmul_rn(x, tw[4 * f + h + 1]));
      *z = v;
    }
  }
}

struct Nf2ffFace {
  int a, b, c;
  long long p;            // node plane along a
  long long lo_b, lo_c;   // first node along b and c
  long long nb, nc, np;   // node grid of the face (np = nb nc)
  double2* acc;           // [nf][4][np]: Eb, Ec, Hb, Hc
};

struct Nf2ffAccArgs {
  const float* e[3];
  const float* h[3];
  long long ny, nzp;
  int nfaces, nf;
  Nf2ffFace face[6];
  long long off[7];       // prefix sums of np over the faces
  const double* tw;
  const int* sampled;
  const long long* d_base;
  int local;
};

__global__ void k_nf2ff_acc(const Nf2ffAccArgs a) {
  const long long s = *a.d_base + a.local;
  if (!a.sampled[s]) return;
  const long long g = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (g >= a.off[a.nfaces]) return;
  int fi = 0;
  while (g >= a.off[fi + 1]) ++fi;
  const Nf2ffFace& F = a.face[fi];
  const long long m = g - a.off[fi];
  const long long jb = m / F.nc, kc = m % F.nc;
  long long pos[3];
  pos[F.a] = F.p;
  pos[F.b] = F.lo_b + jb;
  pos[F.c] = F.lo_c + kc;
  const long long q = (pos[0] * a.ny + pos[1]) * a.nzp + pos[2];
  pos[F.a] = F.p - 1;
  const long long qm = (pos[0] * a.ny + pos[1]) * a.nzp + pos[2];
  const double v[4] = {(double)a.e[F.b][q], (double)a.e[F.c][q],
                       __dmul_rn(0.5, __dadd_rn((double)a.h[F.b][qm], (double)a.h[F.b][q])),
                       __dmul_rn(0.5, __dadd_rn((double)a.h[F.c][qm], (double)a.h[F.c][q]))};
  const double* tw = a.tw + s * (long long)a.nf * 4;
  for (int f = 0; f < a.nf; ++f) {
#pragma unroll
    for (int k = 0; k < 4; ++k) {
      const int h = k < 2 ? 0 : 2;
      double2* z = F.acc + ((long long)f * 4 + k) * F.np + m;
      double2 w = *z;
      w.x = __dadd_rn(w.x, __dmul_rn(v[k], tw[4 * f + h]));
      w.y = __dadd_rn(w.y, __dmul_rn(v[k], tw[4 * f + h + 1]));
      *z = w;
    }
  }
}

// Point list of the recorded faces at one frequency.  Per face: first the
// (b node, c cell) points carrying J_c = s Hb, M_b = s Ec, b-major; then the
// (b cell, c node) points carrying J_b = -s Hc, M_c = -s Eb; s = -1 on a min
// face, +1 on a max face (n = s e_a, J = n x H, M = -n x E).  Weights are the
// dual-cell widths (half at the box edges) times the cell widths.
struct Nf2ffPointsArgs {
  int nfaces;
  Nf2ffFace face[6];
  int sign[6];
  long long off[7];        // prefix sums of the point counts per face
  int f;                   // frequency index
  const double* lines[3];  // mesh lines (m) per axis, device
  double* pts;             // [n][16]
};

__device__ __forceinline__ double dual_width(const double* l, long long lo, long long hi, long long j) {
  const long long j0 = j - 1 < lo ? lo : j - 1, j1 = j + 1 > hi ? hi : j + 1;
  return 0.5 * (l[j1] - l[j0]);
}

__global__ void k_nf2ff_points(const Nf2ffPointsArgs a) {
  const long long g = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (g >= a.off[a.nfaces]) return;
  int fi = 0;
  while (g >= a.off[fi + 1]) ++fi;
  const Nf2ffFace& F = a.face[fi];
  const double s = (double)a.sign[fi];
  long long m = g - a.off[fi];
  const double* lb = a.lines[F.b];
  const double* lc = a.lines[F.c];
  const long long hb = F.lo_b + F.nb - 1, hc = F.lo_c + F.nc - 1;
  const long long set1 = F.nb * (F.nc - 1);
  double r[16];
#pragma unroll
  for (int t = 0; t < 16; ++t) r[t] = 0.0;
  r[F.a] = a.lines[F.a][F.p];
  const double2* acc = F.acc + (long long)a.f * 4 * F.np;
  if (m < set1) {
    const long long jb = m / (F.nc - 1), kc = m % (F.nc - 1);
    const long long B = F.lo_b + jb, C = F.lo_c + kc;
    r[F.b] = lb[B];
    r[F.c] = 0.5 * (lc[C] + lc[C + 1]);
    r[3] = dual_width(lb, F.lo_b, hb, B) * (lc[C + 1] - lc[C]);
    const long long q = jb * F.nc + kc;
    const double2 hbv = acc[2 * F.np + q], ecv = acc[1 * F.np + q];
    r[4 + 2 * F.c] = s * hbv.x;
    r[5 + 2 * F.c] = s * hbv.y;
    r[10 + 2 * F.b] = s * ecv.x;
    r[11 + 2 * F.b] = s * ecv.y;
  } else {
    m -= set1;
    const long long jb = m / F.nc, kc = m % F.nc;
    const long long B = F.lo_b + jb, C = F.lo_c + kc;
    r[F.b] = 0.5 * (lb[B] + lb[B + 1]);
    r[F.c] = lc[C];
    r[3] = (lb[B + 1] - lb[B]) * dual_width(lc, F.lo_c, hc, C);
    const long long q = jb * F.nc + kc;
    const double2 hcv = acc[3 * F.np + q], ebv = acc[0 * F.np + q];
    r[4 + 2 * F.b] = -s * hcv.x;
    r[5 + 2 * F.b] = -s * hcv.y;
    r[10 + 2 * F.c] = -s * ebv.x;
    r[11 + 2 * F.c] = -s * ebv.y;
  }
  double* o = a.pts + g * 16;
#pragma unroll
  for (int t = 0; t < 16; ++t) o[t] = r[t];
}

constexpr int kFarThreads = 128;  // directions per block
constexpr int kFarTile = 64;      // points per shared-memory tile

struct Nf2ffFarArgs {
  const double* pts;   // [npts][16]
  long long npts;
  long long chunk;     // points per blockIdx.y
  const double* dirs;  // [ndir][3] unit vectors r^
  int ndir;
  double k, cx, cy, cz;
  double* partial;     // [gridDim.y][ndir][12]: N (re, im) x 3, L (re, im) x 3
};

__global__ void __launch_bounds__(kFarThreads) k_nf2ff_far(const Nf2ffFarArgs a) {
  __shared__ double tile[kFarTile * 16];
  const int d = blockIdx.x * kFarThreads + threadIdx.x;
  double rx = 0.0, ry = 0.0, rz = 0.0;
  if (d < a.ndir) {
    rx = a.dirs[3 * d];
    ry = a.dirs[3 * d + 1];
    rz = a.dirs[3 * d + 2];
  }
  double acc[12];
#pragma unroll
  for (int t = 0; t < 12; ++t) acc[t] = 0.0;
  const long long p0 = (long long)blockIdx.y * a.chunk;
  long long p1 = p0 + a.chunk;
  if (p1 > a.npts) p1 = a.npts;
  for (long long t0 = p0; t0 < p1; t0 += kFarTile) {
    const int nt = (int)((p1 - t0) < kFarTile ? (p1 - t0) : kFarTile);
    __syncthreads();
    for (int u = threadIdx.x; u < nt * 16; u += kFarThreads) tile[u] = a.pts[t0 * 16 + u];
    __syncthreads();
    for (int u = 0; u < nt; ++u) {
      const double* P = tile + 16 * u;
      const double ph = a.k * (rx * (P[0] - a.cx) + ry * (P[1] - a.cy) + rz * (P[2] - a.cz));
      double sn, cs;
      sincos(ph, &sn, &cs);
      cs *= P[3];
      sn *= P[3];
#pragma unroll
      for (int v = 0; v < 6; ++v) {
        const double re = P[4 + 2 * v], im = P[5 + 2 * v];
        acc[2 * v] += re * cs - im * sn;
        acc[2 * v + 1] += re * sn + im * cs;
      }
    }
  }
  if (d < a.ndir) {
    double* o = a.partial + ((long long)blockIdx.y * a.ndir + d) * 12;
#pragma unroll
    for (int t = 0; t < 12; ++t) o[t] = acc[t];
  }
}

__global__ void k_nf2ff_reduce(const double* partial, int nchunks, int ndir, double* out) {
  const int g = blockIdx.x * blockDim.x + threadIdx.x;
  if (g >= ndir * 12) return;
  double s = 0.0;
  for (int c = 0; c < nchunks; ++c) s += partial[(long long)c * ndir * 12 + g];
  out[g] = s;
}

}  // namespace oems
