// yee_kernels.cuh -- sm_100a Yee update kernels (H and E half-steps).
//
// Semantics follow the reference scalar engine:
//   H: src/fdtd/basic_engine.rs:191-254  (every cell; a forward difference that
//      would reach index n is 0)
//   E: src/fdtd/basic_engine.rs:262-306  (only i, j, k >= 1 are written)
// Every product and sum is rounded separately (__fmul_rn / __fadd_rn /
// __fsub_rn, no FMA contraction) in the reference's order, so an FP32 run is
// bit-identical to the unfused Rust arithmetic.  The stencil is HBM-bound; the
// rounding mode costs nothing.
//
// Data layout in HBM: one array per component, z fastest, rows padded to
// nzp = round_up(nz, 4) floats so every (i, j) row starts 16-byte aligned.
// Thread mapping: one thread owns one float4 chunk (4 consecutive k) of an
// x-plane; a warp covers 32 consecutive chunks of the flattened (j, k) plane,
// so every access is a fully coalesced 128-bit load or store whatever nz is.
// Each CTA marches its tile of chunks through `ichunk` consecutive x-planes,
// carrying the x-neighbour plane in registers (register-blocked marching along
// x).  z-neighbours come from the adjacent lane by warp shuffle; y-neighbours
// are the same tile one row over and hit L1.  CTAs loop over (tile, x-chunk)
// work items, so the grid is sized to the number of resident CTAs.
//
// Per plane, a thread first issues every load it needs (fields, neighbours,
// coefficients and, in CPML slabs, the psi values) and only then shuffles and
// computes, so all of its memory requests are in flight together.
//
// CPML (standard Roden-Gedney recursive convolution with the profile of
// src/extensions/cpml.rs:68-177) is fused: in a slab cell the difference d
// along the slab normal becomes d*inv_kappa + psi with psi = b*psi + c*d.
#pragma once

#include <cuda_bf16.h>
#include <cuda_fp16.h>

#include <cuda_runtime.h>
#include <stdint.h>

namespace oems {

constexpr unsigned kFullMask = 0xffffffffu;

// A segment of the update: x-planes [i0, i1) x rows [j0, j0 + n / w) x
// float4 chunks [q0, q0 + w) of each row.  Its n chunks are numbered row by
// row (local index c -> row j0 + c / w, chunk q0 + c % w) and cut into tiles
// of one CTA's chunks and runs of `ichunk` planes; work items of all
// segments are numbered consecutively from work0.  A segment of whole rows
// (q0 = 0, w = chunks per row) is a contiguous range of the plane; a partial
// one (the chunks between or inside the z slabs) is not, and its row ends
// fall inside warps.
struct Seg {
  int i0, i1;
  int j0, q0, w, n;
  int tiles, work0;
};
constexpr int kMaxSeg = 6;

struct Geom {
  int nx, ny, nz, nzp, nzq;  // nzq = nzp / 4 float4 chunks per row
  long long plane;           // floats per x-plane = ny * nzp
  int plane4;                // float4 chunks per x-plane = ny * nzq
  int tiles;                 // CTA tiles per x-plane
  int ichunk;                // x-planes per work item
  int nchunks;               // ceil(nx / ichunk)
  int work;                  // work items over all segments
  int pf;                    // L2 prefetch distance in x-planes (0 = off)
  int nseg;                  // segments (1 = the whole grid)
  Seg seg[kMaxSeg];
};

// Work item w -> segment, tile (local chunks [c0, c1)) and plane run.
struct Item {
  int c0, c1, i0, i1, tile;
  int j0, q0, w;
  bool whole;  // whole rows: c0..c1 is contiguous in the plane
};
__device__ __forceinline__ Item work_item(const Geom& g, int w) {
  int s = 0;
  while (s + 1 < g.nseg && w >= g.seg[s + 1].work0) ++s;
  const Seg& S = g.seg[s];
  const int lw = w - S.work0;
  Item it;
  it.tile = lw % S.tiles;
  it.c0 = it.tile * (int)blockDim.x;
  it.c1 = min(it.c0 + (int)blockDim.x, S.n);
  it.i0 = S.i0 + (lw / S.tiles) * g.ichunk;
  it.i1 = min(it.i0 + g.ichunk, S.i1);
  it.j0 = S.j0;
  it.q0 = S.q0;
  it.w = S.w;
  it.whole = S.w == g.nzq;
  return it;
}

// One thread per CTA asks L2 for the CTA's slice of plane p of an array ahead
// of the loads (cp.async.bulk.prefetch: no registers, no completion to wait
// for).  The slice is the tile's contiguous floats [o, o + n), widened by
// `lo` floats before and `hi` after for the y-neighbour row, clamped to the
// array; every bound is a multiple of 4 floats, so the 16-byte rule holds.
__device__ __forceinline__ void l2_prefetch(const float* arr, long long o, long long n, long long limit) {
  if (o < 0) {
    n += o;
    o = 0;
  }
  if (o + n > limit) n = limit - o;
  if (n <= 0) return;
  asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;" ::"l"(arr + o), "r"((uint32_t)(n * 4)) : "memory");
}

// CPML state on the device.  Faces: 0 xmin 1 xmax 2 ymin 3 ymax 4 zmin 5 zmax.
// psi layout per face:
//   x faces [l][j][k]  (k pitch nzp)
//   y faces [i][l][k]  (k pitch nzp)
//   z faces [i][j][w]  w = k - zbase[f], width zw[f] (multiple of 4) so that a
//                      float4 chunk of k maps to an aligned float4 of psi.
// Slot per axis: x: H {Hy, Hz} E {Ey, Ez}; y: H {Hx, Hz} E {Ex, Ez};
// z: H {Hx, Hy} E {Ex, Ey}.
struct CpmlArgs {
  int L[6];
  int start[6];       // first global index of the slab along its axis
  int prof_off[6];    // offset of face f in prof: 6 rows of L: b_e c_e ik_e b_h c_h ik_h
  int zbase[2];       // z faces: first k of the psi row (multiple of 4)
  int zw[2];          // z faces: psi row width (multiple of 4)
  const float* prof;
  float* psi_h[6][2];
  float* psi_e[6][2];
};

struct HArgs {
  Geom g;
  const float* ex;
  const float* ey;
  const float* ez;
  float* hx;
  float* hy;
  float* hz;
  const float* da[3];
  const float* db[3];
  const void* ids;     // compressed: per-cell material id (uint8 or uint16)
  const float* table;  // compressed: [ntable][12] = ca0..2 cb0..2 da0..2 db0..2
  int ntable;
  CpmlArgs cp;
};

struct EArgs {
  Geom g;
  float* ex;
  float* ey;
  float* ez;
  const float* hx;
  const float* hy;
  const float* hz;
  const float* ca[3];
  const float* cb[3];
  const void* ids;
  const float* table;
  int ntable;
  CpmlArgs cp;
};

__device__ __forceinline__ float4 ld_nc4(const float* p) { return __ldg(reinterpret_cast<const float4*>(p)); }
__device__ __forceinline__ float4 ld_cs4(const float* p) { return __ldcs(reinterpret_cast<const float4*>(p)); }
__device__ __forceinline__ float4 ld4(const float* p) { return *reinterpret_cast<const float4*>(p); }
__device__ __forceinline__ void st4(float* p, float4 v) { *reinterpret_cast<float4*>(p) = v; }

// Field storage: float (the reference's layout), or IEEE half / bfloat16
// with the arithmetic still in float (values converted on load, rounded to
// nearest on store).  Offsets are in elements; a chunk of 4 elements starts
// at a multiple of 4, so it is one 16-byte (float) or 8-byte (2-byte types)
// access.  Field pointers travel as float* and are reinterpreted here.
template <typename T>
struct FieldIO;

template <>
struct FieldIO<float> {
  static constexpr bool kFloat = true;
  __device__ __forceinline__ static float4 ldg4(const float* b, long long q) {
    return __ldg(reinterpret_cast<const float4*>(b + q));
  }
  __device__ __forceinline__ static float4 ld4(const float* b, long long q) {
    return *reinterpret_cast<const float4*>(b + q);
  }
  __device__ __forceinline__ static void st4(float* b, long long q, float4 v) {
    *reinterpret_cast<float4*>(b + q) = v;
  }
  __device__ __forceinline__ static float ldg1(const float* b, long long q) { return __ldg(b + q); }
  __device__ __forceinline__ static float ld1(const float* b, long long q) { return b[q]; }
  __device__ __forceinline__ static void st1(float* b, long long q, float v) { b[q] = v; }
};

template <typename H2, typename H1>
struct FieldIO2 {
  static constexpr bool kFloat = false;
  __device__ __forceinline__ static float4 unpack(uint2 r) {
    const float2 lo = cvt(*reinterpret_cast<const H2*>(&r.x));
    const float2 hi = cvt(*reinterpret_cast<const H2*>(&r.y));
    return make_float4(lo.x, lo.y, hi.x, hi.y);
  }
  __device__ __forceinline__ static float4 ldg4(const float* b, long long q) {
    return unpack(__ldg(reinterpret_cast<const uint2*>(reinterpret_cast<const H1*>(b) + q)));
  }
  __device__ __forceinline__ static float4 ld4(const float* b, long long q) {
    return unpack(*reinterpret_cast<const uint2*>(reinterpret_cast<const H1*>(b) + q));
  }
  __device__ __forceinline__ static void st4(float* b, long long q, float4 v) {
    const H2 lo = pack(v.x, v.y), hi = pack(v.z, v.w);
    uint2 r;
    r.x = *reinterpret_cast<const unsigned int*>(&lo);
    r.y = *reinterpret_cast<const unsigned int*>(&hi);
    *reinterpret_cast<uint2*>(reinterpret_cast<H1*>(b) + q) = r;
  }
  __device__ __forceinline__ static float ldg1(const float* b, long long q) {
    return cvt1(__ldg(reinterpret_cast<const H1*>(b) + q));
  }
  __device__ __forceinline__ static float ld1(const float* b, long long q) {
    return cvt1(reinterpret_cast<const H1*>(b)[q]);
  }
  __device__ __forceinline__ static void st1(float* b, long long q, float v) {
    reinterpret_cast<H1*>(b)[q] = round1(v);
  }
  __device__ __forceinline__ static float2 cvt(H2 h);
  __device__ __forceinline__ static H2 pack(float x, float y);
  __device__ __forceinline__ static float cvt1(H1 h);
  __device__ __forceinline__ static H1 round1(float v);
};

template <>
__device__ __forceinline__ float2 FieldIO2<__half2, __half>::cvt(__half2 h) { return __half22float2(h); }
template <>
__device__ __forceinline__ __half2 FieldIO2<__half2, __half>::pack(float x, float y) {
  return __floats2half2_rn(x, y);
}
template <>
__device__ __forceinline__ float FieldIO2<__half2, __half>::cvt1(__half h) { return __half2float(h); }
template <>
__device__ __forceinline__ __half FieldIO2<__half2, __half>::round1(float v) { return __float2half_rn(v); }
template <>
__device__ __forceinline__ float2 FieldIO2<__nv_bfloat162, __nv_bfloat16>::cvt(__nv_bfloat162 h) {
  return __bfloat1622float2(h);
}
template <>
__device__ __forceinline__ __nv_bfloat162 FieldIO2<__nv_bfloat162, __nv_bfloat16>::pack(float x, float y) {
  return __floats2bfloat162_rn(x, y);
}
template <>
__device__ __forceinline__ float FieldIO2<__nv_bfloat162, __nv_bfloat16>::cvt1(__nv_bfloat16 h) {
  return __bfloat162float(h);
}
template <>
__device__ __forceinline__ __nv_bfloat16 FieldIO2<__nv_bfloat162, __nv_bfloat16>::round1(float v) {
  return __float2bfloat16_rn(v);
}

template <>
struct FieldIO<__half> : FieldIO2<__half2, __half> {};
template <>
struct FieldIO<__nv_bfloat16> : FieldIO2<__nv_bfloat162, __nv_bfloat16> {};

__device__ __forceinline__ void to_arr(float4 v, float (&a)[4]) {
  a[0] = v.x;
  a[1] = v.y;
  a[2] = v.z;
  a[3] = v.w;
}
__device__ __forceinline__ float4 to_f4(const float (&a)[4]) { return make_float4(a[0], a[1], a[2], a[3]); }
__device__ __forceinline__ float4 zero4() { return make_float4(0.f, 0.f, 0.f, 0.f); }

// psi <- b*psi + c*d ; return d*ik + psi (each operation rounded).
__device__ __forceinline__ float cpml_stretch(float d, float& psi, float b, float c, float ik) {
  psi = __fadd_rn(__fmul_rn(b, psi), __fmul_rn(c, d));
  return __fadd_rn(__fmul_rn(d, ik), psi);
}

// Slab lookup along one axis: returns face (or -1) and layer.
__device__ __forceinline__ int cpml_face(const CpmlArgs& cp, int axis, int g, int& l) {
  const int fmin = 2 * axis, fmax = 2 * axis + 1;
  l = 0;
  if (g < cp.L[fmin]) {
    l = g;
    return fmin;
  }
  if (cp.L[fmax] > 0 && g >= cp.start[fmax]) {
    l = g - cp.start[fmax];
    return fmax;
  }
  return -1;
}

// Profile row (b, c, ik) of face f, layer l, for H (is_h) or E positions.
__device__ __forceinline__ void cpml_prof(const CpmlArgs& cp, int f, int l, bool is_h, float& b, float& c,
                                          float& ik) {
  const int L = cp.L[f];
  const float* pr = cp.prof + cp.prof_off[f] + (is_h ? 3 * L : 0);
  b = __ldg(pr + l);
  c = __ldg(pr + L + l);
  ik = __ldg(pr + 2 * L + l);
}

// One slab (x or y): psi float4s already loaded; stretch the 4 elements whose
// `live` bit is set, same layer for all.
__device__ __forceinline__ void stretch_vec(float (&d)[4], float4& p4, float b, float c, float ik, unsigned live) {
  float p[4];
  to_arr(p4, p);
#pragma unroll
  for (int e = 0; e < 4; ++e) {
    if (live & (1u << e)) {
      float pe = p[e];
      d[e] = cpml_stretch(d[e], pe, b, c, ik);
      p[e] = pe;
    }
  }
  p4 = to_f4(p);
}

// z slab: per element, layer = k - start of the face.
__device__ __forceinline__ void stretch_z(const CpmlArgs& cp, int f, int k0, bool is_h, float (&d)[4], float4& p4,
                                          unsigned live) {
  float p[4];
  to_arr(p4, p);
#pragma unroll
  for (int e = 0; e < 4; ++e) {
    const int k = k0 + e;
    const int l = k - cp.start[f];
    if ((live & (1u << e)) && l >= 0 && l < cp.L[f]) {
      float b, c, ik;
      cpml_prof(cp, f, l, is_h, b, c, ik);
      float pe = p[e];
      d[e] = cpml_stretch(d[e], pe, b, c, ik);
      p[e] = pe;
    }
  }
  p4 = to_f4(p);
}

// Per-chunk coefficient fetch: full arrays or compressed table.
template <int kIdBytes>
struct Coef {
  __device__ __forceinline__ static void load(const float* const (&arr)[3], const void* ids, const float* tab,
                                              int off, long long q, float (&c)[3][4]) {
    if constexpr (kIdBytes == 0) {
#pragma unroll
      for (int a = 0; a < 3; ++a) to_arr(ld_cs4(arr[a] + q), c[a]);
    } else if constexpr (kIdBytes == 1) {
      const uint32_t w = __ldcs(reinterpret_cast<const unsigned int*>(static_cast<const uint8_t*>(ids) + q));
#pragma unroll
      for (int e = 0; e < 4; ++e) {
        const int id = (w >> (8 * e)) & 0xff;
#pragma unroll
        for (int a = 0; a < 3; ++a) c[a][e] = tab[id * 12 + off + a];
      }
    } else {
      const uint2 w = __ldcs(reinterpret_cast<const uint2*>(static_cast<const uint16_t*>(ids) + q));
      const uint32_t ws[2] = {w.x, w.y};
#pragma unroll
      for (int e = 0; e < 4; ++e) {
        const int id = (ws[e >> 1] >> (16 * (e & 1))) & 0xffff;
#pragma unroll
        for (int a = 0; a < 3; ++a) c[a][e] = __ldg(tab + id * 12 + off + a);
      }
    }
  }
};

// Loads the compressed table into shared memory (uint8 ids only).
template <int kIdBytes>
__device__ __forceinline__ const float* stage_table(const float* table, int ntable, float* smem) {
  if constexpr (kIdBytes == 1) {
    for (int t = threadIdx.x; t < ntable * 12; t += blockDim.x) smem[t] = __ldg(table + t);
    __syncthreads();
    return smem;
  } else {
    return table;
  }
}

// Which CPML slabs a chunk touches, and where its psi float4s live.
struct SlabInfo {
  int fx, lx, fy, ly;      // x / y face and layer (-1 if none)
  bool zmin, zmax;         // chunk overlaps the z faces
  long long px, py;        // psi offsets (float4 aligned)
  long long pz0, pz1;
};

__device__ __forceinline__ SlabInfo slab_info(const CpmlArgs& cp, const Geom& g, int i, int j, int k0) {
  SlabInfo s;
  s.fx = cpml_face(cp, 0, i, s.lx);
  s.fy = cpml_face(cp, 1, j, s.ly);
  s.px = ((long long)s.lx * g.ny + j) * g.nzp + k0;
  s.py = s.fy >= 0 ? ((long long)i * cp.L[s.fy] + s.ly) * g.nzp + k0 : 0;
  s.zmin = cp.L[4] > 0 && k0 < cp.L[4];
  s.zmax = cp.L[5] > 0 && k0 + 3 >= cp.start[5] && k0 < g.nz;
  const long long zrow = (long long)i * g.ny + j;
  s.pz0 = zrow * cp.zw[0] + k0 - cp.zbase[0];
  s.pz1 = zrow * cp.zw[1] + k0 - cp.zbase[1];
  return s;
}

// L2 prefetch of one CTA's slice of an x-plane for the H / E update, issued
// by thread 0 of the CTA, whose chunk is the first of the slice: o is that
// thread's offset in the plane to prefetch, tn the slice length in floats.
template <int kIdBytes>
__device__ __forceinline__ void prefetch_h_plane(const HArgs& a, long long o, long long tn) {
  const long long lim = (long long)a.g.nx * a.g.plane;
  l2_prefetch(a.ex, o, tn + a.g.nzp, lim);
  l2_prefetch(a.ey, o, tn, lim);
  l2_prefetch(a.ez, o, tn + a.g.nzp, lim);
  l2_prefetch(a.hx, o, tn, lim);
  l2_prefetch(a.hy, o, tn, lim);
  l2_prefetch(a.hz, o, tn, lim);
  if constexpr (kIdBytes == 0)
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      l2_prefetch(a.da[c], o, tn, lim);
      l2_prefetch(a.db[c], o, tn, lim);
    }
}

template <int kIdBytes>
__device__ __forceinline__ void prefetch_e_plane(const EArgs& a, long long o, long long tn) {
  const long long lim = (long long)a.g.nx * a.g.plane;
  l2_prefetch(a.hx, o - a.g.nzp, tn + a.g.nzp, lim);
  l2_prefetch(a.hy, o, tn, lim);
  l2_prefetch(a.hz, o - a.g.nzp, tn + a.g.nzp, lim);
  l2_prefetch(a.ex, o, tn, lim);
  l2_prefetch(a.ey, o, tn, lim);
  l2_prefetch(a.ez, o, tn, lim);
  if constexpr (kIdBytes == 0)
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      l2_prefetch(a.ca[c], o, tn, lim);
      l2_prefetch(a.cb[c], o, tn, lim);
    }
}

// H half-step of one work item w of a.g: H = da*H + db*curl(E).  T: field
// storage type.  Every thread of the CTA calls it with the same w.
template <int kIdBytes, bool kCpml, typename T>
__device__ __forceinline__ void h_item(const HArgs& a, const float* tab, int w) {
  using IO = FieldIO<T>;
  const Geom& g = a.g;
  const int lane = threadIdx.x & 31;
  {
    const Item it = work_item(g, w);
    int c = it.c0 + (int)threadIdx.x;
    const bool valid = c < it.c1;
    if (!valid) c = it.c1 - 1;
    const int jr = c / it.w;
    const int qr = c - jr * it.w;
    const int j = it.j0 + jr;
    const int k0 = (it.q0 + qr) * 4;
    const int i0 = it.i0;
    const int i1 = it.i1;
    const bool has_jp = j + 1 < g.ny;
    // the next chunk comes from lane + 1 unless this lane ends the warp or
    // its segment's part of the row
    const bool need_kn = (lane == 31 || qr == it.w - 1) && k0 + 4 < g.nz;
    unsigned live = 0;
#pragma unroll
    for (int e = 0; e < 4; ++e) live |= (k0 + e < g.nz ? 1u : 0u) << e;
    long long q = (long long)i0 * g.plane + (long long)j * g.nzp + k0;
    if (IO::kFloat && g.pf > 0 && it.whole && threadIdx.x == 0) {
      const long long tn = (long long)(it.c1 - it.c0) * 4;
      for (int p = 0; p < min(g.pf, i1 - i0); ++p) prefetch_h_plane<kIdBytes>(a, q + p * g.plane, tn);
    }
    float4 ey4 = IO::ldg4(a.ey, q);
    float4 ez4 = IO::ldg4(a.ez, q);
    for (int i = i0; i < i1; ++i, q += g.plane) {
      const bool has_ip = i + 1 < g.nx;
      if (IO::kFloat && g.pf > 0 && it.whole && threadIdx.x == 0 && i + g.pf < i1)
        prefetch_h_plane<kIdBytes>(a, q + g.pf * g.plane, (long long)(it.c1 - it.c0) * 4);
      // ---- every load of this plane first
      const float4 ex4 = IO::ldg4(a.ex, q);
      const float4 ey1 = has_ip ? IO::ldg4(a.ey, q + g.plane) : ey4;
      const float4 ez1 = has_ip ? IO::ldg4(a.ez, q + g.plane) : ez4;
      const float4 exj = has_jp ? IO::ldg4(a.ex, q + g.nzp) : ex4;
      const float4 ezj = has_jp ? IO::ldg4(a.ez, q + g.nzp) : ez4;
      const float exn_m = need_kn ? IO::ldg1(a.ex, q + 4) : 0.f;
      const float eyn_m = need_kn ? IO::ldg1(a.ey, q + 4) : 0.f;
      float co_a[3][4], co_b[3][4], h[3][4];
      Coef<kIdBytes>::load(a.da, a.ids, tab, 6, q, co_a);
      Coef<kIdBytes>::load(a.db, a.ids, tab, 9, q, co_b);
      to_arr(IO::ld4(a.hx, q), h[0]);
      to_arr(IO::ld4(a.hy, q), h[1]);
      to_arr(IO::ld4(a.hz, q), h[2]);
      SlabInfo sl;
      float4 px0, px1, py0, py1, pzn0, pzn1, pzx0, pzx1;
      if constexpr (kCpml) {
        sl = slab_info(a.cp, g, i, j, k0);
        px0 = sl.fx >= 0 ? ld4(a.cp.psi_h[sl.fx][0] + sl.px) : zero4();
        px1 = sl.fx >= 0 ? ld4(a.cp.psi_h[sl.fx][1] + sl.px) : zero4();
        py0 = sl.fy >= 0 ? ld4(a.cp.psi_h[sl.fy][0] + sl.py) : zero4();
        py1 = sl.fy >= 0 ? ld4(a.cp.psi_h[sl.fy][1] + sl.py) : zero4();
        pzn0 = sl.zmin ? ld4(a.cp.psi_h[4][0] + sl.pz0) : zero4();
        pzn1 = sl.zmin ? ld4(a.cp.psi_h[4][1] + sl.pz0) : zero4();
        pzx0 = sl.zmax ? ld4(a.cp.psi_h[5][0] + sl.pz1) : zero4();
        pzx1 = sl.zmax ? ld4(a.cp.psi_h[5][1] + sl.pz1) : zero4();
      }
      // ---- neighbours along z: first element of the next chunk (k0 + 4)
      float exn = __shfl_down_sync(kFullMask, ex4.x, 1);
      float eyn = __shfl_down_sync(kFullMask, ey4.x, 1);
      if (need_kn) {
        exn = exn_m;
        eyn = eyn_m;
      }
      float ex[4], ey[4], ez[4], eyp[4], ezp[4], exjv[4], ezjv[4];
      to_arr(ex4, ex);
      to_arr(ey4, ey);
      to_arr(ez4, ez);
      to_arr(ey1, eyp);
      to_arr(ez1, ezp);
      to_arr(exj, exjv);
      to_arr(ezj, ezjv);
      const float exk[4] = {ex[1], ex[2], ex[3], exn};
      const float eyk[4] = {ey[1], ey[2], ey[3], eyn};
      float dez_dy[4], dey_dz[4], dex_dz[4], dez_dx[4], dey_dx[4], dex_dy[4];
#pragma unroll
      for (int e = 0; e < 4; ++e) {
        const bool has_kp = k0 + e + 1 < g.nz;
        dez_dy[e] = has_jp ? __fsub_rn(ezjv[e], ez[e]) : 0.f;
        dey_dz[e] = has_kp ? __fsub_rn(eyk[e], ey[e]) : 0.f;
        dex_dz[e] = has_kp ? __fsub_rn(exk[e], ex[e]) : 0.f;
        dez_dx[e] = has_ip ? __fsub_rn(ezp[e], ez[e]) : 0.f;
        dey_dx[e] = has_ip ? __fsub_rn(eyp[e], ey[e]) : 0.f;
        dex_dy[e] = has_jp ? __fsub_rn(exjv[e], ex[e]) : 0.f;
      }
      if constexpr (kCpml) {
        float b, cc, ik;
        // y-slab: Hx (dEz/dy, slot 0), Hz (dEx/dy, slot 1)
        if (sl.fy >= 0) {
          cpml_prof(a.cp, sl.fy, sl.ly, true, b, cc, ik);
          stretch_vec(dez_dy, py0, b, cc, ik, live);
          stretch_vec(dex_dy, py1, b, cc, ik, live);
        }
        // z-slab: Hx (dEy/dz, slot 0), Hy (dEx/dz, slot 1)
        if (sl.zmin) {
          stretch_z(a.cp, 4, k0, true, dey_dz, pzn0, live);
          stretch_z(a.cp, 4, k0, true, dex_dz, pzn1, live);
        }
        if (sl.zmax) {
          stretch_z(a.cp, 5, k0, true, dey_dz, pzx0, live);
          stretch_z(a.cp, 5, k0, true, dex_dz, pzx1, live);
        }
        // x-slab: Hy (dEz/dx, slot 0), Hz (dEy/dx, slot 1)
        if (sl.fx >= 0) {
          cpml_prof(a.cp, sl.fx, sl.lx, true, b, cc, ik);
          stretch_vec(dez_dx, px0, b, cc, ik, live);
          stretch_vec(dey_dx, px1, b, cc, ik, live);
        }
      }
      float out[3][4];
#pragma unroll
      for (int e = 0; e < 4; ++e) {
        const float curl[3] = {__fsub_rn(dez_dy[e], dey_dz[e]), __fsub_rn(dex_dz[e], dez_dx[e]),
                               __fsub_rn(dey_dx[e], dex_dy[e])};
        const bool lv = (live >> e) & 1u;
#pragma unroll
        for (int cc = 0; cc < 3; ++cc) {
          const float v = __fadd_rn(__fmul_rn(co_a[cc][e], h[cc][e]), __fmul_rn(co_b[cc][e], curl[cc]));
          out[cc][e] = lv ? v : h[cc][e];
        }
      }
      if (valid) {
        IO::st4(a.hx, q, to_f4(out[0]));
        IO::st4(a.hy, q, to_f4(out[1]));
        IO::st4(a.hz, q, to_f4(out[2]));
        if constexpr (kCpml) {
          if (sl.fy >= 0) {
            st4(a.cp.psi_h[sl.fy][0] + sl.py, py0);
            st4(a.cp.psi_h[sl.fy][1] + sl.py, py1);
          }
          if (sl.zmin) {
            st4(a.cp.psi_h[4][0] + sl.pz0, pzn0);
            st4(a.cp.psi_h[4][1] + sl.pz0, pzn1);
          }
          if (sl.zmax) {
            st4(a.cp.psi_h[5][0] + sl.pz1, pzx0);
            st4(a.cp.psi_h[5][1] + sl.pz1, pzx1);
          }
          if (sl.fx >= 0) {
            st4(a.cp.psi_h[sl.fx][0] + sl.px, px0);
            st4(a.cp.psi_h[sl.fx][1] + sl.px, px1);
          }
        }
      }
      ey4 = ey1;
      ez4 = ez1;
    }
  }
}

// H half-step over the grid: CTAs loop over the work items.
template <int kIdBytes, bool kCpml, typename T = float>
__global__ void __launch_bounds__(512) k_update_h(const HArgs a) {
  extern __shared__ float s_table[];
  const float* tab = stage_table<kIdBytes>(a.table, a.ntable, s_table);
  for (int w = blockIdx.x; w < a.g.work; w += gridDim.x) h_item<kIdBytes, kCpml, T>(a, tab, w);
}

// E half-step of one work item w of a.g: E = ca*E + cb*curl(H), cells with
// i, j, k >= 1 only.  T: field storage type.
template <int kIdBytes, bool kCpml, typename T>
__device__ __forceinline__ void e_item(const EArgs& a, const float* tab, int w) {
  using IO = FieldIO<T>;
  const Geom& g = a.g;
  const int lane = threadIdx.x & 31;
  {
    const Item it = work_item(g, w);
    int c = it.c0 + (int)threadIdx.x;
    const bool valid = c < it.c1;
    if (!valid) c = it.c1 - 1;
    const int jr = c / it.w;
    const int qr = c - jr * it.w;
    const int j = it.j0 + jr;
    const int k0 = (it.q0 + qr) * 4;
    const int i0 = it.i0;
    const int i1 = it.i1;
    const bool has_jm = j >= 1;
    // the previous chunk comes from lane - 1 unless this lane starts the
    // warp or its segment's part of the row
    const bool need_km = (lane == 0 || qr == 0) && k0 >= 4;
    // elements that are updated: 1 <= k < nz (i >= 1 and j >= 1 checked per plane)
    unsigned live_k = 0;
#pragma unroll
    for (int e = 0; e < 4; ++e) live_k |= (k0 + e >= 1 && k0 + e < g.nz ? 1u : 0u) << e;
    long long q = (long long)i0 * g.plane + (long long)j * g.nzp + k0;
    if (IO::kFloat && g.pf > 0 && it.whole && threadIdx.x == 0) {
      const long long tn = (long long)(it.c1 - it.c0) * 4;
      for (int p = 0; p < min(g.pf, i1 - i0); ++p) prefetch_e_plane<kIdBytes>(a, q + p * g.plane, tn);
    }
    float4 hym4 = zero4(), hzm4 = zero4();  // H at i-1
    if (i0 > 0) {
      hym4 = IO::ldg4(a.hy, q - g.plane);
      hzm4 = IO::ldg4(a.hz, q - g.plane);
    }
    for (int i = i0; i < i1; ++i, q += g.plane) {
      if (IO::kFloat && g.pf > 0 && it.whole && threadIdx.x == 0 && i + g.pf < i1)
        prefetch_e_plane<kIdBytes>(a, q + g.pf * g.plane, (long long)(it.c1 - it.c0) * 4);
      const bool upd = i >= 1 && has_jm;
      const unsigned live = upd ? live_k : 0u;
      // ---- every load of this plane first
      const float4 hx4 = IO::ldg4(a.hx, q);
      const float4 hy4 = IO::ldg4(a.hy, q);
      const float4 hz4 = IO::ldg4(a.hz, q);
      const float4 hxj4 = upd ? IO::ldg4(a.hx, q - g.nzp) : zero4();
      const float4 hzj4 = upd ? IO::ldg4(a.hz, q - g.nzp) : zero4();
      const float hxm_m = need_km ? IO::ldg1(a.hx, q - 1) : 0.f;
      const float hym_m = need_km ? IO::ldg1(a.hy, q - 1) : 0.f;
      float co_a[3][4], co_b[3][4], ev[3][4];
      if (upd) {
        Coef<kIdBytes>::load(a.ca, a.ids, tab, 0, q, co_a);
        Coef<kIdBytes>::load(a.cb, a.ids, tab, 3, q, co_b);
        to_arr(IO::ld4(a.ex, q), ev[0]);
        to_arr(IO::ld4(a.ey, q), ev[1]);
        to_arr(IO::ld4(a.ez, q), ev[2]);
      }
      SlabInfo sl;
      float4 px0, px1, py0, py1, pzn0, pzn1, pzx0, pzx1;
      if constexpr (kCpml) {
        sl = slab_info(a.cp, g, i, j, k0);
        if (!upd) {
          sl.fx = sl.fy = -1;
          sl.zmin = sl.zmax = false;
        }
        px0 = sl.fx >= 0 ? ld4(a.cp.psi_e[sl.fx][0] + sl.px) : zero4();
        px1 = sl.fx >= 0 ? ld4(a.cp.psi_e[sl.fx][1] + sl.px) : zero4();
        py0 = sl.fy >= 0 ? ld4(a.cp.psi_e[sl.fy][0] + sl.py) : zero4();
        py1 = sl.fy >= 0 ? ld4(a.cp.psi_e[sl.fy][1] + sl.py) : zero4();
        pzn0 = sl.zmin ? ld4(a.cp.psi_e[4][0] + sl.pz0) : zero4();
        pzn1 = sl.zmin ? ld4(a.cp.psi_e[4][1] + sl.pz0) : zero4();
        pzx0 = sl.zmax ? ld4(a.cp.psi_e[5][0] + sl.pz1) : zero4();
        pzx1 = sl.zmax ? ld4(a.cp.psi_e[5][1] + sl.pz1) : zero4();
      }
      // ---- neighbours along z: last element of the previous chunk (k0 - 1)
      float hxm = __shfl_up_sync(kFullMask, hx4.w, 1);
      float hym = __shfl_up_sync(kFullMask, hy4.w, 1);
      if (need_km) {
        hxm = hxm_m;
        hym = hym_m;
      }
      if (upd) {
        float hx[4], hy[4], hz[4], hxj[4], hzj[4], hyi[4], hzi[4];
        to_arr(hx4, hx);
        to_arr(hy4, hy);
        to_arr(hz4, hz);
        to_arr(hxj4, hxj);
        to_arr(hzj4, hzj);
        to_arr(hym4, hyi);
        to_arr(hzm4, hzi);
        const float hxk[4] = {hxm, hx[0], hx[1], hx[2]};
        const float hyk[4] = {hym, hy[0], hy[1], hy[2]};
        float dhz_dy[4], dhy_dz[4], dhx_dz[4], dhz_dx[4], dhy_dx[4], dhx_dy[4];
#pragma unroll
        for (int e = 0; e < 4; ++e) {
          dhz_dy[e] = __fsub_rn(hz[e], hzj[e]);
          dhy_dz[e] = __fsub_rn(hy[e], hyk[e]);
          dhx_dz[e] = __fsub_rn(hx[e], hxk[e]);
          dhz_dx[e] = __fsub_rn(hz[e], hzi[e]);
          dhy_dx[e] = __fsub_rn(hy[e], hyi[e]);
          dhx_dy[e] = __fsub_rn(hx[e], hxj[e]);
        }
        if constexpr (kCpml) {
          float b, cc, ik;
          // y-slab: Ex (dHz/dy, slot 0), Ez (dHx/dy, slot 1)
          if (sl.fy >= 0) {
            cpml_prof(a.cp, sl.fy, sl.ly, false, b, cc, ik);
            stretch_vec(dhz_dy, py0, b, cc, ik, live);
            stretch_vec(dhx_dy, py1, b, cc, ik, live);
          }
          // z-slab: Ex (dHy/dz, slot 0), Ey (dHx/dz, slot 1)
          if (sl.zmin) {
            stretch_z(a.cp, 4, k0, false, dhy_dz, pzn0, live);
            stretch_z(a.cp, 4, k0, false, dhx_dz, pzn1, live);
          }
          if (sl.zmax) {
            stretch_z(a.cp, 5, k0, false, dhy_dz, pzx0, live);
            stretch_z(a.cp, 5, k0, false, dhx_dz, pzx1, live);
          }
          // x-slab: Ey (dHz/dx, slot 0), Ez (dHy/dx, slot 1)
          if (sl.fx >= 0) {
            cpml_prof(a.cp, sl.fx, sl.lx, false, b, cc, ik);
            stretch_vec(dhz_dx, px0, b, cc, ik, live);
            stretch_vec(dhy_dx, px1, b, cc, ik, live);
          }
        }
        float out[3][4];
#pragma unroll
        for (int e = 0; e < 4; ++e) {
          const float curl[3] = {__fsub_rn(dhz_dy[e], dhy_dz[e]), __fsub_rn(dhx_dz[e], dhz_dx[e]),
                                 __fsub_rn(dhy_dx[e], dhx_dy[e])};
          const bool lv = (live >> e) & 1u;
#pragma unroll
          for (int cc = 0; cc < 3; ++cc) {
            const float v = __fadd_rn(__fmul_rn(co_a[cc][e], ev[cc][e]), __fmul_rn(co_b[cc][e], curl[cc]));
            out[cc][e] = lv ? v : ev[cc][e];
          }
        }
        if (valid) {
          IO::st4(a.ex, q, to_f4(out[0]));
          IO::st4(a.ey, q, to_f4(out[1]));
          IO::st4(a.ez, q, to_f4(out[2]));
          if constexpr (kCpml) {
            if (sl.fy >= 0) {
              st4(a.cp.psi_e[sl.fy][0] + sl.py, py0);
              st4(a.cp.psi_e[sl.fy][1] + sl.py, py1);
            }
            if (sl.zmin) {
              st4(a.cp.psi_e[4][0] + sl.pz0, pzn0);
              st4(a.cp.psi_e[4][1] + sl.pz0, pzn1);
            }
            if (sl.zmax) {
              st4(a.cp.psi_e[5][0] + sl.pz1, pzx0);
              st4(a.cp.psi_e[5][1] + sl.pz1, pzx1);
            }
            if (sl.fx >= 0) {
              st4(a.cp.psi_e[sl.fx][0] + sl.px, px0);
              st4(a.cp.psi_e[sl.fx][1] + sl.px, px1);
            }
          }
        }
      }
      hym4 = hy4;
      hzm4 = hz4;
    }
  }
}

// E half-step over the grid: CTAs loop over the work items.
template <int kIdBytes, bool kCpml, typename T = float>
__global__ void __launch_bounds__(512) k_update_e(const EArgs a) {
  extern __shared__ float s_table[];
  const float* tab = stage_table<kIdBytes>(a.table, a.ntable, s_table);
  for (int w = blockIdx.x; w < a.g.work; w += gridDim.x) e_item<kIdBytes, kCpml, T>(a, tab, w);
}

// The same kernels (float fields, full coefficient arrays) with a capped
// register budget: 256-thread CTAs, kMinBlocks of them resident per SM
// (3: <= 85 registers, 4: <= 64), spilling what does not fit, which trades
// spills for more warps to hide the loads' latency.  The autotuner times
// them against the uncapped kernels.
template <bool kCpml, int kMinBlocks>
__global__ void __launch_bounds__(256, kMinBlocks) k_update_h_cap(const HArgs a) {
  for (int w = blockIdx.x; w < a.g.work; w += gridDim.x) h_item<0, kCpml, float>(a, nullptr, w);
}
template <bool kCpml, int kMinBlocks>
__global__ void __launch_bounds__(256, kMinBlocks) k_update_e_cap(const EArgs a) {
  for (int w = blockIdx.x; w < a.g.work; w += gridDim.x) e_item<0, kCpml, float>(a, nullptr, w);
}

// Several grids in one launch (independent instances of a sweep): part p of
// the launch is one grid's update over one geometry (its interior or its
// CPML shell), args[p] its arguments in device memory, its work items
// numbered from off[p]; off[nparts] is the total.  Every part uses the
// launch's block size and full coefficient arrays.
struct PackH {
  int nparts;
  const int* off;
  const HArgs* args;
};
struct PackE {
  int nparts;
  const int* off;
  const EArgs* args;
};

// Part holding global work item w: the last p with off[p] <= w.
__device__ __forceinline__ int pack_part(const int* off, int nparts, int w) {
  int lo = 0, hi = nparts - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (__ldg(off + mid) <= w)
      lo = mid;
    else
      hi = mid - 1;
  }
  return lo;
}

// The arguments of the CTA's current part are staged in shared memory:
// read through a reference into global memory, every field would be
// re-read after each of the kernel's global stores (the compiler cannot
// rule out aliasing), in the innermost loops.
template <typename A>
__device__ __forceinline__ void stage_args(A& dst, const A* src) {
  static_assert(sizeof(A) % 4 == 0, "argument block of whole words");
  __syncthreads();  // every thread is done with the previous part's arguments
  const int* s = reinterpret_cast<const int*>(src);
  int* d = reinterpret_cast<int*>(&dst);
  for (int t = threadIdx.x; t < (int)(sizeof(A) / 4); t += blockDim.x) d[t] = __ldg(s + t);
  __syncthreads();
}

template <bool kCpml, typename T = float>
__global__ void __launch_bounds__(512) k_update_h_pack(const PackH p) {
  __shared__ __align__(16) HArgs sa;
  int cur = -1;
  const int total = __ldg(p.off + p.nparts);
  for (int w = blockIdx.x; w < total; w += gridDim.x) {
    const int q = pack_part(p.off, p.nparts, w);
    if (q != cur) {
      stage_args(sa, p.args + q);
      cur = q;
    }
    h_item<0, kCpml, T>(sa, nullptr, w - __ldg(p.off + q));
  }
}

template <bool kCpml, typename T = float>
__global__ void __launch_bounds__(512) k_update_e_pack(const PackE p) {
  __shared__ __align__(16) EArgs sa;
  int cur = -1;
  const int total = __ldg(p.off + p.nparts);
  for (int w = blockIdx.x; w < total; w += gridDim.x) {
    const int q = pack_part(p.off, p.nparts, w);
    if (q != cur) {
      stage_args(sa, p.args + q);
      cur = q;
    }
    e_item<0, kCpml, T>(sa, nullptr, w - __ldg(p.off + q));
  }
}

}  // namespace oems
