// yee_tma.cuh -- Yee update kernels with bulk-async (TMA) staging of planes.
//
// Same arithmetic and semantics as yee_kernels.cuh (bit-identical results);
// only the data movement differs.  A CTA owns a tile of TJ rows (j) x all of
// z and walks its work items (tile, run of x-planes) in order.  One producer
// warp streams "plane bundles" from HBM into a ring of NS shared-memory stages
// with cp.async.bulk (one contiguous copy per array: the rows j0..j0+TJ of one
// x-plane are contiguous in the z-fastest layout), each stage completed by an
// mbarrier transaction count.  Consumer warps compute one plane from the
// bundle of that plane plus the neighbouring plane's bundle (the x-neighbour),
// read z- and y-neighbours from shared memory, write results straight to HBM
// with 128-bit stores, then release the stage.  Nothing in flight occupies
// registers, so a CTA keeps two or more planes of every operand in flight with
// only nine warps.  The producer runs across work-item boundaries, so the
// pipeline never drains between items.  No multicast is used anywhere.
//
// Bundle contents (H kernel, plane p):
//   F: Ex Ey Ez rows j0 .. j0+TJ (TJ+1 rows: row j+1 for the y-difference)
//   U: Hx Hy Hz rows j0 .. j0+TJ-1
//   C: da0..2 db0..2 rows j0 .. j0+TJ-1
//   CPML psi rows when the plane / rows / z-ends are in a slab
// An E-only bundle for plane i1 closes each work item (x-neighbour of its last
// plane).  E kernel: F holds Hx Hy Hz rows j0-1 .. j0+TJ-1 (row j-1), U holds
// Ex Ey Ez, C holds ca cb; an H-only bundle for plane i0-1 opens each item.
//
// Every wait on an mbarrier is bounded (about one second of clock64 cycles);
// on timeout the CTA sets the engine's error word, stops, and the host
// reports OEMS_ERR_TIMEOUT.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "yee_kernels.cuh"

namespace oems {

struct TmaGeom {
  int TJ;            // rows per tile
  int ntiles;        // ceil((j_hi - j_lo) / TJ)
  int ichunk;        // x-planes per work item
  int nitems;        // ntiles * ceil((i_hi - i_lo) / ichunk)
  int i_lo, i_hi;    // x-planes updated (the whole grid, or the interior
  int j_lo, j_hi;    // box between the x and y CPML slabs)
  int xy_psi;        // stages hold x / y slab psi rows
  int NS;            // pipeline stages
  int stage_floats;  // floats per stage (multiple of 4)
  int off_f, off_u, off_c, off_px, off_py, off_pz;  // float offsets inside a stage
  int zwmax;         // max z-slab psi row width
  int nconsumer;     // consumer threads (multiple of 32)
  int prof_floats;   // CPML profile floats staged in shared memory
};

struct TmaArgs {
  Geom g;
  TmaGeom t;
  const float* f[3];  // neighbour-read fields (E for the H kernel, H for the E kernel)
  float* u[3];        // updated fields
  const float* c[6];  // coefficients: H kernel da0..2 db0..2, E kernel ca0..2 cb0..2
  CpmlArgs cp;
  bool cpml;
  int* err;           // error word (timeouts)
};

// ---- PTX wrappers -----------------------------------------------------------

__device__ __forceinline__ uint32_t smem_addr(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(bar)), "r"(count) : "memory");
}

__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(bar)), "r"(bytes)
               : "memory");
}

__device__ __forceinline__ void mbar_arrive(uint64_t* bar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_addr(bar)) : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}"
      : "=r"(ok)
      : "r"(smem_addr(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}

// 1-D bulk copy global -> shared, completing `bytes` on `bar`.  Both addresses
// 16-byte aligned, bytes a multiple of 16 (guaranteed by the nzp padding).
__device__ __forceinline__ void bulk_g2s(void* dst, const void* src, uint32_t bytes, uint64_t* bar) {
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
          smem_addr(dst)),
      "l"(src), "r"(bytes), "r"(smem_addr(bar))
      : "memory");
}

constexpr long long kWaitCycles = 2000000000LL;  // ~1 s at 2 GHz

// Bounded wait.  Returns false (and sets *err) when the wait gives up or when
// another warp already gave up.
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity, int* err) {
  if (mbar_try_wait(bar, parity)) return true;
  const long long t0 = clock64();
  while (true) {
    if (mbar_try_wait(bar, parity)) return true;
    if (*reinterpret_cast<volatile int*>(err) != 0) return false;
    if (clock64() - t0 > kWaitCycles) {
      atomicExch(err, 1);
      return false;
    }
  }
}

// ---- bundle sequence ------------------------------------------------------------

// Bundle kinds: full plane, neighbour-only (F arrays) plane.
enum : int { kFull = 0, kFOnly = 1 };

// Issues the copies of one bundle; returns the byte count (the caller arms
// the barrier with it first, so it is computed before any copy is issued).
template <bool kIsH>
__device__ __forceinline__ uint32_t bundle_bytes_or_issue(const TmaArgs& a, int tile, int p, int kind, float* st,
                                                          uint64_t* bar, bool issue) {
  const Geom& g = a.g;
  const TmaGeom& t = a.t;
  const int j0 = t.j_lo + tile * t.TJ;
  const int rows_u = min(t.TJ, t.j_hi - j0);
  const size_t rowb = (size_t)g.nzp * sizeof(float);
  uint32_t bytes = 0;
  // F arrays: H kernel rows j0..j0+rows_u (+1 if it exists); E kernel rows j0-1..j0+rows_u-1.
  int fr0, frn, fdst;
  if (kIsH) {
    fr0 = j0;
    frn = min(t.TJ + 1, g.ny - j0);
    fdst = 0;
  } else {
    fr0 = j0 > 0 ? j0 - 1 : 0;
    frn = rows_u + (j0 > 0 ? 1 : 0);
    fdst = j0 > 0 ? 0 : 1;
  }
  const long long plane_off = (long long)p * g.plane;
  for (int c = 0; c < 3; ++c) {
    const uint32_t nb = (uint32_t)(frn * rowb);
    if (issue)
      bulk_g2s(st + t.off_f + (c * (t.TJ + 1) + fdst) * g.nzp, a.f[c] + plane_off + (long long)fr0 * g.nzp, nb, bar);
    bytes += nb;
  }
  if (kind == kFOnly) return bytes;
  const uint32_t nbu = (uint32_t)(rows_u * rowb);
  const long long q0 = plane_off + (long long)j0 * g.nzp;
  for (int c = 0; c < 3; ++c) {
    if (issue) bulk_g2s(st + t.off_u + c * t.TJ * g.nzp, a.u[c] + q0, nbu, bar);
    bytes += nbu;
  }
  for (int c = 0; c < 6; ++c) {
    if (issue) bulk_g2s(st + t.off_c + c * t.TJ * g.nzp, a.c[c] + q0, nbu, bar);
    bytes += nbu;
  }
  if (a.cpml) {
    const CpmlArgs& cp = a.cp;
    float* const* psi = kIsH ? &cp.psi_h[0][0] : &cp.psi_e[0][0];  // [face*2 + slot]
    // x slab: whole plane rows j0..j0+rows_u
    int lx;
    const int fx = t.xy_psi ? cpml_face(cp, 0, p, lx) : -1;
    if (fx >= 0) {
      const long long src = ((long long)lx * g.ny + j0) * g.nzp;
      for (int s = 0; s < 2; ++s) {
        if (issue) bulk_g2s(st + t.off_px + s * t.TJ * g.nzp, psi[fx * 2 + s] + src, nbu, bar);
        bytes += nbu;
      }
    }
    // y slabs: rows of the tile inside each y face
    for (int f = 2; f < 4; ++f) {
      if (cp.L[f] == 0 || !t.xy_psi) continue;
      const int lo = max(j0, cp.start[f]), hi = min(j0 + rows_u, cp.start[f] + cp.L[f]);
      if (hi <= lo) continue;
      const uint32_t nb = (uint32_t)((hi - lo) * rowb);
      const long long src = ((long long)p * cp.L[f] + (lo - cp.start[f])) * g.nzp;
      for (int s = 0; s < 2; ++s) {
        if (issue) bulk_g2s(st + t.off_py + (s * t.TJ + (lo - j0)) * g.nzp, psi[f * 2 + s] + src, nb, bar);
        bytes += nb;
      }
    }
    // z slabs: rows j0..j0+rows_u of [i][j][zw]
    for (int f = 4; f < 6; ++f) {
      if (cp.L[f] == 0) continue;
      const int zw = cp.zw[f - 4];
      const uint32_t nb = (uint32_t)(rows_u * zw * sizeof(float));
      const long long src = ((long long)p * g.ny + j0) * zw;
      for (int s = 0; s < 2; ++s) {
        if (issue)
          bulk_g2s(st + t.off_pz + (((f - 4) * 2 + s) * t.TJ) * t.zwmax, psi[f * 2 + s] + src, nb, bar);
        bytes += nb;
      }
    }
  }
  return bytes;
}

// Visits the bundle sequence of this CTA: calls fn(tile, plane, kind) per bundle.
template <bool kIsH, typename Fn>
__device__ __forceinline__ void for_each_bundle(const TmaArgs& a, Fn&& fn) {
  const Geom& g = a.g;
  const TmaGeom& t = a.t;
  for (int w = blockIdx.x; w < t.nitems; w += gridDim.x) {
    const int chunk = w / t.ntiles, tile = w % t.ntiles;
    const int i0 = t.i_lo + chunk * t.ichunk, i1 = min(i0 + t.ichunk, t.i_hi);
    if (kIsH) {
      for (int p = i0; p < i1; ++p)
        if (!fn(tile, p, kFull)) return;
      if (i1 < g.nx && !fn(tile, i1, kFOnly)) return;
    } else {
      if (i0 > 0 && !fn(tile, i0 - 1, kFOnly)) return;
      for (int p = i0; p < i1; ++p)
        if (!fn(tile, p, kFull)) return;
    }
  }
}

__device__ __forceinline__ float4 lds4(const float* p) { return *reinterpret_cast<const float4*>(p); }

// Profile row (b, c, ik) from the shared-memory copy of the CPML profile.
__device__ __forceinline__ void sprof(const CpmlArgs& cp, const float* sp, int f, int l, bool is_h, float& b,
                                      float& c, float& ik) {
  const int L = cp.L[f];
  const float* pr = sp + cp.prof_off[f] + (is_h ? 3 * L : 0);
  b = pr[l];
  c = pr[L + l];
  ik = pr[2 * L + l];
}

__device__ __forceinline__ void stretch_vec_s(float (&d)[4], float (&p)[4], float b, float c, float ik,
                                              unsigned live) {
#pragma unroll
  for (int e = 0; e < 4; ++e) {
    if (live & (1u << e)) {
      float pe = p[e];
      d[e] = cpml_stretch(d[e], pe, b, c, ik);
      p[e] = pe;
    }
  }
}

__device__ __forceinline__ void stretch_z_s(const CpmlArgs& cp, const float* sp, int f, int k0, bool is_h,
                                            float (&d)[4], float (&p)[4], unsigned live) {
#pragma unroll
  for (int e = 0; e < 4; ++e) {
    const int l = k0 + e - cp.start[f];
    if ((live & (1u << e)) && l >= 0 && l < cp.L[f]) {
      float b, c, ik;
      sprof(cp, sp, f, l, is_h, b, c, ik);
      float pe = p[e];
      d[e] = cpml_stretch(d[e], pe, b, c, ik);
      p[e] = pe;
    }
  }
}

// One plane of the H update for the chunks of a tile.  cur: bundle of plane
// i; nxt: bundle of plane i+1 (F arrays), or null at the last plane.
__device__ __forceinline__ void h_plane(const TmaArgs& a, const float* sprof_, const float* cur, const float* nxt,
                                        int tile, int i, int ctid) {
  const Geom& g = a.g;
  const TmaGeom& t = a.t;
  const int j0 = t.j_lo + tile * t.TJ;
  const int rows_u = min(t.TJ, t.j_hi - j0);
  const int nchunk = rows_u * g.nzq;
  const int FS = (t.TJ + 1) * g.nzp;  // F array stride
  const int US = t.TJ * g.nzp;        // U / C array stride
  const bool has_ip = nxt != nullptr;
  int lx = 0;
  const int fx = a.cpml ? cpml_face(a.cp, 0, i, lx) : -1;
  for (int cidx = ctid; cidx < nchunk; cidx += t.nconsumer) {
    const int r = cidx / g.nzq;
    const int k0 = (cidx - r * g.nzq) * 4;
    const int j = j0 + r;
    const bool has_jp = j + 1 < g.ny;
    const int so = r * g.nzp + k0;  // offset of this chunk in a TJ-row array
    const float* fx_ = cur + t.off_f;
    float ex[4], ey[4], ez[4], eyp[4], ezp[4], exj[4], ezj[4];
    to_arr(lds4(fx_ + so), ex);
    to_arr(lds4(fx_ + FS + so), ey);
    to_arr(lds4(fx_ + 2 * FS + so), ez);
    const float exn = k0 + 4 < g.nz ? fx_[so + 4] : 0.f;
    const float eyn = k0 + 4 < g.nz ? fx_[FS + so + 4] : 0.f;
    if (has_jp) {
      to_arr(lds4(fx_ + so + g.nzp), exj);
      to_arr(lds4(fx_ + 2 * FS + so + g.nzp), ezj);
    }
    if (has_ip) {
      to_arr(lds4(nxt + t.off_f + FS + so), eyp);
      to_arr(lds4(nxt + t.off_f + 2 * FS + so), ezp);
    }
    unsigned live = 0;
#pragma unroll
    for (int e = 0; e < 4; ++e) live |= (k0 + e < g.nz ? 1u : 0u) << e;
    const float exk[4] = {ex[1], ex[2], ex[3], exn};
    const float eyk[4] = {ey[1], ey[2], ey[3], eyn};
    float dez_dy[4], dey_dz[4], dex_dz[4], dez_dx[4], dey_dx[4], dex_dy[4];
#pragma unroll
    for (int e = 0; e < 4; ++e) {
      const bool has_kp = k0 + e + 1 < g.nz;
      dez_dy[e] = has_jp ? __fsub_rn(ezj[e], ez[e]) : 0.f;
      dey_dz[e] = has_kp ? __fsub_rn(eyk[e], ey[e]) : 0.f;
      dex_dz[e] = has_kp ? __fsub_rn(exk[e], ex[e]) : 0.f;
      dez_dx[e] = has_ip ? __fsub_rn(ezp[e], ez[e]) : 0.f;
      dey_dx[e] = has_ip ? __fsub_rn(eyp[e], ey[e]) : 0.f;
      dex_dy[e] = has_jp ? __fsub_rn(exj[e], ex[e]) : 0.f;
    }
    const long long q = (long long)i * g.plane + (long long)j * g.nzp + k0;
    if (a.cpml) {
      const CpmlArgs& cp = a.cp;
      float b, cc, ik;
      int ly;
      const int fy = cpml_face(cp, 1, j, ly);
      if (fy >= 0) {
        float p0[4], p1[4];
        to_arr(lds4(cur + t.off_py + so), p0);
        to_arr(lds4(cur + t.off_py + US + so), p1);
        sprof(cp, sprof_, fy, ly, true, b, cc, ik);
        stretch_vec_s(dez_dy, p0, b, cc, ik, live);
        stretch_vec_s(dex_dy, p1, b, cc, ik, live);
        const long long pg = ((long long)i * cp.L[fy] + ly) * g.nzp + k0;
        st4(cp.psi_h[fy][0] + pg, to_f4(p0));
        st4(cp.psi_h[fy][1] + pg, to_f4(p1));
      }
      for (int f = 4; f < 6; ++f) {
        if (cp.L[f] == 0) continue;
        const bool in = f == 4 ? k0 < cp.L[4] : (k0 + 3 >= cp.start[5] && k0 < g.nz);
        if (!in) continue;
        const int zw = cp.zw[f - 4];
        const int zo = k0 - cp.zbase[f - 4];
        // [face][slot] regions of TJ * zwmax floats, rows packed with pitch zw
        const float* ps = cur + t.off_pz + (f - 4) * 2 * t.TJ * t.zwmax + r * zw + zo;
        float p0[4], p1[4];
        to_arr(lds4(ps), p0);
        to_arr(lds4(ps + t.TJ * t.zwmax), p1);
        stretch_z_s(cp, sprof_, f, k0, true, dey_dz, p0, live);
        stretch_z_s(cp, sprof_, f, k0, true, dex_dz, p1, live);
        const long long pg = ((long long)i * g.ny + j) * zw + zo;
        st4(cp.psi_h[f][0] + pg, to_f4(p0));
        st4(cp.psi_h[f][1] + pg, to_f4(p1));
      }
      if (fx >= 0) {
        float p0[4], p1[4];
        to_arr(lds4(cur + t.off_px + so), p0);
        to_arr(lds4(cur + t.off_px + US + so), p1);
        sprof(cp, sprof_, fx, lx, true, b, cc, ik);
        stretch_vec_s(dez_dx, p0, b, cc, ik, live);
        stretch_vec_s(dey_dx, p1, b, cc, ik, live);
        const long long pg = ((long long)lx * g.ny + j) * g.nzp + k0;
        st4(cp.psi_h[fx][0] + pg, to_f4(p0));
        st4(cp.psi_h[fx][1] + pg, to_f4(p1));
      }
    }
    float h[3][4], ca[3][4], cb[3][4];
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      to_arr(lds4(cur + t.off_u + c * US + so), h[c]);
      to_arr(lds4(cur + t.off_c + c * US + so), ca[c]);
      to_arr(lds4(cur + t.off_c + (3 + c) * US + so), cb[c]);
    }
    float out[3][4];
#pragma unroll
    for (int e = 0; e < 4; ++e) {
      const float curl[3] = {__fsub_rn(dez_dy[e], dey_dz[e]), __fsub_rn(dex_dz[e], dez_dx[e]),
                             __fsub_rn(dey_dx[e], dex_dy[e])};
      const bool lv = (live >> e) & 1u;
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        const float v = __fadd_rn(__fmul_rn(ca[c][e], h[c][e]), __fmul_rn(cb[c][e], curl[c]));
        out[c][e] = lv ? v : h[c][e];
      }
    }
#pragma unroll
    for (int c = 0; c < 3; ++c) st4(a.u[c] + q, to_f4(out[c]));
  }
}

// One plane of the E update.  cur: bundle of plane i; prv: bundle of plane
// i-1 (F arrays = H), null at i = 0 (plane 0 is never written).
__device__ __forceinline__ void e_plane(const TmaArgs& a, const float* sprof_, const float* cur, const float* prv,
                                        int tile, int i, int ctid) {
  const Geom& g = a.g;
  const TmaGeom& t = a.t;
  if (i == 0) return;
  const int j0 = t.j_lo + tile * t.TJ;
  const int rows_u = min(t.TJ, t.j_hi - j0);
  const int nchunk = rows_u * g.nzq;
  const int FS = (t.TJ + 1) * g.nzp;
  const int US = t.TJ * g.nzp;
  int lx = 0;
  const int fx = a.cpml ? cpml_face(a.cp, 0, i, lx) : -1;
  for (int cidx = ctid; cidx < nchunk; cidx += t.nconsumer) {
    const int r = cidx / g.nzq;
    const int k0 = (cidx - r * g.nzq) * 4;
    const int j = j0 + r;
    if (j == 0) continue;
    const int so = r * g.nzp + k0;
    const int fo = (r + 1) * g.nzp + k0;  // F arrays start one row earlier (row j-1)
    const float* fh = cur + t.off_f;
    float hx[4], hy[4], hz[4], hxj[4], hzj[4], hyi[4], hzi[4];
    to_arr(lds4(fh + fo), hx);
    to_arr(lds4(fh + FS + fo), hy);
    to_arr(lds4(fh + 2 * FS + fo), hz);
    to_arr(lds4(fh + fo - g.nzp), hxj);
    to_arr(lds4(fh + 2 * FS + fo - g.nzp), hzj);
    to_arr(lds4(prv + t.off_f + FS + fo), hyi);
    to_arr(lds4(prv + t.off_f + 2 * FS + fo), hzi);
    const float hxm = k0 >= 4 ? fh[fo - 1] : 0.f;
    const float hym = k0 >= 4 ? fh[FS + fo - 1] : 0.f;
    unsigned live = 0;
#pragma unroll
    for (int e = 0; e < 4; ++e) live |= (k0 + e >= 1 && k0 + e < g.nz ? 1u : 0u) << e;
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
    const long long q = (long long)i * g.plane + (long long)j * g.nzp + k0;
    if (a.cpml) {
      const CpmlArgs& cp = a.cp;
      float b, cc, ik;
      int ly;
      const int fy = cpml_face(cp, 1, j, ly);
      if (fy >= 0) {
        float p0[4], p1[4];
        to_arr(lds4(cur + t.off_py + so), p0);
        to_arr(lds4(cur + t.off_py + US + so), p1);
        sprof(cp, sprof_, fy, ly, false, b, cc, ik);
        stretch_vec_s(dhz_dy, p0, b, cc, ik, live);
        stretch_vec_s(dhx_dy, p1, b, cc, ik, live);
        const long long pg = ((long long)i * cp.L[fy] + ly) * g.nzp + k0;
        st4(cp.psi_e[fy][0] + pg, to_f4(p0));
        st4(cp.psi_e[fy][1] + pg, to_f4(p1));
      }
      for (int f = 4; f < 6; ++f) {
        if (cp.L[f] == 0) continue;
        const bool in = f == 4 ? k0 < cp.L[4] : (k0 + 3 >= cp.start[5] && k0 < g.nz);
        if (!in) continue;
        const int zw = cp.zw[f - 4];
        const int zo = k0 - cp.zbase[f - 4];
        // [face][slot] regions of TJ * zwmax floats, rows packed with pitch zw
        const float* ps = cur + t.off_pz + (f - 4) * 2 * t.TJ * t.zwmax + r * zw + zo;
        float p0[4], p1[4];
        to_arr(lds4(ps), p0);
        to_arr(lds4(ps + t.TJ * t.zwmax), p1);
        stretch_z_s(cp, sprof_, f, k0, false, dhy_dz, p0, live);
        stretch_z_s(cp, sprof_, f, k0, false, dhx_dz, p1, live);
        const long long pg = ((long long)i * g.ny + j) * zw + zo;
        st4(cp.psi_e[f][0] + pg, to_f4(p0));
        st4(cp.psi_e[f][1] + pg, to_f4(p1));
      }
      if (fx >= 0) {
        float p0[4], p1[4];
        to_arr(lds4(cur + t.off_px + so), p0);
        to_arr(lds4(cur + t.off_px + US + so), p1);
        sprof(cp, sprof_, fx, lx, false, b, cc, ik);
        stretch_vec_s(dhz_dx, p0, b, cc, ik, live);
        stretch_vec_s(dhy_dx, p1, b, cc, ik, live);
        const long long pg = ((long long)lx * g.ny + j) * g.nzp + k0;
        st4(cp.psi_e[fx][0] + pg, to_f4(p0));
        st4(cp.psi_e[fx][1] + pg, to_f4(p1));
      }
    }
    float ev[3][4], ca[3][4], cb[3][4];
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      to_arr(lds4(cur + t.off_u + c * US + so), ev[c]);
      to_arr(lds4(cur + t.off_c + c * US + so), ca[c]);
      to_arr(lds4(cur + t.off_c + (3 + c) * US + so), cb[c]);
    }
    float out[3][4];
#pragma unroll
    for (int e = 0; e < 4; ++e) {
      const float curl[3] = {__fsub_rn(dhz_dy[e], dhy_dz[e]), __fsub_rn(dhx_dz[e], dhz_dx[e]),
                             __fsub_rn(dhy_dx[e], dhx_dy[e])};
      const bool lv = (live >> e) & 1u;
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        const float v = __fadd_rn(__fmul_rn(ca[c][e], ev[c][e]), __fmul_rn(cb[c][e], curl[c]));
        out[c][e] = lv ? v : ev[c][e];
      }
    }
#pragma unroll
    for (int c = 0; c < 3; ++c) st4(a.u[c] + q, to_f4(out[c]));
  }
}

// Shared memory: [NS stages][stage_floats] | CPML profile | full[NS] empty[NS] barriers.
template <bool kIsH>
__global__ void __launch_bounds__(288, 1) k_update_tma(const TmaArgs a) {
  extern __shared__ __align__(128) float smem[];
  const TmaGeom& t = a.t;
  float* sprof_ = smem + (size_t)t.NS * t.stage_floats;
  uint64_t* full = reinterpret_cast<uint64_t*>(sprof_ + ((t.prof_floats + 3) / 4 * 4));
  uint64_t* empty = full + t.NS;
  const int warp = threadIdx.x >> 5;
  const int nwarps_c = t.nconsumer / 32;
  const bool producer = warp == nwarps_c;  // last warp produces
  if (threadIdx.x == 0) {
    for (int s = 0; s < t.NS; ++s) {
      mbar_init(&full[s], 1);
      mbar_init(&empty[s], nwarps_c);
    }
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (a.cpml)
    for (int x = threadIdx.x; x < t.prof_floats; x += blockDim.x) sprof_[x] = a.cp.prof[x];
  __syncthreads();

  if (producer) {
    if ((threadIdx.x & 31) != 0) return;
    int n = 0;  // bundle number
    bool ok = true;
    for_each_bundle<kIsH>(a, [&](int tile, int p, int kind) {
      const int s = n % t.NS;
      const uint32_t use = (uint32_t)(n / t.NS);
      if (use > 0 && !mbar_wait(&empty[s], (use - 1) & 1u, a.err)) {
        ok = false;
        return false;
      }
      float* st = smem + (size_t)s * t.stage_floats;
      const uint32_t bytes = bundle_bytes_or_issue<kIsH>(a, tile, p, kind, st, &full[s], false);
      mbar_expect_tx(&full[s], bytes);
      bundle_bytes_or_issue<kIsH>(a, tile, p, kind, st, &full[s], true);
      ++n;
      return true;
    });
    // drain: wait (bounded) for the copies this thread issued into stages that
    // no consumer will read any more, so no copy is in flight at exit
    if (!ok || *reinterpret_cast<volatile int*>(a.err) != 0) {
      for (int m = max(0, n - t.NS); m < n; ++m) {
        const int s = m % t.NS;
        mbar_wait(&full[s], (uint32_t)(m / t.NS) & 1u, a.err);
      }
    }
    return;
  }

  // consumers: walk the same sequence, holding at most two bundles at a time
  const int ctid = threadIdx.x;
  const int lane = threadIdx.x & 31;
  int n = 0;  // next bundle number to acquire
  int held = -1, held_tile = -1, held_p = -1;
  auto stage_of = [&](int m) { return smem + (size_t)(m % t.NS) * t.stage_floats; };
  auto release = [&](int m) {
    __syncwarp();
    if (lane == 0) mbar_arrive(&empty[m % t.NS]);
  };
  for_each_bundle<kIsH>(a, [&](int tile, int p, int kind) {
    const int m = n++;
    if (!mbar_wait(&full[m % t.NS], (uint32_t)(m / t.NS) & 1u, a.err)) return false;
    if (kIsH) {
      // the held plane's x-neighbour (plane + 1, same tile) is always the next bundle
      if (held >= 0) {
        h_plane(a, sprof_, stage_of(held), stage_of(m), held_tile, held_p, ctid);
        release(held);
        held = -1;
      }
      if (kind == kFOnly) {
        release(m);
      } else if (p + 1 < a.g.nx) {
        held = m;
        held_tile = tile;
        held_p = p;
      } else {
        h_plane(a, sprof_, stage_of(m), nullptr, tile, p, ctid);
        release(m);
      }
    } else {
      // the held bundle is plane p - 1 of the same tile whenever p > 0
      if (kind == kFull) {
        const bool prev = held >= 0 && held_tile == tile && held_p + 1 == p;
        if (p > 0 && prev) e_plane(a, sprof_, stage_of(m), stage_of(held), tile, p, ctid);
      }
      if (held >= 0) release(held);
      held = m;
      held_tile = tile;
      held_p = p;
    }
    return true;
  });
  if (held >= 0) release(held);
}

}  // namespace oems
