// yee_pipe.cuh -- pipelined register kernels for the H and E half-steps
// (float fields, full coefficient arrays, the whole grid in one geometry).
//
// Same work items, arithmetic and rounding as k_update_h / k_update_e
// (yee_kernels.cuh), so the results are the same bits.  What differs is how
// a plane's operands arrive.  The register kernels issue a plane's loads
// and then wait for them; at 128 registers (CPML) an SM holds 16 warps and
// the waits are not covered.  Here every thread copies its own chunk of the
// planes ahead into shared memory with cp.async (no registers held while
// the copies fly) and computes from shared memory:
//
//   * a CTA of 256 threads walks the x-planes of its work items as one
//     sequence of steps; step n's bundle (the 12 arrays a thread reads at
//     one plane: fields and coefficients, 192 bytes) goes into stage
//     n % NS of a ring, NS - 2 bundles ahead of the one being computed;
//   * neighbours along y and z are other threads' chunks of the same
//     bundle, or, at the tile's edge, a halo row of the neighbouring tile
//     (nzq chunks of 3 arrays) copied with the bundle;
//   * the x-neighbour plane is the next bundle (H) or the previous one (E);
//     a work item's sequence therefore carries one load-only step: plane i1
//     after its last plane (H: E_y, E_z only) or plane i0 - 1 before its
//     first (E: H_y, H_z only);
//   * CPML psi values are loaded into registers one compute step ahead.
// One __syncthreads per step: after it every thread's bundle for the step
// has landed, and the stage being refilled was last read in the step
// before.  One CTA per SM (~200 KB of shared memory), 8 warps.
#pragma once

#include "yee_kernels.cuh"

namespace oems {

constexpr int kPipeThreads = 256;
constexpr int kPipeArrays = 12;

// shared memory of an NS-stage pipe kernel for a grid with nzq chunks per row
__host__ __device__ constexpr size_t pipe_smem_bytes(int ns, int nzq) {
  return (size_t)ns * (kPipeArrays * kPipeThreads + 3 * nzq) * sizeof(float4);
}

__device__ __forceinline__ void pipe_cp16(float4* dst, const float* src) {
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"((uint32_t)__cvta_generic_to_shared(dst)), "l"(src)
               : "memory");
}
__device__ __forceinline__ void pipe_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int N>
__device__ __forceinline__ void pipe_wait() {
  asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory");
}

// One step of a CTA's sequence: plane i of work item w, compute or load-only.
struct PipeStep {
  int w;       // work item; >= g.work past the end of the sequence
  int i;       // plane
  int i1;      // the item's end plane
  int c0, c1;  // the item's tile of chunks
  bool load;   // load-only: the neighbour plane before (E) or after (H) the item
};

__device__ __forceinline__ void pipe_first(const Geom& g, int w, bool is_h, PipeStep& s) {
  s.w = w;
  if (w >= g.work) return;
  const Item it = work_item(g, w);
  s.c0 = it.c0;
  s.c1 = it.c1;
  s.i1 = it.i1;
  s.load = !is_h && it.i0 > 0;
  s.i = s.load ? it.i0 - 1 : it.i0;
}

__device__ __forceinline__ void pipe_next(const Geom& g, bool is_h, PipeStep& s) {
  if (s.w >= g.work) return;
  if (is_h) {
    if (!s.load) {
      if (s.i + 1 < s.i1) {
        ++s.i;
        return;
      }
      if (s.i1 < g.nx) {  // plane i1: the x-neighbour of the item's last plane
        s.i = s.i1;
        s.load = true;
        return;
      }
    }
  } else {
    if (s.load || s.i + 1 < s.i1) {
      ++s.i;
      s.load = false;
      return;
    }
  }
  pipe_first(g, s.w + (int)gridDim.x, is_h, s);
}

// the next compute step after s (s itself excluded)
__device__ __forceinline__ PipeStep pipe_next_compute(const Geom& g, bool is_h, PipeStep s) {
  pipe_next(g, is_h, s);
  if (s.w < g.work && s.load) pipe_next(g, is_h, s);
  return s;
}

// Bundle array slots.  H: 0 ex 1 ey 2 ez 3 hx 4 hy 5 hz 6-8 da 9-11 db;
// halo (the nzq chunks after the tile) 0 ex 1 ey 2 ez.  E: 0 ex 1 ey 2 ez
// 3 hx 4 hy 5 hz 6-8 ca 9-11 cb; halo (the nzq chunks before the tile)
// 0 hx 1 hy 2 hz.
struct PipeSmem {
  float4* bun;  // [NS][12][kPipeThreads]
  float4* hal;  // [NS][3][nzq]
  int nzq;
  __device__ __forceinline__ float4* b(int st, int arr) const {
    return bun + ((size_t)st * kPipeArrays + arr) * kPipeThreads;
  }
  __device__ __forceinline__ float4* h(int st, int arr) const { return hal + ((size_t)st * 3 + arr) * nzq; }
};

__device__ __forceinline__ void pipe_issue_h(const HArgs& a, const PipeStep& s, const PipeSmem& sm, int st) {
  const Geom& g = a.g;
  if (s.w < g.work) {
    const int t = threadIdx.x;
    const int c = s.c0 + t;
    if (c < s.c1) {
      const long long q = (long long)s.i * g.plane + 4LL * c;
      if (s.load) {
        pipe_cp16(sm.b(st, 1) + t, a.ey + q);
        pipe_cp16(sm.b(st, 2) + t, a.ez + q);
      } else {
        pipe_cp16(sm.b(st, 0) + t, a.ex + q);
        pipe_cp16(sm.b(st, 1) + t, a.ey + q);
        pipe_cp16(sm.b(st, 2) + t, a.ez + q);
        pipe_cp16(sm.b(st, 3) + t, a.hx + q);
        pipe_cp16(sm.b(st, 4) + t, a.hy + q);
        pipe_cp16(sm.b(st, 5) + t, a.hz + q);
#pragma unroll
        for (int k = 0; k < 3; ++k) {
          pipe_cp16(sm.b(st, 6 + k) + t, a.da[k] + q);
          pipe_cp16(sm.b(st, 9 + k) + t, a.db[k] + q);
        }
      }
    }
    if (!s.load && t < g.nzq) {
      const int ch = s.c1 + t;
      if (ch < g.plane4) {
        const long long q = (long long)s.i * g.plane + 4LL * ch;
        pipe_cp16(sm.h(st, 0) + t, a.ex + q);
        pipe_cp16(sm.h(st, 1) + t, a.ey + q);
        pipe_cp16(sm.h(st, 2) + t, a.ez + q);
      }
    }
  }
  pipe_commit();
}

__device__ __forceinline__ void pipe_issue_e(const EArgs& a, const PipeStep& s, const PipeSmem& sm, int st) {
  const Geom& g = a.g;
  if (s.w < g.work) {
    const int t = threadIdx.x;
    const int c = s.c0 + t;
    if (c < s.c1) {
      const long long q = (long long)s.i * g.plane + 4LL * c;
      if (s.load) {
        pipe_cp16(sm.b(st, 4) + t, a.hy + q);
        pipe_cp16(sm.b(st, 5) + t, a.hz + q);
      } else {
        pipe_cp16(sm.b(st, 0) + t, a.ex + q);
        pipe_cp16(sm.b(st, 1) + t, a.ey + q);
        pipe_cp16(sm.b(st, 2) + t, a.ez + q);
        pipe_cp16(sm.b(st, 3) + t, a.hx + q);
        pipe_cp16(sm.b(st, 4) + t, a.hy + q);
        pipe_cp16(sm.b(st, 5) + t, a.hz + q);
#pragma unroll
        for (int k = 0; k < 3; ++k) {
          pipe_cp16(sm.b(st, 6 + k) + t, a.ca[k] + q);
          pipe_cp16(sm.b(st, 9 + k) + t, a.cb[k] + q);
        }
      }
    }
    if (!s.load && t < g.nzq) {
      const int ch = s.c0 - g.nzq + t;
      if (ch >= 0) {
        const long long q = (long long)s.i * g.plane + 4LL * ch;
        pipe_cp16(sm.h(st, 0) + t, a.hx + q);
        pipe_cp16(sm.h(st, 1) + t, a.hy + q);
        pipe_cp16(sm.h(st, 2) + t, a.hz + q);
      }
    }
  }
  pipe_commit();
}

// CPML psi of one chunk at one plane, held in registers between the step
// that loads it and the step that computes with it.
struct PipePsi {
  SlabInfo sl;
  float4 px0, px1, py0, py1, pzn0, pzn1, pzx0, pzx1;
};

// Slab membership and psi values of the compute step s (this thread's chunk).
__device__ __forceinline__ void pipe_psi_load(const CpmlArgs& cp, const Geom& g, const PipeStep& s, bool is_h,
                                              PipePsi& p) {
  if (s.w >= g.work) {
    p.sl.fx = p.sl.fy = -1;
    p.sl.zmin = p.sl.zmax = false;
    return;
  }
  int c = s.c0 + (int)threadIdx.x;
  if (c >= s.c1) c = s.c1 - 1;
  const int j = c / g.nzq;
  const int k0 = (c - j * g.nzq) * 4;
  p.sl = slab_info(cp, g, s.i, j, k0);
  if (!is_h && !(s.i >= 1 && j >= 1)) {  // E cells that are not updated
    p.sl.fx = p.sl.fy = -1;
    p.sl.zmin = p.sl.zmax = false;
  }
  float* const* ps = is_h ? &cp.psi_h[0][0] : &cp.psi_e[0][0];
  // psi arrays of face f, slot k: ps[2 f + k]
  p.px0 = p.sl.fx >= 0 ? ld4(ps[2 * p.sl.fx] + p.sl.px) : zero4();
  p.px1 = p.sl.fx >= 0 ? ld4(ps[2 * p.sl.fx + 1] + p.sl.px) : zero4();
  p.py0 = p.sl.fy >= 0 ? ld4(ps[2 * p.sl.fy] + p.sl.py) : zero4();
  p.py1 = p.sl.fy >= 0 ? ld4(ps[2 * p.sl.fy + 1] + p.sl.py) : zero4();
  p.pzn0 = p.sl.zmin ? ld4(ps[8] + p.sl.pz0) : zero4();
  p.pzn1 = p.sl.zmin ? ld4(ps[9] + p.sl.pz0) : zero4();
  p.pzx0 = p.sl.zmax ? ld4(ps[10] + p.sl.pz1) : zero4();
  p.pzx1 = p.sl.zmax ? ld4(ps[11] + p.sl.pz1) : zero4();
}

// H half-step of compute step s from stages st (plane i) and st1 (plane i + 1).
template <bool kCpml>
__device__ __forceinline__ void pipe_h_compute(const HArgs& a, const PipeStep& s, const PipeSmem& sm, int st, int st1,
                                               PipePsi& ps) {
  const Geom& g = a.g;
  int c = s.c0 + (int)threadIdx.x;
  const bool valid = c < s.c1;
  if (!valid) c = s.c1 - 1;
  const int t = c - s.c0;
  const int j = c / g.nzq;
  const int k0 = (c - j * g.nzq) * 4;
  const int i = s.i;
  const bool has_ip = i + 1 < g.nx;
  const bool has_jp = j + 1 < g.ny;
  unsigned live = 0;
#pragma unroll
  for (int e = 0; e < 4; ++e) live |= (k0 + e < g.nz ? 1u : 0u) << e;
  const float4 ex4 = sm.b(st, 0)[t];
  const float4 ey4 = sm.b(st, 1)[t];
  const float4 ez4 = sm.b(st, 2)[t];
  const float4 ey1 = has_ip ? sm.b(st1, 1)[t] : ey4;
  const float4 ez1 = has_ip ? sm.b(st1, 2)[t] : ez4;
  float4 exj = ex4, ezj = ez4;
  if (has_jp) {
    const int cy = c + g.nzq;
    if (cy < s.c1) {
      exj = sm.b(st, 0)[cy - s.c0];
      ezj = sm.b(st, 2)[cy - s.c0];
    } else {
      exj = sm.h(st, 0)[cy - s.c1];
      ezj = sm.h(st, 2)[cy - s.c1];
    }
  }
  float exn = 0.f, eyn = 0.f;
  if (k0 + 4 < g.nz) {
    const int cz = c + 1;
    if (cz < s.c1) {
      exn = sm.b(st, 0)[cz - s.c0].x;
      eyn = sm.b(st, 1)[cz - s.c0].x;
    } else {
      exn = sm.h(st, 0)[0].x;
      eyn = sm.h(st, 1)[0].x;
    }
  }
  float co_a[3][4], co_b[3][4], h[3][4];
#pragma unroll
  for (int k = 0; k < 3; ++k) {
    to_arr(sm.b(st, 6 + k)[t], co_a[k]);
    to_arr(sm.b(st, 9 + k)[t], co_b[k]);
    to_arr(sm.b(st, 3 + k)[t], h[k]);
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
    const SlabInfo& sl = ps.sl;
    float b, cc, ik;
    if (sl.fy >= 0) {
      cpml_prof(a.cp, sl.fy, sl.ly, true, b, cc, ik);
      stretch_vec(dez_dy, ps.py0, b, cc, ik, live);
      stretch_vec(dex_dy, ps.py1, b, cc, ik, live);
    }
    if (sl.zmin) {
      stretch_z(a.cp, 4, k0, true, dey_dz, ps.pzn0, live);
      stretch_z(a.cp, 4, k0, true, dex_dz, ps.pzn1, live);
    }
    if (sl.zmax) {
      stretch_z(a.cp, 5, k0, true, dey_dz, ps.pzx0, live);
      stretch_z(a.cp, 5, k0, true, dex_dz, ps.pzx1, live);
    }
    if (sl.fx >= 0) {
      cpml_prof(a.cp, sl.fx, sl.lx, true, b, cc, ik);
      stretch_vec(dez_dx, ps.px0, b, cc, ik, live);
      stretch_vec(dey_dx, ps.px1, b, cc, ik, live);
    }
  }
  float out[3][4];
#pragma unroll
  for (int e = 0; e < 4; ++e) {
    const float curl[3] = {__fsub_rn(dez_dy[e], dey_dz[e]), __fsub_rn(dex_dz[e], dez_dx[e]),
                           __fsub_rn(dey_dx[e], dex_dy[e])};
    const bool lv = (live >> e) & 1u;
#pragma unroll
    for (int k = 0; k < 3; ++k) {
      const float v = __fadd_rn(__fmul_rn(co_a[k][e], h[k][e]), __fmul_rn(co_b[k][e], curl[k]));
      out[k][e] = lv ? v : h[k][e];
    }
  }
  if (valid) {
    const long long q = (long long)i * g.plane + 4LL * c;
    st4(a.hx + q, to_f4(out[0]));
    st4(a.hy + q, to_f4(out[1]));
    st4(a.hz + q, to_f4(out[2]));
    if constexpr (kCpml) {
      const SlabInfo& sl = ps.sl;
      if (sl.fy >= 0) {
        st4(a.cp.psi_h[sl.fy][0] + sl.py, ps.py0);
        st4(a.cp.psi_h[sl.fy][1] + sl.py, ps.py1);
      }
      if (sl.zmin) {
        st4(a.cp.psi_h[4][0] + sl.pz0, ps.pzn0);
        st4(a.cp.psi_h[4][1] + sl.pz0, ps.pzn1);
      }
      if (sl.zmax) {
        st4(a.cp.psi_h[5][0] + sl.pz1, ps.pzx0);
        st4(a.cp.psi_h[5][1] + sl.pz1, ps.pzx1);
      }
      if (sl.fx >= 0) {
        st4(a.cp.psi_h[sl.fx][0] + sl.px, ps.px0);
        st4(a.cp.psi_h[sl.fx][1] + sl.px, ps.px1);
      }
    }
  }
}

// E half-step of compute step s from stages st (plane i) and stp (plane i - 1).
template <bool kCpml>
__device__ __forceinline__ void pipe_e_compute(const EArgs& a, const PipeStep& s, const PipeSmem& sm, int st, int stp,
                                               PipePsi& ps) {
  const Geom& g = a.g;
  int c = s.c0 + (int)threadIdx.x;
  const bool valid = c < s.c1;
  if (!valid) c = s.c1 - 1;
  const int t = c - s.c0;
  const int j = c / g.nzq;
  const int k0 = (c - j * g.nzq) * 4;
  const int i = s.i;
  const bool upd = i >= 1 && j >= 1;
  if (!upd) return;
  unsigned live = 0;
#pragma unroll
  for (int e = 0; e < 4; ++e) live |= (k0 + e >= 1 && k0 + e < g.nz ? 1u : 0u) << e;
  const float4 hx4 = sm.b(st, 3)[t];
  const float4 hy4 = sm.b(st, 4)[t];
  const float4 hz4 = sm.b(st, 5)[t];
  const float4 hym4 = sm.b(stp, 4)[t];
  const float4 hzm4 = sm.b(stp, 5)[t];
  float4 hxj4, hzj4;
  {
    const int cy = c - g.nzq;
    if (cy >= s.c0) {
      hxj4 = sm.b(st, 3)[cy - s.c0];
      hzj4 = sm.b(st, 5)[cy - s.c0];
    } else {
      hxj4 = sm.h(st, 0)[cy - s.c0 + g.nzq];
      hzj4 = sm.h(st, 2)[cy - s.c0 + g.nzq];
    }
  }
  float hxm = 0.f, hym = 0.f;
  if (k0 >= 4) {
    const int cz = c - 1;
    if (cz >= s.c0) {
      hxm = sm.b(st, 3)[cz - s.c0].w;
      hym = sm.b(st, 4)[cz - s.c0].w;
    } else {
      hxm = sm.h(st, 0)[g.nzq - 1].w;
      hym = sm.h(st, 1)[g.nzq - 1].w;
    }
  }
  float co_a[3][4], co_b[3][4], ev[3][4];
#pragma unroll
  for (int k = 0; k < 3; ++k) {
    to_arr(sm.b(st, 6 + k)[t], co_a[k]);
    to_arr(sm.b(st, 9 + k)[t], co_b[k]);
    to_arr(sm.b(st, k)[t], ev[k]);
  }
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
    const SlabInfo& sl = ps.sl;
    float b, cc, ik;
    if (sl.fy >= 0) {
      cpml_prof(a.cp, sl.fy, sl.ly, false, b, cc, ik);
      stretch_vec(dhz_dy, ps.py0, b, cc, ik, live);
      stretch_vec(dhx_dy, ps.py1, b, cc, ik, live);
    }
    if (sl.zmin) {
      stretch_z(a.cp, 4, k0, false, dhy_dz, ps.pzn0, live);
      stretch_z(a.cp, 4, k0, false, dhx_dz, ps.pzn1, live);
    }
    if (sl.zmax) {
      stretch_z(a.cp, 5, k0, false, dhy_dz, ps.pzx0, live);
      stretch_z(a.cp, 5, k0, false, dhx_dz, ps.pzx1, live);
    }
    if (sl.fx >= 0) {
      cpml_prof(a.cp, sl.fx, sl.lx, false, b, cc, ik);
      stretch_vec(dhz_dx, ps.px0, b, cc, ik, live);
      stretch_vec(dhy_dx, ps.px1, b, cc, ik, live);
    }
  }
  float out[3][4];
#pragma unroll
  for (int e = 0; e < 4; ++e) {
    const float curl[3] = {__fsub_rn(dhz_dy[e], dhy_dz[e]), __fsub_rn(dhx_dz[e], dhz_dx[e]),
                           __fsub_rn(dhy_dx[e], dhx_dy[e])};
    const bool lv = (live >> e) & 1u;
#pragma unroll
    for (int k = 0; k < 3; ++k) {
      const float v = __fadd_rn(__fmul_rn(co_a[k][e], ev[k][e]), __fmul_rn(co_b[k][e], curl[k]));
      out[k][e] = lv ? v : ev[k][e];
    }
  }
  if (valid) {
    const long long q = (long long)i * g.plane + 4LL * c;
    st4(a.ex + q, to_f4(out[0]));
    st4(a.ey + q, to_f4(out[1]));
    st4(a.ez + q, to_f4(out[2]));
    if constexpr (kCpml) {
      const SlabInfo& sl = ps.sl;
      if (sl.fy >= 0) {
        st4(a.cp.psi_e[sl.fy][0] + sl.py, ps.py0);
        st4(a.cp.psi_e[sl.fy][1] + sl.py, ps.py1);
      }
      if (sl.zmin) {
        st4(a.cp.psi_e[4][0] + sl.pz0, ps.pzn0);
        st4(a.cp.psi_e[4][1] + sl.pz0, ps.pzn1);
      }
      if (sl.zmax) {
        st4(a.cp.psi_e[5][0] + sl.pz1, ps.pzx0);
        st4(a.cp.psi_e[5][1] + sl.pz1, ps.pzx1);
      }
      if (sl.fx >= 0) {
        st4(a.cp.psi_e[sl.fx][0] + sl.px, ps.px0);
        st4(a.cp.psi_e[sl.fx][1] + sl.px, ps.px1);
      }
    }
  }
}

// H: compute step n reads stages n % NS and (n + 1) % NS; step n + NS - 1 is
// issued into stage (n - 1) % NS after the barrier of step n.
template <bool kCpml, int NS>
__global__ void __launch_bounds__(kPipeThreads, 1) k_update_h_pipe(const HArgs a) {
  static_assert(NS >= 3, "two stages in use plus at least one in flight");
  extern __shared__ __align__(16) float4 pipe_sm[];
  const Geom& g = a.g;
  PipeSmem sm{pipe_sm, pipe_sm + (size_t)NS * kPipeArrays * kPipeThreads, g.nzq};
  PipeStep is, cs;
  pipe_first(g, blockIdx.x, true, is);
  cs = is;
  for (int p = 0; p < NS - 1; ++p) {
    pipe_issue_h(a, is, sm, p);
    pipe_next(g, true, is);
  }
  PipePsi cur{}, nxt{};
  if constexpr (kCpml) pipe_psi_load(a.cp, g, cs, true, cur);
  for (int n = 0; cs.w < g.work; ++n) {
    pipe_wait<NS - 3>();
    __syncthreads();
    pipe_issue_h(a, is, sm, (n + NS - 1) % NS);
    pipe_next(g, true, is);
    if (!cs.load) {
      if constexpr (kCpml) pipe_psi_load(a.cp, g, pipe_next_compute(g, true, cs), true, nxt);
      pipe_h_compute<kCpml>(a, cs, sm, n % NS, (n + 1) % NS, cur);
      if constexpr (kCpml) cur = nxt;
    }
    pipe_next(g, true, cs);
  }
  pipe_wait<0>();
}

// E: compute step n reads stages n % NS and (n - 1) % NS; step n + NS - 2 is
// issued into stage (n - 2) % NS after the barrier of step n.
template <bool kCpml, int NS>
__global__ void __launch_bounds__(kPipeThreads, 1) k_update_e_pipe(const EArgs a) {
  static_assert(NS >= 3, "two stages in use plus at least one in flight");
  extern __shared__ __align__(16) float4 pipe_sm[];
  const Geom& g = a.g;
  PipeSmem sm{pipe_sm, pipe_sm + (size_t)NS * kPipeArrays * kPipeThreads, g.nzq};
  PipeStep is, cs;
  pipe_first(g, blockIdx.x, false, is);
  cs = is;
  for (int p = 0; p < NS - 2; ++p) {
    pipe_issue_e(a, is, sm, p);
    pipe_next(g, false, is);
  }
  PipePsi cur{}, nxt{};
  if constexpr (kCpml) {
    PipeStep f = cs;
    if (f.w < g.work && f.load) pipe_next(g, false, f);
    pipe_psi_load(a.cp, g, f, false, cur);
  }
  for (int n = 0; cs.w < g.work; ++n) {
    pipe_wait<NS - 3>();
    __syncthreads();
    pipe_issue_e(a, is, sm, (n + NS - 2) % NS);
    pipe_next(g, false, is);
    if (!cs.load) {
      if constexpr (kCpml) pipe_psi_load(a.cp, g, pipe_next_compute(g, false, cs), false, nxt);
      pipe_e_compute<kCpml>(a, cs, sm, n % NS, (n + NS - 1) % NS, cur);
      if constexpr (kCpml) cur = nxt;
    }
    pipe_next(g, false, cs);
  }
  pipe_wait<0>();
}

}  // namespace oems
