// gemm_tc.cuh -- BF16 GEMM on the 5th-generation tensor cores (tcgen05).
//
//   C[M, N] (f32, row-major) = A[M, K] B[N, K]^T (+ beta C) (+ bias[N])
//
// A and B are bf16, K-major (row-major with the reduction along the row),
// row pitches multiples of 8 elements, K a multiple of 8; M and N are free.
// A persistent grid (one CTA per SM) walks the 128 x BN output tiles; each
// CTA is warp-specialised:
//   warp 0      one thread issues the TMA tile loads (cp.async.bulk.tensor,
//               128-byte swizzle, zero fill past the matrix edge) of 64-wide
//               K-blocks into a ring of shared-memory stages, each completed
//               by its "full" mbarrier's transaction count;
//   warp 1      allocates tensor memory (two accumulators of BN columns) and
//               one thread issues the four tcgen05.mma (K = 16 each) of a
//               block, commits them to the stage's "empty" mbarrier (which
//               frees the stage for the next load) and, after a tile's last
//               block, to the accumulator's "full" mbarrier;
//   warps 2-5   the epilogue: each reads its 32 accumulator lanes with
//               tcgen05.ld, applies bias / beta, stores C and releases the
//               accumulator, so the next tile's MMAs run into the other one
//               while this one drains.
// The stage layout is the 128-byte swizzled K-major one (8-row atoms of 1024
// bytes, the 16-byte chunk j of row r at chunk j ^ (r mod 8)), which is what
// TMA writes with CU_TENSOR_MAP_SWIZZLE_128B and what the MMA descriptors
// describe.  No multicast.  Every mbarrier wait is bounded: on timeout the
// CTA sets the error word, its roles stop, the MMA thread waits (bounded
// again) for its last commit and the producer for its copies in flight, and
// the tensor memory is released before the CTA returns.
#pragma once

#include <cuda.h>
#include <cuda_runtime.h>
#include <stdint.h>
namespace oems {

namespace tc {

__device__ __forceinline__ uint32_t smem_u32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

// Shared-memory matrix descriptor (tcgen05): start address >> 4 in bits
// 0-13, leading byte offset >> 4 in 16-29 (unused for swizzled K-major; 1),
// stride byte offset >> 4 in 32-45 (1024 bytes between 8-row atoms),
// version 1 in bits 46-47, layout 2 (128-byte swizzle) in bits 61-63.
__device__ __forceinline__ uint64_t sw128_desc(uint32_t saddr) {
  uint64_t d = 0;
  d |= (uint64_t)((saddr >> 4) & 0x3FFF);
  d |= (uint64_t)1 << 16;
  d |= (uint64_t)(1024 >> 4) << 32;
  d |= (uint64_t)1 << 46;
  d |= (uint64_t)2 << 61;
  return d;
}

// Instruction descriptor, kind::f16: D f32 (bits 4-5 = 1), A and B bf16
// (bits 7-9 and 10-12 = 1), both K-major (bits 15, 16 = 0), N >> 3 in bits
// 17-22, M >> 4 in bits 24-28.
__host__ __device__ constexpr uint32_t idesc_bf16_f32(int M, int N) {
  return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(N >> 3) << 17) | ((uint32_t)(M >> 4) << 24);
}

__device__ __forceinline__ void mbar_init(uint64_t* b, uint32_t n) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(b)), "r"(n) : "memory");
}

__device__ __forceinline__ bool mbar_try(uint64_t* b, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}"
      : "=r"(ok)
      : "r"(smem_u32(b)), "r"(parity)
      : "memory");
  return ok != 0;
}

constexpr long long kTcWait = 2000000000LL;  // ~1 s of clock64

// Bounded wait; false when it gave up (error word set) or another CTA did.
__device__ __forceinline__ bool mbar_wait(uint64_t* b, uint32_t parity, int* err) {
  if (mbar_try(b, parity)) return true;
  const long long t0 = clock64();
  while (!mbar_try(b, parity)) {
    if (*reinterpret_cast<volatile int*>(err) != 0) return false;
    if (clock64() - t0 > kTcWait) {
      atomicExch(err, 1);
      return false;
    }
  }
  return true;
}

__device__ __forceinline__ void mbar_expect_tx(uint64_t* b, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(b)), "r"(bytes) : "memory");
}

__device__ __forceinline__ void mbar_arrive(uint64_t* b) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(b)) : "memory");
}

// Bounded by time only (not by the error word): the drain of work already
// issued before a CTA gives up.
__device__ __forceinline__ bool mbar_drain(uint64_t* b, uint32_t parity) {
  const long long t0 = clock64();
  while (!mbar_try(b, parity))
    if (clock64() - t0 > kTcWait) return false;
  return true;
}

// 2D tiled TMA load of box (x = K offset, y = row offset) into shared memory,
// completing `bytes` on the mbarrier.  x is a multiple of 64 bf16 = 128 bytes.
__device__ __forceinline__ void tma_load_2d(uint32_t dst, const CUtensorMap* map, int x, int y, uint64_t* bar) {
  asm volatile(
      "cp.async.bulk.tensor.2d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], [%4];" ::"r"(
          dst),
      "l"(reinterpret_cast<uint64_t>(map)), "r"(x), "r"(y), "r"(smem_u32(bar))
      : "memory");
}

}  // namespace tc

struct GemmArgs {
  float* c;
  const float* bias;  // may be null
  int ldc;
  int M, N, K;
  float beta;
  int* err;
};

template <int BN>
struct GemmCfg {
  static_assert(BN == 64 || BN == 128 || BN == 256, "BN");
  static constexpr int BM = 128, BK = 64;
  static constexpr int S = BN == 256 ? 4 : (BN == 128 ? 6 : 8);  // ~192 KB of stages
  static constexpr int kStageA = BM * 128, kStageB = BN * 128, kStage = kStageA + kStageB;
  static constexpr uint32_t kCols = 2 * BN;  // two accumulators (a power of two >= 128)
  static constexpr size_t smem = 1024 + (size_t)S * kStage + (2 * S + 4) * 8 + 16;
};

template <int BN>
__global__ void __launch_bounds__(192, 1)
    k_gemm_tc(const __grid_constant__ CUtensorMap ta, const __grid_constant__ CUtensorMap tb, const GemmArgs p) {
  using G = GemmCfg<BN>;
  constexpr int BM = G::BM, BK = G::BK, S = G::S;
  extern __shared__ __align__(1024) uint8_t smem_raw[];
  uint8_t* base = reinterpret_cast<uint8_t*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
  uint64_t* full = reinterpret_cast<uint64_t*>(base + S * G::kStage);
  uint64_t* empty = full + S;
  uint64_t* acc_full = empty + S;    // [2]
  uint64_t* acc_empty = acc_full + 2;  // [2]
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(acc_empty + 2);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int tn = (p.N + BN - 1) / BN, tiles = ((p.M + BM - 1) / BM) * tn;
  const int nkb = (p.K + BK - 1) / BK;
  const uint32_t sbase = tc::smem_u32(base);

  if (warp == 1) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(tc::smem_u32(tmem_slot)),
                 "r"(G::kCols)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  if (threadIdx.x == 0) {
    for (int st = 0; st < S; ++st) {
      tc::mbar_init(full + st, 1);
      tc::mbar_init(empty + st, 1);
    }
    for (int b = 0; b < 2; ++b) {
      tc::mbar_init(acc_full + b, 1);
      tc::mbar_init(acc_empty + b, 4);  // one arrival per epilogue warp
    }
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  const uint32_t tmem = *tmem_slot;

  if (warp == 0 && lane == 0) {
    // ---- producer: K-block `it` (counted over all of this CTA's tiles)
    // goes to stage it % S once the MMAs of block it - S have released it
    asm volatile("prefetch.tensormap [%0];" ::"l"(reinterpret_cast<uint64_t>(&ta)) : "memory");
    asm volatile("prefetch.tensormap [%0];" ::"l"(reinterpret_cast<uint64_t>(&tb)) : "memory");
    int it = 0;
    bool ok = true;
    for (int t = blockIdx.x; t < tiles && ok; t += gridDim.x) {
      const int m0 = (t / tn) * BM, n0 = (t % tn) * BN;
      for (int kb = 0; kb < nkb; ++kb, ++it) {
        const int st = it % S;
        if (!tc::mbar_wait(empty + st, (uint32_t)(((it / S) & 1) ^ 1), p.err)) {
          ok = false;
          break;
        }
        tc::mbar_expect_tx(full + st, (uint32_t)G::kStage);
        const uint32_t sa = sbase + st * G::kStage;
        tc::tma_load_2d(sa, &ta, kb * BK, m0, full + st);
        tc::tma_load_2d(sa + G::kStageA, &tb, kb * BK, n0, full + st);
      }
    }
    if (!ok)  // the copies still in flight land before shared memory goes away
      for (int j = it > S ? it - S : 0; j < it; ++j) (void)tc::mbar_drain(full + j % S, (uint32_t)((j / S) & 1));
  } else if (warp == 1 && lane == 0) {
    // ---- MMA issuer: tile tl accumulates into tensor-memory columns
    // (tl & 1) * BN once the epilogue has drained that accumulator
    constexpr uint32_t idesc = tc::idesc_bf16_f32(BM, BN);
    int it = 0, last = -1;  // last: the K-block of the latest commit
    bool ok = true;
    int tl = 0;
    for (int t = blockIdx.x; t < tiles && ok; t += gridDim.x, ++tl) {
      const int b = tl & 1;
      if (!tc::mbar_wait(acc_empty + b, (uint32_t)(((tl >> 1) & 1) ^ 1), p.err)) {
        ok = false;
        break;
      }
      asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
      const uint32_t acc = tmem + (uint32_t)(b * BN);
      for (int kb = 0; kb < nkb; ++kb, ++it) {
        const int st = it % S;
        if (!tc::mbar_wait(full + st, (uint32_t)((it / S) & 1), p.err)) {
          ok = false;
          break;
        }
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        const uint32_t a_addr = sbase + st * G::kStage, b_addr = a_addr + G::kStageA;
#pragma unroll
        for (int k = 0; k < BK / 16; ++k) {
          // K = 16 bf16 = 32 bytes further along the swizzled row
          const uint64_t ad = tc::sw128_desc(a_addr + k * 32);
          const uint64_t bd = tc::sw128_desc(b_addr + k * 32);
          const uint32_t accum = (kb > 0 || k > 0) ? 1u : 0u;
          asm volatile(
              "{\n\t.reg .pred p;\n\t"
              "setp.ne.b32 p, %4, 0;\n\t"
              "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}" ::"r"(acc),
              "l"(ad), "l"(bd), "r"(idesc), "r"(accum)
              : "memory");
        }
        asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                         tc::smem_u32(empty + st))
                     : "memory");
        last = it;
      }
      if (!ok) break;
      asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                       tc::smem_u32(acc_full + b))
                   : "memory");
    }
    // a commit tracks every earlier MMA of this thread: after an error, wait
    // for the latest one before the tensor memory is released
    if (!ok && last >= 0) (void)tc::mbar_drain(empty + last % S, (uint32_t)((last / S) & 1));
  } else if (warp >= 2) {
    // ---- epilogue: warp w reads accumulator lanes 32 (w % 4) .. + 31
    const int q = warp & 3;
    const bool vec = (p.ldc % 4 == 0) && ((reinterpret_cast<uintptr_t>(p.c) & 15) == 0);
    int tl = 0;
    for (int t = blockIdx.x; t < tiles; t += gridDim.x, ++tl) {
      const int b = tl & 1;
      int fine = 1;
      if (lane == 0) fine = tc::mbar_wait(acc_full + b, (uint32_t)((tl >> 1) & 1), p.err) ? 1 : 0;
      if (!__shfl_sync(0xffffffffu, fine, 0)) break;
      asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
      const int m0 = (t / tn) * BM, n0 = (t % tn) * BN;
      const int row = m0 + q * 32 + lane;
      for (int c0 = 0; c0 < BN && n0 + c0 < p.N; c0 += 32) {
        uint32_t v[32];
        const uint32_t taddr = tmem + ((uint32_t)(q * 32) << 16) + (uint32_t)(b * BN + c0);
        asm volatile(
            "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, "
            "%14, %15, %16, %17, %18, %19, %20, %21, %22, %23, %24, %25, %26, %27, %28, %29, %30, %31}, [%32];"
            : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]), "=r"(v[7]),
              "=r"(v[8]), "=r"(v[9]), "=r"(v[10]), "=r"(v[11]), "=r"(v[12]), "=r"(v[13]), "=r"(v[14]), "=r"(v[15]),
              "=r"(v[16]), "=r"(v[17]), "=r"(v[18]), "=r"(v[19]), "=r"(v[20]), "=r"(v[21]), "=r"(v[22]),
              "=r"(v[23]), "=r"(v[24]), "=r"(v[25]), "=r"(v[26]), "=r"(v[27]), "=r"(v[28]), "=r"(v[29]),
              "=r"(v[30]), "=r"(v[31])
            : "r"(taddr)
            : "memory");
        asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
        if (row < p.M) {
          float* crow = p.c + (size_t)row * p.ldc;
#pragma unroll
          for (int e = 0; e < 32; e += 4) {
            const int col = n0 + c0 + e;
            float x[4];
#pragma unroll
            for (int u = 0; u < 4; ++u) {
              x[u] = __uint_as_float(v[e + u]);
              if (p.bias && col + u < p.N) x[u] += __ldg(p.bias + col + u);
            }
            if (vec && col + 3 < p.N) {
              float4* cp = reinterpret_cast<float4*>(crow + col);
              if (p.beta != 0.0f) {
                const float4 o = *cp;
                x[0] += p.beta * o.x;
                x[1] += p.beta * o.y;
                x[2] += p.beta * o.z;
                x[3] += p.beta * o.w;
              }
              *cp = make_float4(x[0], x[1], x[2], x[3]);
            } else {
#pragma unroll
              for (int u = 0; u < 4; ++u) {
                if (col + u >= p.N) break;
                float* cp = crow + col + u;
                *cp = p.beta != 0.0f ? x[u] + p.beta * *cp : x[u];
              }
            }
          }
        }
      }
      asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
      __syncwarp();
      if (lane == 0) tc::mbar_arrive(acc_empty + b);
    }
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  if (warp == 1) {
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(G::kCols) : "memory");
  }
}

// One CTA waits, through the GEMM's own bounded wait, on an mbarrier that no
// thread or copy ever arrives at: the wait gives up after its limit and sets
// the error word.  Nothing is in flight on the barrier, so the CTA exits
// cleanly.  For tests of the timeout path: the host reads the error word
// (oems_tc_check) and the context stays usable.
__global__ void k_tc_wait_probe(int* err) {
  __shared__ uint64_t bar;
  if (threadIdx.x == 0) {
    tc::mbar_init(&bar, 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  __syncthreads();
  if (threadIdx.x == 0) (void)tc::mbar_wait(&bar, 0, err);
  __syncthreads();
}

}  // namespace oems
