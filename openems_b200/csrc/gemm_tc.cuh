// gemm_tc.cuh -- BF16 GEMM on the 5th-generation tensor cores (tcgen05).
//
//   C[M, N] (f32, row-major) = A[M, K] B[N, K]^T (+ beta C) (+ bias[N])
//
// A and B are bf16, K-major (row-major with the reduction along the row),
// row pitches multiples of 8 elements, K a multiple of 8; M and N are free.
// One CTA computes a 128 x BN tile.  Blocks of 64 along K go through a ring
// of kStages shared-memory stages in the 128-byte swizzled K-major layout
// (8-row atoms of 1024 bytes, the 16-byte chunk j of row r at chunk
// j ^ (r mod 8)): all 128 threads fill a stage with 16-byte cp.async copies
// (zero-filled past the matrix edge) kStages - 1 blocks ahead, one thread
// issues the four tcgen05.mma (K = 16 each) of a block with the accumulator
// in tensor memory and commits them to the stage's mbarrier, and a stage is
// refilled only after that mbarrier says its MMAs are done.  After the last
// block each warp reads its 32 accumulator lanes with tcgen05.ld.  Every
// mbarrier wait is bounded: on timeout the CTA sets the error word, skips its
// remaining work, releases its tensor memory and returns.
#pragma once

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

}  // namespace tc

struct GemmArgs {
  const uint16_t* a;  // bf16 bits
  const uint16_t* b;
  float* c;
  const float* bias;  // may be null
  int lda, ldb, ldc;
  int M, N, K;
  float beta;
  int* err;
};

constexpr int kGemmStages = 4;

__device__ __forceinline__ void cp_async16(uint32_t dst, const void* src, bool in_range) {
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;" ::"r"(dst), "l"(src), "r"(in_range ? 16 : 0)
               : "memory");
}

template <int BN>
__global__ void __launch_bounds__(128) k_gemm_tc(const GemmArgs p) {
  static_assert(BN == 64 || BN == 128, "BN");
  constexpr int BM = 128, BK = 64, S = kGemmStages;
  constexpr int kStageA = BM * 128, kStageB = BN * 128, kStage = kStageA + kStageB;
  extern __shared__ __align__(1024) uint8_t smem_raw[];
  // 1024-byte aligned operand stages, then the mbarriers and the TMEM slot
  uint8_t* base = reinterpret_cast<uint8_t*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
  uint64_t* bar = reinterpret_cast<uint64_t*>(base + S * kStage);
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(bar + S);
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int m0 = blockIdx.y * BM, n0 = blockIdx.x * BN;
  const uint32_t sbase = tc::smem_u32(base);

  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(tc::smem_u32(tmem_slot)),
                 "r"(BN)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  if (tid == 0) {
    for (int st = 0; st < S; ++st) tc::mbar_init(bar + st, 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  const uint32_t tmem = *tmem_slot;
  constexpr uint32_t idesc = tc::idesc_bf16_f32(BM, BN);
  const int nkb = (p.K + BK - 1) / BK;

  // copies of K-block kb into its stage: chunk j of row r at
  // (r / 8) * 1024 + (r % 8) * 128 + ((j ^ (r % 8)) * 16); one commit group
  // per block (empty past the last block, so group counting stays uniform)
  auto load_block = [&](int kb) {
    if (kb < nkb) {
      const int k0 = kb * BK;
      const uint32_t sa = sbase + (kb % S) * kStage, sb = sa + kStageA;
      for (int q = tid; q < BM * 8; q += 128) {
        const int r = q >> 3, j = q & 7;
        const int gm = m0 + r, gk = k0 + j * 8;
        const bool in = gm < p.M && gk < p.K;
        cp_async16(sa + (r >> 3) * 1024 + (r & 7) * 128 + ((j ^ (r & 7)) << 4),
                   in ? (const void*)(p.a + (size_t)gm * p.lda + gk) : (const void*)p.a, in);
      }
      for (int q = tid; q < BN * 8; q += 128) {
        const int r = q >> 3, j = q & 7;
        const int gn = n0 + r, gk = k0 + j * 8;
        const bool in = gn < p.N && gk < p.K;
        cp_async16(sb + (r >> 3) * 1024 + (r & 7) * 128 + ((j ^ (r & 7)) << 4),
                   in ? (const void*)(p.b + (size_t)gn * p.ldb + gk) : (const void*)p.b, in);
      }
    }
    asm volatile("cp.async.commit_group;" ::: "memory");
  };

  for (int kb = 0; kb < S - 1; ++kb) load_block(kb);
  bool ok = true;
  int issued = 0;  // K-blocks whose MMAs thread 0 has committed
  for (int kb = 0; kb < nkb && ok; ++kb) {
    // block kb has landed (at most S - 2 younger groups in flight); its
    // generic-proxy writes are made visible to the tensor cores
    asm volatile("cp.async.wait_group %0;" ::"n"(S - 2) : "memory");
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    __syncthreads();
    if (tid == 0) {
      asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
      const uint32_t a_addr = sbase + (kb % S) * kStage, b_addr = a_addr + kStageA;
#pragma unroll
      for (int k = 0; k < BK / 16; ++k) {
        // K = 16 bf16 = 32 bytes further along the swizzled row
        const uint64_t ad = tc::sw128_desc(a_addr + k * 32);
        const uint64_t bd = tc::sw128_desc(b_addr + k * 32);
        const uint32_t acc = (kb > 0 || k > 0) ? 1u : 0u;
        asm volatile(
            "{\n\t.reg .pred p;\n\t"
            "setp.ne.b32 p, %4, 0;\n\t"
            "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}" ::"r"(tmem),
            "l"(ad), "l"(bd), "r"(idesc), "r"(acc)
            : "memory");
      }
      asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                       tc::smem_u32(bar + kb % S))
                   : "memory");
    }
    issued = kb + 1;
    // the stage of block kb - 1 is refilled with block kb + S - 1 once that
    // block's MMAs are done; a block-wide vote keeps every thread on the
    // same iteration count
    bool fine = true;
    if (kb > 0) fine = tc::mbar_wait(bar + (kb - 1) % S, (uint32_t)(((kb - 1) / S) & 1), p.err);
    ok = __syncthreads_and(fine) != 0;
    if (ok) load_block(kb + S - 1);
  }
  // the last block's MMAs (and with them every earlier one) are done
  if (ok && nkb > 0) ok = __syncthreads_and(tc::mbar_wait(bar + (nkb - 1) % S, (uint32_t)(((nkb - 1) / S) & 1),
                                                          p.err)) != 0;
  else if (!ok && issued > 0)
    // a wait gave up: before tensor memory and shared memory are released,
    // wait (bounded again) for the last committed block, whose commit
    // tracks every earlier MMA; if that wait gives up too the CTA's tile is
    // left undefined (the error word is already set)
    (void)__syncthreads_and(
        tc::mbar_wait(bar + (issued - 1) % S, (uint32_t)(((issued - 1) / S) & 1), p.err));
  asm volatile("cp.async.wait_all;" ::: "memory");
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");

  if (ok) {
    // epilogue: warp w owns accumulator lanes (rows) 32w .. 32w + 31
    const int row = m0 + warp * 32 + lane;
#pragma unroll
    for (int c0 = 0; c0 < BN; c0 += 8) {
      uint32_t v[8];
      const uint32_t taddr = tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)c0;
      asm volatile("tcgen05.ld.sync.aligned.32x32b.x8.b32 {%0, %1, %2, %3, %4, %5, %6, %7}, [%8];"
                   : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]), "=r"(v[7])
                   : "r"(taddr)
                   : "memory");
      asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
      if (row < p.M) {
#pragma unroll
        for (int e = 0; e < 8; ++e) {
          const int col = n0 + c0 + e;
          if (col >= p.N) break;
          float x = nkb > 0 ? __uint_as_float(v[e]) : 0.0f;
          if (p.bias) x += p.bias[col];
          float* cp = p.c + (size_t)row * p.ldc + col;
          if (p.beta != 0.0f) x += p.beta * *cp;
          *cp = x;
        }
      }
    }
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  if (warp == 0) {
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(BN) : "memory");
  }
}

template <int BN>
constexpr size_t gemm_tc_smem() {
  return 1024 + (size_t)kGemmStages * (128 * 128 + (size_t)BN * 128) + kGemmStages * 8 + 16;
}

}  // namespace oems
