// Tensor-core (tcgen05) building blocks of the DFT-matrix transforms.
//
// A transform of L points over a batch of columns is the product Y = F X with
// F[k][j] = exp(-2 pi i j k / L).  It runs on the 5th-generation tensor cores as
// real BF16 products accumulated in FP32 in tensor memory (TMEM):
//   D1 = Fr [Xr | Xi],  D2 = Fi [Xr | Xi]   (M = 128 outputs k, N = 2 W, K = 128)
//   Y = (D1[:, c] - s D2[:, W + c]) + i (D1[:, W + c] + s D2[:, c]),  s = +1 forward, -1 inverse
// Every operand is split into two BF16 terms, a = a_hi + a_lo with a_hi = bf16(a)
// and a_lo = bf16(a - a_hi) (16 significant bits together), and each product is
// the three-term sum F_hi X_hi + F_hi X_lo + F_lo X_hi, so the result carries about
// FP32's relative error (2^-16 per term against 2^-8 for one BF16 product).
//
// Shared-memory operand layouts (no swizzle, the canonical UMMA core matrices of
// 8 rows x 16 bytes):
//   A (F, M x K = 128 x 128, K-major):  byte (m, k) = (m / 8) 2048 + (k / 8) 128 + (m % 8) 16 + (k % 8) 2
//   B (X, N x K, MN-major, N = 2 W):    byte (n, k) = (n / 8) 128 + (k / 8) LBO + (k % 8) 16 + (n % 8) 2,
//                                       LBO = (N / 8) 128
// The MMA instruction is M = 128, N = 2 W, K = 16 (kind::f16, BF16 inputs, FP32
// accumulator), issued by one thread; completion is signalled on an mbarrier by
// tcgen05.commit.
#pragma once

#include <cuda_bf16.h>
#include <stdint.h>

namespace cvdv {
namespace tc {

constexpr int kM = 128;           // MMA M = DFT outputs per tile
constexpr int kK = 128;           // DFT inputs per tile
constexpr int kABytes = kM * kK * 2;  // one BF16 copy of A (32 KB)

__device__ __forceinline__ uint32_t saddr(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

// ---- UMMA descriptors
__host__ __device__ constexpr uint32_t instr_desc_bf16(int M, int N, bool bMN) {
  return (1u << 4)                      // D: F32
         | (1u << 7)                    // A: BF16
         | (1u << 10)                   // B: BF16
         | (0u << 15)                   // A K-major
         | ((bMN ? 1u : 0u) << 16)      // B MN-major
         | ((uint32_t)(N >> 3) << 17)   // N / 8
         | ((uint32_t)(M >> 4) << 24);  // M / 16
}

// shared-memory matrix descriptor, no swizzle: start, leading and stride byte offsets
__device__ __forceinline__ uint64_t smem_desc(uint32_t start, uint32_t lbo, uint32_t sbo) {
  uint64_t d = 0;
  d |= (uint64_t)((start >> 4) & 0x3FFF);
  d |= (uint64_t)((lbo >> 4) & 0x3FFF) << 16;
  d |= (uint64_t)((sbo >> 4) & 0x3FFF) << 32;
  d |= (uint64_t)1 << 46;  // descriptor version of sm_100
  return d;                // base offset 0, layout type 0 (no swizzle)
}

// ---- TMEM
__device__ __forceinline__ void tmem_alloc(uint32_t dstSmem, uint32_t ncols) {
  asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(dstSmem), "r"(ncols)
               : "memory");
  asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}
__device__ __forceinline__ void tmem_dealloc(uint32_t taddr, uint32_t ncols) {
  asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(ncols) : "memory");
}
__device__ __forceinline__ void fence_before_sync() {
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
}
__device__ __forceinline__ void fence_after_sync() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
// generic-proxy shared-memory writes become visible to the tensor cores
__device__ __forceinline__ void fence_async_smem() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

__device__ __forceinline__ void mma_bf16(uint32_t dTmem, uint64_t aDesc, uint64_t bDesc, uint32_t idesc,
                                         uint32_t accumulate) {
  asm volatile(
      "{\n .reg .pred p;\n setp.ne.b32 p, %4, 0;\n"
      " tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n}\n" ::"r"(dTmem),
      "l"(aDesc), "l"(bDesc), "r"(idesc), "r"(accumulate)
      : "memory");
}
// arrive on a local mbarrier once every MMA issued so far by this thread is done
__device__ __forceinline__ void mma_commit(uint32_t bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(bar)
               : "memory");
}

// 16 consecutive 32-bit TMEM columns of this thread's lane (warp w reads lanes 32 w .. 32 w + 31)
__device__ __forceinline__ void tmem_ld16(uint32_t taddr, float (&r)[16]) {
  uint32_t u[16];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, "
      "%15}, [%16];"
      : "=r"(u[0]), "=r"(u[1]), "=r"(u[2]), "=r"(u[3]), "=r"(u[4]), "=r"(u[5]), "=r"(u[6]), "=r"(u[7]),
        "=r"(u[8]), "=r"(u[9]), "=r"(u[10]), "=r"(u[11]), "=r"(u[12]), "=r"(u[13]), "=r"(u[14]), "=r"(u[15])
      : "r"(taddr));
#pragma unroll
  for (int i = 0; i < 16; ++i) r[i] = __uint_as_float(u[i]);
}
__device__ __forceinline__ void tmem_ld_wait() { asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory"); }

// ---- mbarrier (CTA-local)
__device__ __forceinline__ void bar_init(uint32_t bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(bar), "r"(count) : "memory");
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}
__device__ __forceinline__ bool bar_try_wait(uint32_t bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
      : "=r"(ok)
      : "r"(bar), "r"(parity)
      : "memory");
  return ok != 0;
}
// Bounded wait: after ~2^22 polls a wait that never completes is recorded in *err
// (when err is non-null) and the caller goes on, so the kernel still frees its TMEM
// and ends.
__device__ __forceinline__ bool bar_wait(uint32_t bar, uint32_t parity, unsigned int* err) {
  for (uint32_t it = 0; it < (1u << 22); ++it)
    if (bar_try_wait(bar, parity)) return true;
  if (err) atomicOr(err, 2u);
  return false;
}

// ---- BF16 split of FP32 values: 8 values -> 16 bytes of hi, 16 bytes of lo
__device__ __forceinline__ void split8(const float (&x)[8], uint4& hi, uint4& lo) {
  uint32_t h[4], l[4];
#pragma unroll
  for (int i = 0; i < 4; ++i) {
    const __nv_bfloat162 hb = __floats2bfloat162_rn(x[2 * i], x[2 * i + 1]);
    const float2 hf = __bfloat1622float2(hb);
    const __nv_bfloat162 lb = __floats2bfloat162_rn(x[2 * i] - hf.x, x[2 * i + 1] - hf.y);
    h[i] = *reinterpret_cast<const uint32_t*>(&hb);
    l[i] = *reinterpret_cast<const uint32_t*>(&lb);
  }
  hi = make_uint4(h[0], h[1], h[2], h[3]);
  lo = make_uint4(l[0], l[1], l[2], l[3]);
}

// byte offset of element (n, k) of B (MN-major, N rows of the operand)
__host__ __device__ constexpr uint32_t b_off(int n, int k, int N) {
  return (uint32_t)((n >> 3) * 128 + (k >> 3) * (N / 8) * 128 + (k & 7) * 16 + (n & 7) * 2);
}
// byte offset of element (m, k) of A (K-major, K = 128)
__host__ __device__ constexpr uint32_t a_off(int m, int k) {
  return (uint32_t)((m >> 3) * 2048 + (k >> 3) * 128 + (m & 7) * 16 + (k & 7) * 2);
}

}  // namespace tc
}  // namespace cvdv
