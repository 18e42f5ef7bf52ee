// Fifth-generation tensor-core (tcgen05) building blocks for sm_100a:
// shared-memory matrix descriptors, the instruction descriptor of
// kind::tf32 / kind::f16 MMAs, tensor-memory (TMEM) allocation, MMA issue,
// completion through an mbarrier and TMEM -> register loads.
//
// Operands are in shared memory in the canonical K-major layout without
// swizzling: a "core matrix" is 8 rows of 16 contiguous bytes (128 bytes in
// all); consecutive 8-row groups along M (or N) are SBO bytes apart and the
// two 16-byte halves of one MMA's K extent (32 bytes: 8 TF32 or 16 BF16
// values) are LBO bytes apart.  Row m, K byte k of an operand therefore sits
// at  start + (m/8)*SBO + (m%8)*16 + (k/16)*LBO + k%16.
//
// The accumulator of an M = 128, cta_group::1 MMA occupies TMEM lanes
// 0..127 (row m -> lane m) and N consecutive 32-bit columns; warp w of the
// CTA may read lanes 32*(w%4) .. 32*(w%4)+31 only.
#pragma once
#include <stdint.h>
#include "tma.cuh"

namespace tara {
namespace umma {

// Shared-memory matrix descriptor (no swizzle, K-major): start address, LBO
// and SBO in 16-byte units; bits 46-47 hold the descriptor version (1 on
// sm_100); base offset, LBO mode and layout type (0 = no swizzle) are zero.
__device__ __forceinline__ uint64_t smem_desc(unsigned saddr, unsigned lbo_bytes, unsigned sbo_bytes) {
  uint64_t d = 0;
  d |= (uint64_t)((saddr >> 4) & 0x3FFFu);
  d |= (uint64_t)((lbo_bytes >> 4) & 0x3FFFu) << 16;
  d |= (uint64_t)((sbo_bytes >> 4) & 0x3FFFu) << 32;
  d |= (uint64_t)1 << 46;
  return d;
}

// Instruction descriptor of a dense MMA with an FP32 accumulator: A and B of
// format fmt (0 F16, 1 BF16, 2 TF32), both K-major, M x N.
__host__ __device__ constexpr uint32_t instr_desc(unsigned fmt, int M, int N) {
  return (1u << 4)                        // accumulator format: F32
         | (fmt << 7) | (fmt << 10)        // A and B formats
         | ((uint32_t)(N >> 3) << 17)      // N / 8
         | ((uint32_t)(M >> 4) << 24);     // M / 16
}
constexpr unsigned kFmtTF32 = 2;

// TMEM allocation of ncols columns (a power of two >= 32) by one whole warp;
// the address is written to the shared-memory word `slot`.  The
// instruction is warp-collective (.sync.aligned): the warp is reconverged
// first, since a lane may arrive from a branch only it took (without this,
// results were wrong intermittently on the GPU).
__device__ __forceinline__ void tmem_alloc(unsigned* slot, unsigned ncols) {
  __syncwarp();
  asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(slot)),
               "r"(ncols)
               : "memory");
  asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}
__device__ __forceinline__ void tmem_dealloc(unsigned taddr, unsigned ncols) {
  __syncwarp();
  asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(ncols) : "memory");
}
__device__ __forceinline__ void fence_before_sync() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void fence_after_sync() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }

// D[tmem] (+)= A[adesc] * B[bdesc]^T, TF32 operands (one thread issues)
__device__ __forceinline__ void mma_tf32(unsigned dtmem, uint64_t adesc, uint64_t bdesc, uint32_t idesc,
                                         bool accumulate) {
  asm volatile(
      "{\n .reg .pred p;\n setp.ne.b32 p, %4, 0;\n"
      " tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, p;\n}\n" ::"r"(dtmem),
      "l"(adesc), "l"(bdesc), "r"(idesc), "r"((unsigned)accumulate)
      : "memory");
}
// The barrier receives one arrival once every MMA this thread issued before
// has completed.
__device__ __forceinline__ void commit(uint64_t* bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_u32(bar))
               : "memory");
}

// 32 consecutive 32-bit TMEM columns of this thread's lane into v[0..31]
// (lane = taddr lane field + lane of the thread in its warp).
__device__ __forceinline__ void ld_32x32b_x32(unsigned taddr, float* v) {
  unsigned r[32];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, "
      "%15, %16, %17, %18, %19, %20, %21, %22, %23, %24, %25, %26, %27, %28, %29, %30, %31}, [%32];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
        "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15]),
        "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]),
        "=r"(r[24]), "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
      : "r"(taddr)
      : "memory");
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
  for (int k = 0; k < 32; k++) v[k] = __uint_as_float(r[k]);
}

// FP32 -> TF32, round to nearest (ties away), kept in a 32-bit float
__device__ __forceinline__ float to_tf32(float x) {
  unsigned r;
  asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(r) : "f"(x));
  return __uint_as_float(r);
}

}  // namespace umma
}  // namespace tara
