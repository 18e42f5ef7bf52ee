// Tensor-memory-accelerator (TMA) tile loads for the column pass.
//
// A spectral field [Ny][ld] of Cx<T> is described to the TMA unit as a 2D
// tensor of T with inner extent 2*ld (re, im interleaved) and outer extent
// Ny.  A column tile of CB complex columns and BOX rows is one box
// {2*CB, BOX}; its x coordinate 2*c0 is always a multiple of 16 bytes.  The
// box lands in shared memory row-major: element (t, i) of the tile at
// i*CB + t.  Completion is tracked by an mbarrier with a transaction count.
// Every wait is bounded (Tables::wait_ns of %globaltimer, one second unless
// the session sets another limit); a kernel whose wait runs out records
// TARA_ETIMEOUT in the grid's status word and stops.
#pragma once
#include <cuda.h>
#include <cudaTypedefs.h>
#include <cuda_runtime.h>
#include <stdint.h>
#include "spectral.cuh"

namespace tara {

// ---------------------------------------------------------------- host
// cuTensorMapEncodeTiled through the runtime's driver entry point.
int tma_encode_tile(CUtensorMap* map, CUtensorMapDataType dt, void* base, uint64_t inner_elems,
                    uint64_t rows, uint64_t row_bytes, uint32_t box_inner, uint32_t box_rows);

// A pool of nf fields back to back ([nf][Ny][ld]) as one 3D tensor; box
// {2*CB, box_rows, 1}.
int tma_encode_tile3(CUtensorMap* map, CUtensorMapDataType dt, void* base, uint64_t inner_elems, uint64_t rows,
                     uint64_t nf, uint64_t row_bytes, uint64_t field_bytes, uint32_t box_inner, uint32_t box_rows);
template <class T>
inline int make_pool_tile_map(CUtensorMap* map, const Cx<T>* base, int ld, int Ny, int nf, int CB, int box_rows) {
  const CUtensorMapDataType dt = sizeof(T) == 8 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT64 : CU_TENSOR_MAP_DATA_TYPE_FLOAT32;
  return tma_encode_tile3(map, dt, const_cast<Cx<T>*>(base), 2ull * ld, (uint64_t)Ny, (uint64_t)nf,
                          (uint64_t)ld * sizeof(Cx<T>), (uint64_t)ld * Ny * sizeof(Cx<T>), 2u * CB, (uint32_t)box_rows);
}
template <class T>
inline int make_col_tile_map(CUtensorMap* map, const Cx<T>* base, int ld, int Ny, int CB, int box_rows) {
  const CUtensorMapDataType dt = sizeof(T) == 8 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT64 : CU_TENSOR_MAP_DATA_TYPE_FLOAT32;
  return tma_encode_tile(map, dt, const_cast<Cx<T>*>(base), 2ull * ld, (uint64_t)Ny, (uint64_t)ld * sizeof(Cx<T>),
                         2u * CB, (uint32_t)box_rows);
}

// ---------------------------------------------------------------- device
__device__ __forceinline__ unsigned smem_u32(const void* p) {
  return static_cast<unsigned>(__cvta_generic_to_shared(p));
}
__device__ __forceinline__ void mbar_init(uint64_t* bar, unsigned count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_init_fence() {
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}
__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, unsigned bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes) : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, unsigned parity) {
  unsigned ok;
  asm volatile(
      "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
      : "=r"(ok)
      : "r"(smem_u32(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}
__device__ __forceinline__ unsigned long long global_ns() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %globaltimer;" : "=l"(t));
  return t;
}
// Waits for phase `parity` of the barrier for at most limit_ns nanoseconds of
// %globaltimer (the kernels take the limit from Tables::wait_ns, one second
// by default); false on timeout.
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t* bar, unsigned parity, unsigned long long limit_ns) {
  if (mbar_try_wait(bar, parity)) return true;
  const unsigned long long t0 = global_ns();
  while (true) {
    if (mbar_try_wait(bar, parity)) return true;
    if (global_ns() - t0 > limit_ns) return false;
  }
}
// Orders this thread's earlier generic-proxy shared-memory accesses before
// later async-proxy (TMA) accesses of the same memory.
__device__ __forceinline__ void fence_proxy_async_smem() {
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}
__device__ __forceinline__ void tma_load_3d(void* dst, const CUtensorMap* map, int x, int y, int z, uint64_t* bar) {
  asm volatile(
      "cp.async.bulk.tensor.3d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4}], [%5];"
      ::"r"(smem_u32(dst)), "l"(reinterpret_cast<unsigned long long>(map)), "r"(x), "r"(y), "r"(z), "r"(smem_u32(bar))
      : "memory");
}
__device__ __forceinline__ void tma_load_2d(void* dst, const CUtensorMap* map, int x, int y, uint64_t* bar) {
  asm volatile(
      "cp.async.bulk.tensor.2d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], [%4];"
      ::"r"(smem_u32(dst)), "l"(reinterpret_cast<unsigned long long>(map)), "r"(x), "r"(y), "r"(smem_u32(bar))
      : "memory");
}

}  // namespace tara
