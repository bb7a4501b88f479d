// pb_tma.cuh -- Tensor Memory Accelerator (TMA) staging for the block-vector
// kernels on sm_100a.
//
// A row-major block vector (nrows x ncols, leading dimension ld) is described
// to the TMA unit by a 2D tensor map (dims {ncols, nrows}, row stride ld);
// one cp.async.bulk.tensor.2d instruction moves a box of R rows x BOX
// columns into shared memory.  Columns past ncols and rows past nrows are
// filled with zeros by the hardware, so widths are padded for free.  Copies
// complete on an mbarrier (expect_tx / complete_tx); every wait is bounded
// and a timed-out wait is reported through an error word in mapped host
// memory (plain store; the host reads it after its next stream
// synchronisation) instead of hanging the GPU.
//
// Only plain (non-multicast) loads from this GPU's own memory are issued.
#pragma once
#include <cuda.h>
#include <cuda_runtime.h>

#include <cstdint>

namespace pb {

// error codes written to the device error word
enum : int { PB_DEVERR_NONE = 0, PB_DEVERR_MBAR_TIMEOUT = 1 };

__device__ __forceinline__ unsigned smem_u32(const void* p)
{
  return (unsigned)__cvta_generic_to_shared(p);
}

__device__ __forceinline__ void mbar_init(uint64_t* bar, unsigned count)
{
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;\n" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}

// make the initialised barriers visible to the async (TMA) proxy
__device__ __forceinline__ void mbar_fence_init()
{
  asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
}

__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t* bar, unsigned bytes)
{
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;\n" ::"r"(smem_u32(bar)), "r"(bytes)
               : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, unsigned parity)
{
  unsigned ok;
  asm volatile(
      "{\n"
      ".reg .pred p;\n"
      "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n"
      "selp.u32 %0, 1, 0, p;\n"
      "}\n"
      : "=r"(ok)
      : "r"(smem_u32(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}

__device__ __forceinline__ uint64_t global_ns()
{
  uint64_t t;
  asm volatile("mov.u64 %0, %%globaltimer;\n" : "=l"(t));
  return t;
}

// Bounded wait for the phase with the given parity: gives up after about one
// second of wall time (far beyond any copy of a few tens of KiB), stores the
// error code and returns false.
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, unsigned parity, int* err)
{
  if (mbar_try_wait(bar, parity)) return true;
  const uint64_t t0 = global_ns();
  for (;;) {
    for (int it = 0; it < 256; it++)
      if (mbar_try_wait(bar, parity)) return true;
    if (global_ns() - t0 > 1000000000ull) break;
  }
  if (err) *(volatile int*)err = PB_DEVERR_MBAR_TIMEOUT;
  return false;
}

// 2D box load: box at (x = column, y = row) of the tensor map into dst,
// completing on bar.  x must be a multiple of 16 bytes' worth of elements
// (the kernels here always load from column 0).
__device__ __forceinline__ void tma_load_2d(void* dst, const CUtensorMap* map, int x, int y, uint64_t* bar)
{
  asm volatile(
      "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], "
      "[%4];\n" ::"r"(smem_u32(dst)),
      "l"((uint64_t)map), "r"(x), "r"(y), "r"(smem_u32(bar))
      : "memory");
}

__device__ __forceinline__ void tma_prefetch_desc(const CUtensorMap* map)
{
  asm volatile("prefetch.tensormap [%0];\n" ::"l"((uint64_t)map) : "memory");
}

}  // namespace pb
