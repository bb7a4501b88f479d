// pb_reduce.cuh -- deterministic two-level reductions.
//
// Level 1: every block reduces its threads' partial sums in a fixed order
// and writes one partial vector to scratch[blockIdx.x][0..nout).
// Level 2: the last block to finish (arrival counter) sums the partial
// vectors in block order and writes the result.  The summation order never
// depends on scheduling, so results are bitwise reproducible run to run for
// a given launch shape.
#pragma once
#include <cuda_runtime.h>

namespace pb {

template <class T>
struct Acc;  // accumulation type
template <>
struct Acc<double> { typedef double type; };
template <>
struct Acc<float> { typedef float type; };

// Called by ALL threads of the block after the block partial has been written
// to part[blockIdx.x*nout + o].  Returns true in the one block that performed
// the final reduction (its threads wrote out[o] = alpha*sum + beta*out[o],
// with out[o] not read when beta == 0).
template <class T>
__device__ __forceinline__ bool last_block_reduce(const T* part, int nout, int nblocks,
                                                  unsigned int* counter, T* out,
                                                  int64_t out_stride_rows, int out_rows,
                                                  int64_t ld_out, T alpha, T beta)
{
  __shared__ bool am_last;
  __threadfence();
  __syncthreads();
  if (threadIdx.x == 0) {
    unsigned int prev = atomicAdd(counter, 1u);
    am_last = (prev == (unsigned int)nblocks - 1);
  }
  __syncthreads();
  if (!am_last) return false;
  __threadfence();
  // out index o -> (row = o % out_rows, col = o / out_rows) for matrix outputs
  for (int o = threadIdx.x; o < nout; o += blockDim.x) {
    T s = T(0);
    for (int b = 0; b < nblocks; b++) s += __ldcg(part + (int64_t)b * nout + o);
    int r = o % out_rows, c = o / out_rows;
    T* dst = out + r * out_stride_rows + (int64_t)c * ld_out;
    *dst = (beta == T(0)) ? alpha * s : alpha * s + beta * (*dst);
  }
  if (threadIdx.x == 0) *counter = 0u;  // ready for the next launch
  return true;
}

}  // namespace pb
