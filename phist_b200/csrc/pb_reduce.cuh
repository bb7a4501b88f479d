// pb_reduce.cuh -- deterministic two-level reductions.
//
// Level 1: every block reduces its threads' partial sums in a fixed order
// and writes one partial vector to scratch[blockIdx.x][0..nout).
// Level 2: the last block to finish (arrival counter) sums the partial
// vectors.  All of its threads take part: with G = blockDim/nout groups,
// thread (g, o) sums the partials of blocks g, g+G, g+2G, ... in increasing
// block order, then thread o adds the G group sums in increasing g.  The
// summation order depends only on (nblocks, blockDim, nout), never on
// scheduling, so results are bitwise reproducible run to run for a given
// launch shape.
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
// with out[o] not read when beta == 0).  Output o goes to
// out[(o % out_rows)*out_stride_rows + (o / out_rows)*ld_out].
// Outputs whose row is >= vrows or whose column is >= vcols are padding and
// are not written.
template <class T>
__device__ __forceinline__ bool last_block_reduce(const T* part, int nout, int nblocks,
                                                  unsigned int* counter, T* out,
                                                  int64_t out_stride_rows, int out_rows,
                                                  int64_t ld_out, T alpha, T beta,
                                                  int vrows = 1 << 30, int vcols = 1 << 30)
{
  __shared__ bool am_last;
  __shared__ T red[256];  // all callers launch at most 256 threads per block
  __threadfence();
  __syncthreads();
  if (threadIdx.x == 0) {
    unsigned int prev = atomicAdd(counter, 1u);
    am_last = (prev == (unsigned int)nblocks - 1);
  }
  __syncthreads();
  if (!am_last) return false;
  __threadfence();
  const int nt = blockDim.x;
  const int G = (nout < nt) ? (nt / nout) : 1;  // groups of blocks
  for (int o0 = 0; o0 < nout; o0 += nt) {
    // thread t: output o = o0 + t % nout', group g = t / nout'
    const int span = (nout - o0 < nt) ? (nout - o0) : nt;
    const int g = threadIdx.x / span, oo = threadIdx.x - g * span;
    T s = T(0);
    if (g < G) {
      const T* p = part + o0 + oo;
      int b = g;
      // 4 independent loads in flight, added in block order
      for (; b + 3 * G < nblocks; b += 4 * G) {
        const T v0 = __ldcg(p + (int64_t)b * nout);
        const T v1 = __ldcg(p + (int64_t)(b + G) * nout);
        const T v2 = __ldcg(p + (int64_t)(b + 2 * G) * nout);
        const T v3 = __ldcg(p + (int64_t)(b + 3 * G) * nout);
        s += v0;
        s += v1;
        s += v2;
        s += v3;
      }
      for (; b < nblocks; b += G) s += __ldcg(p + (int64_t)b * nout);
    }
    if (G > 1) {
      __syncthreads();
      if (g < G) red[g * span + oo] = s;
      __syncthreads();
      if (threadIdx.x < span) {
        s = T(0);
        for (int gg = 0; gg < G; gg++) s += red[gg * span + threadIdx.x];
      }
    }
    if (threadIdx.x < span) {
      const int o = o0 + threadIdx.x;
      const int r = o % out_rows, c = o / out_rows;
      if (r < vrows && c < vcols) {
        T* dst = out + r * out_stride_rows + (int64_t)c * ld_out;
        *dst = (beta == T(0)) ? alpha * s : alpha * s + beta * (*dst);
      }
    }
  }
  if (threadIdx.x == 0) *counter = 0u;  // ready for the next launch
  return true;
}

}  // namespace pb
