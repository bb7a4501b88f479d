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
// Sum of v over the threads t == c (mod w) of a 256-thread block, for each
// residue c < w (w a power of two <= 256), returned to thread c; other threads
// get an unspecified value.  Fixed order: a butterfly over the lanes of each
// warp, then the warp (or w-strided) partial sums in ascending order.  red
// holds 256 entries; the caller syncs before it reuses red.
template <class T>
__device__ __forceinline__ T block_sum_mod(T v, int w, T* red)
{
  for (int off = 16; off >= w; off >>= 1) v += __shfl_xor_sync(0xffffffffu, v, off);
  red[threadIdx.x] = v;
  __syncthreads();
  T s = T(0);
  if ((int)threadIdx.x < w) {
    const int step = w > 32 ? w : 32;
    for (int k = threadIdx.x; k < 256; k += step) s += red[k];
  }
  return s;
}

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
      // the G group sums of each output are added in a fixed tree: groups
      // [P, G) onto [0, G-P) (P the largest power of two <= G), then halves
      __syncthreads();
      if (g < G) red[g * span + oo] = s;
      __syncthreads();
      int P = 1;
      while (2 * P <= G) P *= 2;
      if (P < G) {
        if (g < G - P) red[g * span + oo] += red[(g + P) * span + oo];
        __syncthreads();
      }
      for (int h = P / 2; h >= 1; h >>= 1) {
        if (g < h) red[g * span + oo] += red[(g + h) * span + oo];
        __syncthreads();
      }
      if (threadIdx.x < span) s = red[threadIdx.x];
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

namespace pb {

// Second pass of a two-level reduction for many outputs.  The last-block
// reduction above runs on one SM; with nout*nblocks partials in the tens of
// thousands that SM's serial chains of L2 loads dominate the call.  Here a
// block owns 32 consecutive outputs (lanes: coalesced rows of the partials)
// and splits the partial blocks into 8 fixed chunks (warps); chunk sums are
// combined in chunk order, so the result is independent of timing.
//   out(i, j) = alpha * sum_b part[b*nout + o] + beta * out(i, j),
//   o = i + j*mrows, out(i, j) at C[i + j*ldc]
template <class T>
__device__ __forceinline__ void k_reduce_partials_body(const T* __restrict__ part, int nblocks, int nout, T* C,
                                                       int mrows, int64_t ldc, T alpha, T beta)
{
  __shared__ T red[8][32];
  const int ol = threadIdx.x & 31, ch = threadIdx.x >> 5;
  const int o = blockIdx.x * 32 + ol;
  T s = T(0);
  if (o < nout) {
    const int per = (nblocks + 7) / 8;
    const int b0 = ch * per;
    const int b1 = min(nblocks, b0 + per);
    T s0 = T(0), s1 = T(0), s2 = T(0), s3 = T(0);
    int b = b0;
    for (; b + 4 <= b1; b += 4) {
      s0 += __ldcg(part + (int64_t)b * nout + o);
      s1 += __ldcg(part + (int64_t)(b + 1) * nout + o);
      s2 += __ldcg(part + (int64_t)(b + 2) * nout + o);
      s3 += __ldcg(part + (int64_t)(b + 3) * nout + o);
    }
    for (; b < b1; b++) s0 += __ldcg(part + (int64_t)b * nout + o);
    s = (s0 + s1) + (s2 + s3);
  }
  red[ch][ol] = s;
  __syncthreads();
  if (ch == 0 && o < nout) {
    T t = T(0);
#pragma unroll
    for (int c = 0; c < 8; c++) t += red[c][ol];
    T* dst = C + (o % mrows) + (int64_t)(o / mrows) * ldc;
    *dst = (beta == T(0)) ? alpha * t : alpha * t + beta * *dst;
  }
}

template <class T>
__global__ void __launch_bounds__(256) k_reduce_partials(const T* __restrict__ part, int nblocks, int nout,
                                                         T* C, int mrows, int64_t ldc, T alpha, T beta)
{
  k_reduce_partials_body<T>(part, nblocks, nout, C, mrows, ldc, alpha, beta);
}

}  // namespace pb
