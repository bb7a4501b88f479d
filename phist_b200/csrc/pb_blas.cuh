// pb_blas.cuh -- BLAS1-type kernels on row-major block vectors
// (phist_kernels_decl.h:448-548): fill, random, scale, axpby, element-wise
// product, column dots, block copies, precision conversion.  All are pure
// streaming kernels bound by HBM bandwidth; the column dots use the
// deterministic two-level reduction of pb_reduce.cuh.
#pragma once
#include "pb_core.hpp"
#include "pb_reduce.cuh"

namespace pb {

// grid-stride over all (row, col) elements of an n x nvec view
#define PB_FOR_ELEMS(n, nvec, i, j)                                                  \
  for (int64_t t_ = blockIdx.x * (int64_t)blockDim.x + threadIdx.x, tot_ = (n) * (nvec); \
       t_ < tot_; t_ += (int64_t)gridDim.x * blockDim.x)                              \
    for (int64_t i = t_ / (nvec), j = t_ - i * (nvec), once_ = 0; once_ < 1; once_++)

template <class T>
__global__ void k_put_value(T* v, int64_t ld, int64_t n, int nvec, T val)
{
  PB_FOR_ELEMS(n, nvec, i, j) v[i * ld + j] = val;
}

// counter-based uniform[-1,1) numbers: a splitmix64 hash of (seed, global
// row, column), so the value of element (i,j) depends on nothing else
__device__ __host__ __forceinline__ uint64_t pb_mix64(uint64_t z)
{
  z += 0x9E3779B97F4A7C15ull;
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return z ^ (z >> 31);
}
__device__ __host__ __forceinline__ double pb_unif(uint64_t seed, uint64_t idx)
{
  const uint64_t h = pb_mix64(seed * 0x632BE59BD9B4E019ull + pb_mix64(idx));
  return (double)(h >> 11) * (1.0 / 9007199254740992.0) * 2.0 - 1.0;
}

template <class T>
__global__ void k_random(T* v, int64_t ld, int64_t n, int nvec, int64_t gcols, int col0,
                         uint64_t seed)
{
  PB_FOR_ELEMS(n, nvec, i, j) v[i * ld + j] = T(pb_unif(seed, (uint64_t)i * gcols + col0 + j));
}

template <class T>
__global__ void k_vscale(T* v, int64_t ld, int64_t n, int nvec, const T* __restrict__ s)
{
  PB_FOR_ELEMS(n, nvec, i, j) v[i * ld + j] *= s[j];
}

// Y = alpha_j X + beta Y; valpha == nullptr -> scalar alpha; beta == 0 -> Y not read
template <class T>
__global__ void k_axpby(const T* __restrict__ x, int64_t ldx, T* y, int64_t ldy, int64_t n,
                        int nvec, T alpha, const T* __restrict__ valpha, T beta)
{
  PB_FOR_ELEMS(n, nvec, i, j)
  {
    const T a = valpha ? valpha[j] : alpha;
    const T xv = (a == T(0)) ? T(0) : a * x[i * ldx + j];
    y[i * ldy + j] = (beta == T(0)) ? xv : xv + beta * y[i * ldy + j];
  }
}

// per-column coefficients passed by value (no host-to-device copy)
template <class T>
struct Coef64 {
  T v[64];
};

template <class T>
__global__ void k_axpby_v(const T* __restrict__ x, int64_t ldx, T* y, int64_t ldy, int64_t n,
                          int nvec, Coef64<T> alpha, T beta)
{
  PB_FOR_ELEMS(n, nvec, i, j)
  {
    const T a = alpha.v[j];
    const T xv = (a == T(0)) ? T(0) : a * x[i * ldx + j];
    y[i * ldy + j] = (beta == T(0)) ? xv : xv + beta * y[i * ldy + j];
  }
}

template <class T>
__global__ void k_vscale_v(T* v, int64_t ld, int64_t n, int nvec, Coef64<T> s)
{
  PB_FOR_ELEMS(n, nvec, i, j) v[i * ld + j] *= s.v[j];
}

// W(i,j) = alpha * V(i, bc ? 0 : j) * W(i,j)
template <class T>
__global__ void k_elemwise(const T* __restrict__ v, int64_t ldv, T* w, int64_t ldw, int64_t n,
                           int nvec, T alpha, int bcast)
{
  PB_FOR_ELEMS(n, nvec, i, j) w[i * ldw + j] = alpha * v[i * ldv + (bcast ? 0 : j)] * w[i * ldw + j];
}

template <class TI, class TO>
__global__ void k_copy(const TI* __restrict__ x, int64_t ldx, TO* y, int64_t ldy, int64_t n,
                       int nvec)
{
  PB_FOR_ELEMS(n, nvec, i, j) y[i * ldy + j] = TO(x[i * ldx + j]);
}

// column dots d[j] = sum_i V(i,j) W(i,j), j < nvec <= 64.  Each thread walks
// rows with a grid stride and keeps NV partial sums (columns masked to nvec).
template <class T, int NV>
__global__ void __launch_bounds__(256)
k_coldot(const T* __restrict__ v, int64_t ldv, const T* __restrict__ w, int64_t ldw, int64_t n,
         int nvec, T* part, unsigned int* counter, T* out, int ext = 0)
{
  T acc[NV];
#pragma unroll
  for (int q = 0; q < NV; q++) acc[q] = T(0);
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x) {
#pragma unroll
    for (int q = 0; q < NV; q++)
      if (q < nvec) acc[q] += v[i * ldv + q] * w[i * ldw + q];
  }
#pragma unroll
  for (int off = 16; off >= 1; off >>= 1)
#pragma unroll
    for (int q = 0; q < NV; q++) acc[q] += __shfl_xor_sync(0xffffffffu, acc[q], off);
  __shared__ T red[8][NV];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  if (lane == 0)
#pragma unroll
    for (int q = 0; q < NV; q++) red[warp][q] = acc[q];
  __syncthreads();
  if (threadIdx.x < NV) {
    T s = T(0);
    for (int w2 = 0; w2 < (int)(blockDim.x >> 5); w2++) s += red[w2][threadIdx.x];
    part[(int64_t)blockIdx.x * NV + threadIdx.x] = s;
  }
  if (ext) return;  // second pass: k_reduce_partials
  last_block_reduce<T>(part, NV, gridDim.x, counter, out, 1, NV, 0, T(1), T(0));
}

// Column dots of two contiguous blocks (ld == nvec, nvec a power of two up
// to 64, 16-byte aligned) read as flat arrays with 16-byte vector loads:
// thread t owns the element pair starting at 2t of every chunk of
// 512*gridDim.x elements, i.e. always the same columns c = 2t mod nvec (and
// c + 1), so each thread keeps two partial sums.  Four chunks are loaded
// before they are consumed.  The block sum of column q adds the threads that
// own q in a fixed tree order; the cross-block sum is the usual fixed-order
// pass.
template <class T>
__global__ void __launch_bounds__(256)
k_coldot_flat(const T* __restrict__ v, const T* __restrict__ w, int64_t total, int nvec, T* part,
              unsigned int* counter, T* out, int ext)
{
  static_assert(sizeof(T) == 8, "double only");
  __shared__ T red[2][256];
  const int tid = threadIdx.x;
  const int64_t stride = (int64_t)gridDim.x * 512;
  T s0 = T(0), s1 = T(0);
  int64_t e = (int64_t)blockIdx.x * 512 + 2 * tid;
  for (; e + 3 * stride + 1 < total; e += 4 * stride) {
    double2 a[4], b[4];
#pragma unroll
    for (int u = 0; u < 4; u++) {
      a[u] = __ldg(reinterpret_cast<const double2*>(v + e + u * stride));
      b[u] = __ldg(reinterpret_cast<const double2*>(w + e + u * stride));
    }
#pragma unroll
    for (int u = 0; u < 4; u++) {
      s0 += a[u].x * b[u].x;
      s1 += a[u].y * b[u].y;
    }
  }
  for (; e + 1 < total; e += stride) {
    const double2 a = __ldg(reinterpret_cast<const double2*>(v + e));
    const double2 b = __ldg(reinterpret_cast<const double2*>(w + e));
    s0 += a.x * b.x;
    s1 += a.y * b.y;
  }
  if (e < total) s0 += v[e] * w[e];  // odd total (nvec == 1 only)
  if (nvec == 1) {
    const T t = block_sum_mod<T>(s0 + s1, 1, red[0]);
    if (tid == 0) part[blockIdx.x] = t;
  } else {
    // threads t and t' own the same columns iff t == t' (mod nvec/2)
    const int half = nvec / 2;
    const T t0 = block_sum_mod<T>(s0, half, red[0]);
    const T t1 = block_sum_mod<T>(s1, half, red[1]);
    if (tid < half) {
      part[(int64_t)blockIdx.x * nvec + 2 * tid] = t0;
      part[(int64_t)blockIdx.x * nvec + 2 * tid + 1] = t1;
    }
  }
  if (ext) return;  // second pass: k_reduce_partials
  last_block_reduce<T>(part, nvec, gridDim.x, counter, out, 1, nvec, 0, T(1), T(0));
}

// compensated column dots (PHIST_ROBUST_REDUCTIONS): Dot2 of Ogita, Rump and
// Oishi per thread, partial (sum, error) pairs combined with TwoSum in a fixed
// order.  out[2*j] = high part, out[2*j+1] = low part.
__device__ __forceinline__ void pb_two_sum(double a, double b, double& s, double& e)
{
  s = a + b;
  const double z = s - a;
  e = (a - (s - z)) + (b - z);
}
template <int NV>
__global__ void __launch_bounds__(256)
k_coldot_prec(const double* __restrict__ v, int64_t ldv, const double* __restrict__ w,
              int64_t ldw, int64_t n, int nvec, double* part, unsigned int* counter, double* out)
{
  double s[NV], c[NV];
#pragma unroll
  for (int q = 0; q < NV; q++) { s[q] = 0.0; c[q] = 0.0; }
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x) {
#pragma unroll
    for (int q = 0; q < NV; q++)
      if (q < nvec) {
        const double x = v[i * ldv + q], y = w[i * ldw + q];
        const double p = x * y;
        const double ep = fma(x, y, -p);
        double t, et;
        pb_two_sum(s[q], p, t, et);
        s[q] = t;
        c[q] += ep + et;
      }
  }
  // butterfly combine of (s, c) pairs
#pragma unroll
  for (int off = 16; off >= 1; off >>= 1)
#pragma unroll
    for (int q = 0; q < NV; q++) {
      const double so = __shfl_xor_sync(0xffffffffu, s[q], off);
      const double co = __shfl_xor_sync(0xffffffffu, c[q], off);
      double t, et;
      pb_two_sum(s[q], so, t, et);
      s[q] = t;
      c[q] += co + et;
    }
  __shared__ double red[8][2 * NV];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  if (lane == 0)
#pragma unroll
    for (int q = 0; q < NV; q++) { red[warp][2 * q] = s[q]; red[warp][2 * q + 1] = c[q]; }
  __syncthreads();
  if (threadIdx.x < NV) {
    const int q = threadIdx.x;
    double ss = 0.0, cc = 0.0;
    for (int w2 = 0; w2 < (int)(blockDim.x >> 5); w2++) {
      double t, et;
      pb_two_sum(ss, red[w2][2 * q], t, et);
      ss = t;
      cc += red[w2][2 * q + 1] + et;
    }
    part[(int64_t)blockIdx.x * 2 * NV + 2 * q] = ss;
    part[(int64_t)blockIdx.x * 2 * NV + 2 * q + 1] = cc;
  }
  __shared__ bool am_last;
  __threadfence();
  __syncthreads();
  if (threadIdx.x == 0) am_last = (atomicAdd(counter, 1u) == gridDim.x - 1);
  __syncthreads();
  if (!am_last) return;
  __threadfence();
  if (threadIdx.x < NV) {
    const int q = threadIdx.x;
    double ss = 0.0, cc = 0.0;
    for (int b = 0; b < (int)gridDim.x; b++) {
      double t, et;
      pb_two_sum(ss, __ldcg(part + (int64_t)b * 2 * NV + 2 * q), t, et);
      ss = t;
      cc += __ldcg(part + (int64_t)b * 2 * NV + 2 * q + 1) + et;
    }
    double hi, lo;
    pb_two_sum(ss, cc, hi, lo);
    out[2 * q] = hi;
    out[2 * q + 1] = lo;
  }
  if (threadIdx.x == 0) *counter = 0u;
}

// sdMat (column-major) element-wise kernels on the device
template <class T>
__global__ void k_sd_copy(const T* __restrict__ a, int64_t lda, T* b, int64_t ldb, int nr, int nc,
                          int trans)
{
  for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < nr * nc; t += gridDim.x * blockDim.x) {
    const int i = t % nr, j = t / nr;
    b[i + j * ldb] = trans ? a[j + i * lda] : a[i + j * lda];
  }
}

}  // namespace pb
