// pb_spmmv.cuh -- SELL-C-sigma sparse matrix times row-major block vector.
//
//   Y = alpha*(A + diag(shifts)) X + beta*Y          (sparseMat_times_mvec*,
//                                                     phist_kernels_decl.h:651-667)
//   optional epilogues in the same pass:
//     WdotW[j] = Y_j'Y_j,  VdotW[j] = X_j'Y_j          (fused_spmv_mvdot)
//     U = gamma*Y + delta*U                           (fused_spmv_mvdot_mvadd)
//   (phist_kernels_fused_decl.h:45-80)
//
// Thread mapping: a SELL row is handled by TPR consecutive threads, each
// owning VPT of the block vector's columns; the row's entries are streamed
// chunk-column by chunk-column (val/col reads are coalesced across the C rows
// of a chunk), the X rows they address are gathered with 16-byte vector loads
// (columns interleaved across the TPR threads so one warp-wide load covers a
// contiguous segment of each X row).  Arithmetic follows the builtin loop of
// spmvm_kernels.F90:494-523: tmp = shift*x_i, then the row's entries in stored
// order, then y = alpha*tmp + beta*y.
#pragma once
#include "pb_core.hpp"
#include "pb_reduce.cuh"

namespace pb {

template <class T>
struct SellDev {
  int64_t nrows;      // original rows
  int64_t nchunks;
  int C;
  const int64_t* __restrict__ chunk_ptr;
  const int32_t* __restrict__ chunk_len;
  const int32_t* __restrict__ col;
  const T* __restrict__ val;
  const int32_t* __restrict__ perm;  // nullptr: identity
};

template <class T>
struct SpmvArgs {
  T alpha, beta;
  int has_shift;                 // shifts sh[0..nvec) present
  T sh[32];                      // per-column shifts of this column tile
  const T* __restrict__ x;
  int64_t ldx;
  T* y;
  int64_t ldy;
  int nvec;                      // columns actually present (<= NV)
  int col0;                      // first column of this launch (column tiles)
  // epilogues
  int want_wdw, want_vdw;
  T* part;                       // per-block partials [grid][2*NV]
  unsigned int* counter;
  T* dots_out;                   // device [2*NV]: WdotW then VdotW
  T gamma, delta;
  T* u;
  int64_t ldu;
  // fused Gram products of the prefetching kernel (pb_spmmv_pf.cuh):
  // per-block partial sums of W'W (gram_w) and V'W (gram_v), NV*NV each;
  // store_y = 0 computes W only for the products (W = NULL in PHIST's call)
  T* gram_w;
  T* gram_v;
  int no_store;
};

template <class T, int W>
struct VecLd;
template <>
struct VecLd<double, 2> {
  static __device__ __forceinline__ void ld(const double* p, double* o)
  {
    double2 v = __ldg(reinterpret_cast<const double2*>(p));
    o[0] = v.x; o[1] = v.y;
  }
  static __device__ __forceinline__ void ld_plain(const double* p, double* o)
  {
    double2 v = *reinterpret_cast<const double2*>(p);
    o[0] = v.x; o[1] = v.y;
  }
  static __device__ __forceinline__ void ld_ordered(const double* p, double* o)
  {
    asm volatile("ld.global.nc.v2.f64 {%0, %1}, [%2];\n" : "=d"(o[0]), "=d"(o[1]) : "l"(p));
  }
  static __device__ __forceinline__ void st(double* p, const double* o)
  {
    *reinterpret_cast<double2*>(p) = make_double2(o[0], o[1]);
  }
};
// 256-bit forms (sm_100): one load or store moves 32 bytes
template <>
struct VecLd<double, 4> {
  static __device__ __forceinline__ void ld(const double* p, double* o) { ld_ordered(p, o); }
  static __device__ __forceinline__ void ld_plain(const double* p, double* o)
  {
    asm volatile("ld.global.v4.f64 {%0, %1, %2, %3}, [%4];\n"
                 : "=d"(o[0]), "=d"(o[1]), "=d"(o[2]), "=d"(o[3])
                 : "l"(p));
  }
  static __device__ __forceinline__ void ld_ordered(const double* p, double* o)
  {
    asm volatile("ld.global.nc.v4.f64 {%0, %1, %2, %3}, [%4];\n"
                 : "=d"(o[0]), "=d"(o[1]), "=d"(o[2]), "=d"(o[3])
                 : "l"(p));
  }
  static __device__ __forceinline__ void st(double* p, const double* o)
  {
    asm volatile("st.global.v4.f64 [%0], {%1, %2, %3, %4};\n" ::"l"(p), "d"(o[0]), "d"(o[1]), "d"(o[2]), "d"(o[3])
                 : "memory");
  }
};
template <>
struct VecLd<float, 8> {
  static __device__ __forceinline__ void ld(const float* p, float* o) { ld_ordered(p, o); }
  static __device__ __forceinline__ void ld_plain(const float* p, float* o)
  {
    asm volatile("ld.global.v8.f32 {%0, %1, %2, %3, %4, %5, %6, %7}, [%8];\n"
                 : "=f"(o[0]), "=f"(o[1]), "=f"(o[2]), "=f"(o[3]), "=f"(o[4]), "=f"(o[5]), "=f"(o[6]), "=f"(o[7])
                 : "l"(p));
  }
  static __device__ __forceinline__ void ld_ordered(const float* p, float* o)
  {
    asm volatile("ld.global.nc.v8.f32 {%0, %1, %2, %3, %4, %5, %6, %7}, [%8];\n"
                 : "=f"(o[0]), "=f"(o[1]), "=f"(o[2]), "=f"(o[3]), "=f"(o[4]), "=f"(o[5]), "=f"(o[6]), "=f"(o[7])
                 : "l"(p));
  }
  static __device__ __forceinline__ void st(float* p, const float* o)
  {
    asm volatile("st.global.v8.f32 [%0], {%1, %2, %3, %4, %5, %6, %7, %8};\n" ::"l"(p), "f"(o[0]), "f"(o[1]),
                 "f"(o[2]), "f"(o[3]), "f"(o[4]), "f"(o[5]), "f"(o[6]), "f"(o[7])
                 : "memory");
  }
};
template <>
struct VecLd<float, 4> {
  static __device__ __forceinline__ void ld(const float* p, float* o)
  {
    float4 v = __ldg(reinterpret_cast<const float4*>(p));
    o[0] = v.x; o[1] = v.y; o[2] = v.z; o[3] = v.w;
  }
  static __device__ __forceinline__ void ld_plain(const float* p, float* o)
  {
    float4 v = *reinterpret_cast<const float4*>(p);
    o[0] = v.x; o[1] = v.y; o[2] = v.z; o[3] = v.w;
  }
  static __device__ __forceinline__ void ld_ordered(const float* p, float* o)
  {
    asm volatile("ld.global.nc.v4.f32 {%0, %1, %2, %3}, [%4];\n"
                 : "=f"(o[0]), "=f"(o[1]), "=f"(o[2]), "=f"(o[3])
                 : "l"(p));
  }
  static __device__ __forceinline__ void st(float* p, const float* o)
  {
    *reinterpret_cast<float4*>(p) = make_float4(o[0], o[1], o[2], o[3]);
  }
};
template <>
struct VecLd<float, 2> {
  static __device__ __forceinline__ void ld(const float* p, float* o)
  {
    float2 v = __ldg(reinterpret_cast<const float2*>(p));
    o[0] = v.x; o[1] = v.y;
  }
  static __device__ __forceinline__ void ld_plain(const float* p, float* o)
  {
    float2 v = *reinterpret_cast<const float2*>(p);
    o[0] = v.x; o[1] = v.y;
  }
  static __device__ __forceinline__ void ld_ordered(const float* p, float* o)
  {
    asm volatile("ld.global.nc.v2.f32 {%0, %1}, [%2];\n" : "=f"(o[0]), "=f"(o[1]) : "l"(p));
  }
  static __device__ __forceinline__ void st(float* p, const float* o)
  {
    *reinterpret_cast<float2*>(p) = make_float2(o[0], o[1]);
  }
};
__device__ __forceinline__ void ld_ordered1(const double* p, double* o)
{
  asm volatile("ld.global.nc.f64 %0, [%1];\n" : "=d"(o[0]) : "l"(p));
}
__device__ __forceinline__ void ld_ordered1(const float* p, float* o)
{
  asm volatile("ld.global.nc.f32 %0, [%1];\n" : "=f"(o[0]) : "l"(p));
}
__device__ __forceinline__ void reg_fence(double& v) { asm volatile("" : "+d"(v)); }
__device__ __forceinline__ void reg_fence(float& v) { asm volatile("" : "+f"(v)); }
template <class T>
struct VecLd1 {
  static __device__ __forceinline__ void ld(const T* p, T* o) { o[0] = __ldg(p); }
  static __device__ __forceinline__ void ld_ordered(const T* p, T* o) { ld_ordered1(p, o); }
  static __device__ __forceinline__ void ld_plain(const T* p, T* o) { o[0] = *p; }
  static __device__ __forceinline__ void st(T* p, const T* o) { *p = o[0]; }
};
template <class T, int W>
struct Vec : VecLd<T, W> {};
template <>
struct Vec<double, 1> : VecLd1<double> {};
template <>
struct Vec<float, 1> : VecLd1<float> {};

// column handled by (lane-in-row s, vector v, element w)
template <int TPR, int VW>
__device__ __forceinline__ int spmv_col(int s, int v, int w)
{
  return VW * (s + v * TPR) + w;
}

constexpr int SPMV_BS = 256;

// KMAX > 0: every chunk of the matrix is at most KMAX entries long (fully
// unrolled row loop); KMAX == 0: any length (runtime loop).
// CC > 0: the chunk height is the compile-time constant CC (entry offsets
// become immediates); CC == 0: read from A.C.
// DOTS: the fused column dots are computed (bounded grid walking the row
// tiles); otherwise one row tile per block and no dot code.
template <class T, int NV, int TPR, bool VEC, int KMAX, int CC, bool DOTS>
__global__ void __launch_bounds__(SPMV_BS)
k_sell_spmmv(SellDev<T> A, SpmvArgs<T> p)
{
  constexpr int VPT = NV / TPR;                              // columns per thread
  constexpr int VWMAX = 16 / sizeof(T);
  constexpr int VW = VEC ? (VPT < VWMAX ? VPT : VWMAX) : 1;  // vector width
  constexpr int NVV = VPT / VW;                               // vectors per thread
  constexpr int RPB = SPMV_BS / TPR;                          // rows per block
  typedef typename Acc<T>::type AT;

  const int tid = threadIdx.x;
  const int s = tid % TPR;
  const int C = CC > 0 ? CC : A.C;
  const int nv = p.nvec;
  const T* __restrict__ x = p.x + p.col0;
  T wdw[VPT], vdw[VPT];  // column dot partials of this thread
#pragma unroll
  for (int q = 0; q < VPT; q++) { wdw[q] = T(0); vdw[q] = T(0); }

  // tiles of RPB SELL rows; one tile per block unless the grid was bounded
  // (fused dots: fewer blocks, fewer partial vectors to combine)
  const int64_t ntiles = (A.nchunks * (int64_t)C + RPB - 1) / RPB;
  const int64_t tstep = DOTS ? (int64_t)gridDim.x : ntiles;
  for (int64_t tile = blockIdx.x; tile < ntiles; tile += tstep) {
  const int64_t r = tile * RPB + tid / TPR;  // SELL row
  const int64_t i = (r < A.nrows) ? (A.perm ? (int64_t)A.perm[r] : r) : -1;

  AT acc[VPT];
  T xi[VPT];
#pragma unroll
  for (int q = 0; q < VPT; q++) { acc[q] = AT(0); xi[q] = T(0); }

  if (i >= 0 && (p.has_shift || p.want_vdw)) {
#pragma unroll
    for (int v = 0; v < NVV; v++) {
      const int c = spmv_col<TPR, VW>(s, v, 0);
      if (VEC || c < nv) Vec<T, VW>::ld(x + i * p.ldx + c, &xi[v * VW]);
    }
    if (p.has_shift) {
#pragma unroll
      for (int v = 0; v < NVV; v++)
#pragma unroll
        for (int w = 0; w < VW; w++) {
          const int c = spmv_col<TPR, VW>(s, v, w);
          if (VEC || c < nv) acc[v * VW + w] = AT(p.sh[c]) * AT(xi[v * VW + w]);
        }
    }
  }

  if (KMAX > 0 && r < A.nchunks * (int64_t)C) {
    // chunk length <= KMAX: every entry's val/col load of the row is issued
    // first, then every X-row gather, then the FMAs in entry order -- the
    // loads of one row are all in flight together
    const int64_t ch = r / C;
    const int l = (int)(r - ch * C);
    const int64_t base = A.chunk_ptr[ch] + l;
    const int len = A.chunk_len[ch];
    T av[KMAX > 0 ? KMAX : 1];
    int cv[KMAX > 0 ? KMAX : 1];
#pragma unroll
    for (int k = 0; k < KMAX; k++) {
      av[k] = T(0);
      cv[k] = 0;
      if (k < len) {
        av[k] = __ldcs(A.val + base + (int64_t)k * C);
        cv[k] = __ldcs(A.col + base + (int64_t)k * C);
      }
    }
    // entries past the chunk length gather the row of entry 0 again (an L1
    // hit) and are not accumulated: the gathers carry no predicate and can
    // all be issued before the first one is consumed
#pragma unroll
    for (int k = 1; k < KMAX; k++)
      if (k >= len) cv[k] = cv[0];
    T xv[KMAX > 0 ? KMAX : 1][VPT];
#pragma unroll
    for (int k = 0; k < KMAX; k++) {
      const T* xr = x + (int64_t)cv[k] * p.ldx;
#pragma unroll
      for (int v = 0; v < NVV; v++) {
        const int c = spmv_col<TPR, VW>(s, v, 0);
        if (VEC || c < nv) {
          Vec<T, VW>::ld_ordered(xr + c, &xv[k][v * VW]);
        } else {
#pragma unroll
          for (int w = 0; w < VW; w++) xv[k][v * VW + w] = T(0);
        }
      }
    }
    // compiler fence: every gathered value is an operand here, so the
    // accumulation below cannot be interleaved with (and wait on) the loads
#pragma unroll
    for (int k = 0; k < KMAX; k++)
#pragma unroll
      for (int q = 0; q < VPT; q++) reg_fence(xv[k][q]);
#pragma unroll
    for (int k = 0; k < KMAX; k++)
      if (k < len)
#pragma unroll
        for (int q = 0; q < VPT; q++) acc[q] += AT(av[k]) * AT(xv[k][q]);
  } else if (r < A.nchunks * (int64_t)C) {
    const int64_t ch = r / C;
    const int l = (int)(r - ch * C);
    const int64_t base = A.chunk_ptr[ch] + l;
    const int len = A.chunk_len[ch];
#pragma unroll 4
    for (int k = 0; k < len; k++) {
      const T a = __ldcs(A.val + base + (int64_t)k * C);
      const int64_t cj = __ldcs(A.col + base + (int64_t)k * C);
      const T* xr = x + cj * p.ldx;
#pragma unroll
      for (int v = 0; v < NVV; v++) {
        const int c = spmv_col<TPR, VW>(s, v, 0);
        if (VEC || c < nv) {
          T xv[VW];
          Vec<T, VW>::ld(xr + c, xv);
#pragma unroll
          for (int w = 0; w < VW; w++) acc[v * VW + w] += AT(a) * AT(xv[w]);
        }
      }
    }
  }

  if (i >= 0) {
    T* yr = p.y + p.col0 + i * p.ldy;
#pragma unroll
    for (int v = 0; v < NVV; v++) {
      const int c = spmv_col<TPR, VW>(s, v, 0);
      if (!(VEC || c < nv)) continue;
      T yv[VW];
      if (p.beta != T(0)) {
        Vec<T, VW>::ld_plain(yr + c, yv);
#pragma unroll
        for (int w = 0; w < VW; w++) yv[w] = T(AT(p.alpha) * acc[v * VW + w] + AT(p.beta) * AT(yv[w]));
      } else {
#pragma unroll
        for (int w = 0; w < VW; w++) yv[w] = T(AT(p.alpha) * acc[v * VW + w]);
      }
      Vec<T, VW>::st(yr + c, yv);
#pragma unroll
      for (int w = 0; w < VW; w++) {
        if (DOTS) {
          wdw[v * VW + w] += yv[w] * yv[w];
          vdw[v * VW + w] += xi[v * VW + w] * yv[w];
        }
      }
      if (p.u) {
        T* ur = p.u + p.col0 + i * p.ldu + c;
        T uv[VW];
        if (p.delta != T(0)) {
          Vec<T, VW>::ld_plain(ur, uv);
#pragma unroll
          for (int w = 0; w < VW; w++) uv[w] = p.gamma * yv[w] + p.delta * uv[w];
        } else {
#pragma unroll
          for (int w = 0; w < VW; w++) uv[w] = p.gamma * yv[w];
        }
        Vec<T, VW>::st(ur, uv);
      }
    }
  }
  }  // tiles

  if (!DOTS) return;

  // ---- block reduction of the column dots, fixed order ----
  // lanes with equal s hold the same columns: butterfly over offsets >= TPR
#pragma unroll
  for (int off = 16; off >= TPR; off >>= 1) {
#pragma unroll
    for (int q = 0; q < VPT; q++) {
      wdw[q] += __shfl_xor_sync(0xffffffffu, wdw[q], off);
      vdw[q] += __shfl_xor_sync(0xffffffffu, vdw[q], off);
    }
  }
  constexpr int NW = SPMV_BS / 32;
  __shared__ T red[NW][2 * NV];
  const int lane = tid & 31, warp = tid >> 5;
  if (lane < TPR) {
#pragma unroll
    for (int v = 0; v < NVV; v++)
#pragma unroll
      for (int w = 0; w < VW; w++) {
        const int c = spmv_col<TPR, VW>(lane, v, w);
        red[warp][c] = wdw[v * VW + w];
        red[warp][NV + c] = vdw[v * VW + w];
      }
  }
  __syncthreads();
  T* part = p.part + (int64_t)blockIdx.x * 2 * NV;
  if (tid < 2 * NV) {
    T sacc = T(0);
#pragma unroll
    for (int w = 0; w < NW; w++) sacc += red[w][tid];
    part[tid] = sacc;
  }
  last_block_reduce<T>(p.part, 2 * NV, gridDim.x, p.counter, p.dots_out, 1, 2 * NV, 0, T(1), T(0));
}

// Y = alpha*(s1_j A1 + s2_j A2) X + beta*Y in one pass (fused_spmv_pair,
// phist_kernels_fused_decl.h:45-48).  Per element the arithmetic of PHIST's
// composition (common/kernels_no_fused_spmv_pair.cpp): t1 = alpha*(A1 x)_ij,
// y = s1_j*t1 + beta*y, t2 = alpha*(A2 x)_ij, y = s2_j*t2 + y, each product
// summed in stored (column) order as in spmvm_kernels.F90:494-523.  Thread
// per (row, column); the two matrices may have different SELL layouts, so
// each row is found through the inverse row permutation.
template <class T>
struct PairArgs {
  SellDev<T> A1, A2;
  const int32_t* iperm1;
  const int32_t* iperm2;
  const int32_t* rlen1;
  const int32_t* rlen2;
  T alpha, beta;
  T s1[32], s2[32];
  const T* x;
  int64_t ldx;
  T* y;
  int64_t ldy;
  int64_t n;
  int nvec;  // columns of this launch (<= 32), starting at x and y
};

template <class T>
__device__ __forceinline__ typename Acc<T>::type sell_row_dot(const SellDev<T>& A, const int32_t* iperm,
                                                              const int32_t* rlen, int64_t i, const T* x,
                                                              int64_t ldx, int j)
{
  typedef typename Acc<T>::type AT;
  const int64_t r = iperm ? (int64_t)iperm[i] : i;
  const int64_t ch = r / A.C;
  const int64_t base = A.chunk_ptr[ch] + (r - ch * A.C);
  const int len = rlen[r];
  AT acc = AT(0);
  for (int k = 0; k < len; k++) {
    const T a = __ldg(A.val + base + (int64_t)k * A.C);
    const int64_t c = __ldg(A.col + base + (int64_t)k * A.C);
    acc += AT(a) * AT(__ldg(x + c * ldx + j));
  }
  return acc;
}

template <class T>
__global__ void __launch_bounds__(256) k_sell_spmmv_pair(PairArgs<T> p)
{
  typedef typename Acc<T>::type AT;
  const int64_t tot = p.n * p.nvec;
  for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < tot; t += (int64_t)gridDim.x * blockDim.x) {
    const int64_t i = t / p.nvec;
    const int j = (int)(t - i * p.nvec);
    const AT a1 = sell_row_dot(p.A1, p.iperm1, p.rlen1, i, p.x, p.ldx, j);
    const AT a2 = sell_row_dot(p.A2, p.iperm2, p.rlen2, i, p.x, p.ldx, j);
    const T t1 = T(AT(p.alpha) * a1);
    const T t2 = T(AT(p.alpha) * a2);
    T* yp = p.y + i * p.ldy + j;
    T y = (p.beta == T(0)) ? p.s1[j] * t1 : p.s1[j] * t1 + p.beta * *yp;
    y = p.s2[j] * t2 + y;
    *yp = y;
  }
}

// alpha == 0 / empty matrix: Y = beta*Y (crsmat_module.F90:1508-1511)
template <class T>
__global__ void k_scale_rows(T* y, int64_t ldy, int64_t n, int nvec, T beta)
{
  const int64_t tot = n * nvec;
  for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < tot;
       t += (int64_t)gridDim.x * blockDim.x) {
    const int64_t i = t / nvec;
    const int j = (int)(t - i * nvec);
    y[i * ldy + j] = (beta == T(0)) ? T(0) : beta * y[i * ldy + j];
  }
}

}  // namespace pb
