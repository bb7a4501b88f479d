// pb_tile.cuh -- tall-skinny block products for widths 9..64 with
// asynchronous tile staging.
//
//  k_mvtmv_async : C = alpha*V'W + beta*C        (mvecT_times_mvec)
//  k_mvsd_async  : W = alpha*V*C + beta*W, or W(:,0:k) = W(:,0:m)*C in place
//                  (mvec_times_sdMat, mvec_times_sdMat_inplace)
//
// Row tiles of the block vectors are copied global -> shared with cp.async
// (16-byte copies, no register staging), two buffers deep: the copy of tile
// t+1 is in flight while tile t is computed.  Thread (ty, tx) owns the
// outputs (ty + TY*a, tx + TX*b), a,b < TT: in every shared-memory read a
// warp touches few distinct V values (broadcast) and consecutive W / C
// values (no bank conflicts).  Widths are padded to BM / BK with zero
// columns that the copies never overwrite.
//
// Requirements (checked by the launcher): widths and leading dimensions are
// multiples of the 16-byte vector (2 doubles, 4 floats) and the first
// element of every operand is 16-byte aligned.
#pragma once
#include "pb_block.cuh"

namespace pb {

__device__ __forceinline__ void cp_async16(void* smem, const void* gmem, bool pred)
{
  const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
  const int sz = pred ? 16 : 0;  // 0: zero-fill, nothing read
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(s), "l"(gmem), "r"(sz)
               : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() { asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory"); }

// copy rows [r0, r0+R) x ncols of a row-major block vector into s[R][pitch]
// (rows beyond n are zero-filled); ncols and ld are multiples of VW
template <class T, int R>
__device__ __forceinline__ void issue_rows(T* s, int pitch, const T* __restrict__ g, int64_t ld,
                                           int64_t r0, int64_t n, int ncols)
{
  constexpr int VW = 16 / sizeof(T);
  const int chunks = ncols / VW;
  const int tot = R * chunks;
  for (int q = threadIdx.x; q < tot; q += blockDim.x) {
    const int rr = q / chunks, c = q - rr * chunks;
    const int64_t row = r0 + rr;
    const bool ok = row < n;
    cp_async16(s + rr * pitch + c * VW, g + (ok ? row : 0) * ld + c * VW, ok);
  }
}

// ------------------------------------------------------------ V'W (Gram)
template <class T, int BM, int BK, int TT, int R>
__global__ void __launch_bounds__(256) k_mvtmv_async(MvTmvArgs<T> a)
{
  constexpr int TY = BM / TT, TX = BK / TT, NT = TY * TX, RG = 256 / NT;
  static_assert(RG >= 1, "tile too large");
  extern __shared__ __align__(16) unsigned char smem_raw[];
  T* sV = reinterpret_cast<T*>(smem_raw);  // [2][R][BM]
  T* sW = sV + 2 * R * BM;                  // [2][R][BK]
  const int tid = threadIdx.x;
  const int g = tid / NT, t = tid - g * NT, ty = t / TX, tx = t - ty * TX;

  for (int q = tid; q < 2 * R * (BM + BK); q += blockDim.x) sV[q] = T(0);
  __syncthreads();

  T acc[TT][TT];
#pragma unroll
  for (int p = 0; p < TT; p++)
#pragma unroll
    for (int q = 0; q < TT; q++) acc[p][q] = T(0);

  const int64_t ntiles = (a.n + R - 1) / R;
  int64_t tile = blockIdx.x;
  if (tile < ntiles) {
    issue_rows<T, R>(sV, BM, a.V, a.ldv, tile * R, a.n, a.m);
    issue_rows<T, R>(sW, BK, a.W, a.ldw, tile * R, a.n, a.k);
  }
  cp_async_commit();
  int buf = 0;
  for (; tile < ntiles; tile += gridDim.x) {
    const int64_t next = tile + gridDim.x;
    if (next < ntiles) {
      issue_rows<T, R>(sV + (buf ^ 1) * R * BM, BM, a.V, a.ldv, next * R, a.n, a.m);
      issue_rows<T, R>(sW + (buf ^ 1) * R * BK, BK, a.W, a.ldw, next * R, a.n, a.k);
    }
    cp_async_commit();
    cp_async_wait<1>();
    __syncthreads();
    if (g < RG) {
      const T* v0 = sV + buf * R * BM;
      const T* w0 = sW + buf * R * BK;
#pragma unroll 2
      for (int rr = g; rr < R; rr += RG) {
        T v[TT], w[TT];
#pragma unroll
        for (int p = 0; p < TT; p++) v[p] = v0[rr * BM + ty + TY * p];
#pragma unroll
        for (int q = 0; q < TT; q++) w[q] = w0[rr * BK + tx + TX * q];
#pragma unroll
        for (int p = 0; p < TT; p++)
#pragma unroll
          for (int q = 0; q < TT; q++) acc[p][q] += v[p] * w[q];
      }
    }
    __syncthreads();
    buf ^= 1;
  }
  cp_async_wait<0>();
  __syncthreads();
  // row groups reduced in fixed order in shared memory (reuse the staging)
  T* red = sV;  // [RG][BM*BK]
  if (g < RG) {
#pragma unroll
    for (int p = 0; p < TT; p++)
#pragma unroll
      for (int q = 0; q < TT; q++) red[g * BM * BK + (ty + TY * p) + (tx + TX * q) * BM] = acc[p][q];
  }
  __syncthreads();
  const int nout = a.m * a.k;
  T* part = a.part + (int64_t)blockIdx.x * nout;
  for (int o = tid; o < nout; o += blockDim.x) {
    const int i = o % a.m, j = o / a.m;
    T s = T(0);
    for (int gg = 0; gg < RG; gg++) s += red[gg * BM * BK + i + j * BM];
    part[o] = s;
  }
  last_block_reduce<T>(a.part, nout, gridDim.x, a.counter, a.Cd, 1, a.m, a.ldc, a.alpha, a.beta);
}

// ------------------------------------------------------------ V*C (rows)
// thread (ty, tx): rows ty + TY*p of the tile (p < TR), columns tx + TX*q
// (q < TC); a tile has R = TY*TR rows
template <class T, int BM, int BK, int TR, int TC>
__global__ void __launch_bounds__(256) k_mvsd_async(RowGemmArgs<T> a)
{
  constexpr int TX = BK / TC, TY = 256 / TX, R = TY * TR;
  // row pitch padded by one 16-byte vector: the rows a warp reads at one
  // column fall into different banks
  constexpr int AP = BM + 16 / sizeof(T);
  extern __shared__ __align__(16) unsigned char smem_raw[];
  T* sC = reinterpret_cast<T*>(smem_raw);  // [BM][BK]
  T* sA = sC + BM * BK;                     // [2][R][AP]
  const int tid = threadIdx.x;
  const int ty = tid / TX, tx = tid - ty * TX;
  const bool inplace = (a.mode == RM_MVSDI);
  const T* A = inplace ? (const T*)a.W : a.V;
  const int64_t lda = inplace ? a.ldw : a.ldv;

  for (int q = tid; q < BM * BK + 2 * R * AP; q += blockDim.x) sC[q] = T(0);
  __syncthreads();
  for (int q = tid; q < a.m * a.k; q += blockDim.x) {
    const int i = q % a.m, j = q / a.m;
    sC[i * BK + j] = a.C[i + j * a.ldc];
  }

  T out[TR][TC];
  const int64_t ntiles = (a.n + R - 1) / R;
  int64_t tile = blockIdx.x;
  if (tile < ntiles) issue_rows<T, R>(sA, AP, A, lda, tile * R, a.n, a.m);
  cp_async_commit();
  int buf = 0;
  for (; tile < ntiles; tile += gridDim.x) {
    const int64_t next = tile + gridDim.x;
    if (next < ntiles) issue_rows<T, R>(sA + (buf ^ 1) * R * AP, AP, A, lda, next * R, a.n, a.m);
    cp_async_commit();
    cp_async_wait<1>();
    __syncthreads();
    const T* a0 = sA + buf * R * AP;
#pragma unroll
    for (int p = 0; p < TR; p++)
#pragma unroll
      for (int q = 0; q < TC; q++) out[p][q] = T(0);
#pragma unroll 4
    for (int i = 0; i < BM; i++) {
      T v[TR], c[TC];
#pragma unroll
      for (int p = 0; p < TR; p++) v[p] = a0[(ty + TY * p) * AP + i];
#pragma unroll
      for (int q = 0; q < TC; q++) c[q] = sC[i * BK + tx + TX * q];
#pragma unroll
      for (int p = 0; p < TR; p++)
#pragma unroll
        for (int q = 0; q < TC; q++) out[p][q] += v[p] * c[q];
    }
    const int64_t r0 = tile * R;
#pragma unroll
    for (int p = 0; p < TR; p++) {
      const int64_t row = r0 + ty + TY * p;
      if (row >= a.n) continue;
      T* wr = a.W + row * a.ldw;
#pragma unroll
      for (int q = 0; q < TC; q++) {
        const int j = tx + TX * q;
        if (j < a.k) {
          if (inplace) wr[j] = out[p][q];
          else wr[j] = (a.beta != T(0)) ? a.alpha * out[p][q] + a.beta * wr[j] : a.alpha * out[p][q];
        }
      }
    }
    __syncthreads();
    buf ^= 1;
  }
  cp_async_wait<0>();
}

}  // namespace pb
