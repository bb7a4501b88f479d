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
#include "pb_tma.cuh"

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
// S-stage pipeline: S-1 row tiles of R rows are in flight while one is
// computed, so that each SM keeps enough bytes outstanding to cover the HBM
// latency (about 64 KiB per SM at 6.5 TB/s).  Shared rows are padded by one
// 16-byte vector (pitches PV, PW): the rows a warp touches at one column fall
// into different banks.
template <class T, int BM, int BK, int TT, int R, int S>
__global__ void __launch_bounds__(256) k_mvtmv_async(MvTmvArgs<T> a)
{
  constexpr int TY = BM / TT, TX = BK / TT, NT = TY * TX, RG = 256 / NT;
  constexpr int PV = BM + 16 / sizeof(T), PW = BK + 16 / sizeof(T);
  static_assert(RG >= 1 && S >= 2, "tile too large or too few stages");
  extern __shared__ __align__(16) unsigned char smem_raw[];
  T* sV = reinterpret_cast<T*>(smem_raw);  // [S][R][PV]
  T* sW = sV + S * R * PV;                  // [S][R][PW]
  const int tid = threadIdx.x;
  const int g = tid / NT, t = tid - g * NT, ty = t / TX, tx = t - ty * TX;

  // pad columns (>= m, >= k, and the pitch padding) are never written by copies
  for (int q = tid; q < S * R * (PV + PW); q += blockDim.x) sV[q] = T(0);
  __syncthreads();

  T acc[TT][TT];
#pragma unroll
  for (int p = 0; p < TT; p++)
#pragma unroll
    for (int q = 0; q < TT; q++) acc[p][q] = T(0);

  const int64_t ntiles = (a.n + R - 1) / R;
  // prologue: the first S-1 tiles of this block, one commit group each
#pragma unroll
  for (int st = 0; st < S - 1; st++) {
    const int64_t tl = blockIdx.x + (int64_t)st * gridDim.x;
    if (tl < ntiles) {
      issue_rows<T, R>(sV + st * R * PV, PV, a.V, a.ldv, tl * R, a.n, a.m);
      issue_rows<T, R>(sW + st * R * PW, PW, a.W, a.ldw, tl * R, a.n, a.k);
    }
    cp_async_commit();
  }
  int stage = 0;
  for (int64_t tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
    // refill the stage computed in the previous iteration with tile + (S-1)
    const int64_t nt = tile + (int64_t)(S - 1) * gridDim.x;
    const int ps = (stage + S - 1) % S;
    if (nt < ntiles) {
      issue_rows<T, R>(sV + ps * R * PV, PV, a.V, a.ldv, nt * R, a.n, a.m);
      issue_rows<T, R>(sW + ps * R * PW, PW, a.W, a.ldw, nt * R, a.n, a.k);
    }
    cp_async_commit();
    cp_async_wait<S - 1>();  // this tile's group has landed
    __syncthreads();
    if (g < RG) {
      const T* v0 = sV + stage * R * PV;
      const T* w0 = sW + stage * R * PW;
#pragma unroll 2
      for (int rr = g; rr < R; rr += RG) {
        T v[TT], w[TT];
#pragma unroll
        for (int p = 0; p < TT; p++) v[p] = v0[rr * PV + ty + TY * p];
#pragma unroll
        for (int q = 0; q < TT; q++) w[q] = w0[rr * PW + tx + TX * q];
#pragma unroll
        for (int p = 0; p < TT; p++)
#pragma unroll
          for (int q = 0; q < TT; q++) acc[p][q] += v[p] * w[q];
      }
    }
    __syncthreads();
    stage = (stage + 1) % S;
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
  if (a.ext_reduce) return;  // second pass: k_reduce_partials
  last_block_reduce<T>(a.part, nout, gridDim.x, a.counter, a.Cd, 1, a.m, a.ldc, a.alpha, a.beta);
}

// ------------------------------------------------------------ V'W, TMA-staged
// Same thread mapping and fixed-order reduction as k_mvtmv_async, but every
// row tile of V and W arrives as one 2D TMA box (R rows x PV or PW columns,
// the columns past m / k zero-filled by the hardware) on an mbarrier.  Thread
// 0 issues the copies S-1 tiles ahead; all threads wait on the stage's
// barrier (bounded, see mbar_wait) and the block synchronises once per tile
// before the stage is refilled.
template <class T, int BM, int BK, int TT, int R, int S>
__global__ void __launch_bounds__(256) k_mvtmv_tma(MvTmvArgs<T> a, const __grid_constant__ CUtensorMap mapV,
                                                   const __grid_constant__ CUtensorMap mapW, int* err)
{
  constexpr int TY = BM / TT, TX = BK / TT, NT = TY * TX, RG = 256 / NT;
  constexpr int PV = BM + 16 / sizeof(T), PW = BK + 16 / sizeof(T);
  constexpr unsigned STAGE_BYTES = (unsigned)(R * (PV + PW) * sizeof(T));
  static_assert(RG >= 1 && S >= 2 && R <= 256 && PV <= 256 && PW <= 256, "bad tile shape");
  extern __shared__ __align__(128) unsigned char smem_raw[];
  T* sV = reinterpret_cast<T*>(smem_raw);  // [S][R][PV]
  T* sW = sV + S * R * PV;                  // [S][R][PW]
  uint64_t* bar = reinterpret_cast<uint64_t*>(sW + S * R * PW);
  const int tid = threadIdx.x;
  const int g = tid / NT, t = tid - g * NT, ty = t / TX, tx = t - ty * TX;
  const int64_t ntiles = (a.n + R - 1) / R;

  if (tid == 0) {
    for (int st = 0; st < S; st++) mbar_init(&bar[st], 1);
    mbar_fence_init();
    tma_prefetch_desc(&mapV);
    tma_prefetch_desc(&mapW);
  }
  __syncthreads();
  if (tid == 0) {
    for (int st = 0; st < S - 1; st++) {
      const int64_t tl = blockIdx.x + (int64_t)st * gridDim.x;
      if (tl < ntiles) {
        mbar_arrive_expect_tx(&bar[st], STAGE_BYTES);
        tma_load_2d(sV + st * R * PV, &mapV, 0, (int)(tl * R), &bar[st]);
        tma_load_2d(sW + st * R * PW, &mapW, 0, (int)(tl * R), &bar[st]);
      }
    }
  }

  T acc[TT][TT];
#pragma unroll
  for (int p = 0; p < TT; p++)
#pragma unroll
    for (int q = 0; q < TT; q++) acc[p][q] = T(0);

  bool ok = true;
  int stage = 0;
  int64_t it = 0;
  for (int64_t tile = blockIdx.x; tile < ntiles; tile += gridDim.x, it++) {
    if (tid == 0) {
      // refill the stage consumed in the previous iteration
      const int64_t nt = tile + (int64_t)(S - 1) * gridDim.x;
      const int ps = (stage + S - 1) % S;
      if (nt < ntiles) {
        mbar_arrive_expect_tx(&bar[ps], STAGE_BYTES);
        tma_load_2d(sV + ps * R * PV, &mapV, 0, (int)(nt * R), &bar[ps]);
        tma_load_2d(sW + ps * R * PW, &mapW, 0, (int)(nt * R), &bar[ps]);
      }
    }
    // every issued tile is waited for, also after a timeout, so that no copy
    // is left in flight when the block exits
    const bool landed = mbar_wait(&bar[stage], (unsigned)((it / S) & 1), err);
    ok = ok && landed;
    if (ok && g < RG) {
      const T* v0 = sV + stage * R * PV;
      const T* w0 = sW + stage * R * PW;
#pragma unroll 2
      for (int rr = g; rr < R; rr += RG) {
        T v[TT], w[TT];
#pragma unroll
        for (int p = 0; p < TT; p++) v[p] = v0[rr * PV + ty + TY * p];
#pragma unroll
        for (int q = 0; q < TT; q++) w[q] = w0[rr * PW + tx + TX * q];
#pragma unroll
        for (int p = 0; p < TT; p++)
#pragma unroll
          for (int q = 0; q < TT; q++) acc[p][q] += v[p] * w[q];
      }
    }
    __syncthreads();
    stage = (stage + 1) % S;
  }
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
  if (a.ext_reduce) return;  // second pass: k_reduce_partials
  last_block_reduce<T>(a.part, nout, gridDim.x, a.counter, a.Cd, 1, a.m, a.ldc, a.alpha, a.beta);
}

// ------------------------------------------------------------ V*C (rows)
// thread (ty, tx): rows ty + TY*p of the tile (p < TR), columns tx + TX*q
// (q < TC); a tile has R = TY*TR rows.  S-stage pipeline as in
// k_mvtmv_async: S-1 row tiles of the input are in flight while one is
// computed and written.  In place (W(:,0:k) = W(:,0:m) C) is safe: a tile's
// rows are read completely before they are written, and the tiles in flight
// are other rows.
template <class T, int BM, int BK, int TR, int TC, int S>
__global__ void __launch_bounds__(256) k_mvsd_async(RowGemmArgs<T> a)
{
  constexpr int TX = BK / TC, TY = 256 / TX, R = TY * TR;
  // row pitch padded by one 16-byte vector: the rows a warp reads at one
  // column fall into different banks
  constexpr int AP = BM + 16 / sizeof(T);
  static_assert(S >= 2 && TX * TY == 256, "bad tile shape");
  extern __shared__ __align__(16) unsigned char smem_raw[];
  T* sC = reinterpret_cast<T*>(smem_raw);  // [BM][BK]
  T* sA = sC + BM * BK;                     // [S][R][AP]
  const int tid = threadIdx.x;
  const int ty = tid / TX, tx = tid - ty * TX;
  const bool inplace = (a.mode == RM_MVSDI);
  const T* A = inplace ? (const T*)a.W : a.V;
  const int64_t lda = inplace ? a.ldw : a.ldv;

  for (int q = tid; q < BM * BK + S * R * AP; q += blockDim.x) sC[q] = T(0);
  __syncthreads();
  for (int q = tid; q < a.m * a.k; q += blockDim.x) {
    const int i = q % a.m, j = q / a.m;
    sC[i * BK + j] = a.C[i + j * a.ldc];
  }

  const int64_t ntiles = (a.n + R - 1) / R;
#pragma unroll
  for (int st = 0; st < S - 1; st++) {
    const int64_t tl = blockIdx.x + (int64_t)st * gridDim.x;
    if (tl < ntiles) issue_rows<T, R>(sA + st * R * AP, AP, A, lda, tl * R, a.n, a.m);
    cp_async_commit();
  }
  T out[TR][TC];
  int stage = 0;
  for (int64_t tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
    const int64_t nt = tile + (int64_t)(S - 1) * gridDim.x;
    const int ps = (stage + S - 1) % S;
    if (nt < ntiles) issue_rows<T, R>(sA + ps * R * AP, AP, A, lda, nt * R, a.n, a.m);
    cp_async_commit();
    cp_async_wait<S - 1>();
    __syncthreads();
    const T* a0 = sA + stage * R * AP;
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
    stage = (stage + 1) % S;
  }
  cp_async_wait<0>();
}

// ------------------------------------------------------------ V*C, TMA-staged
// k_mvsd_async with the input row tiles delivered as 2D TMA boxes (R rows x
// AP columns, zero-filled past m) on per-stage mbarriers; thread mapping,
// output writes and the in-place rule are those of k_mvsd_async.
template <class T, int BM, int BK, int TR, int TC, int S>
__global__ void __launch_bounds__(256) k_mvsd_tma(RowGemmArgs<T> a, const __grid_constant__ CUtensorMap mapA,
                                                  int* err)
{
  constexpr int TX = BK / TC, TY = 256 / TX, R = TY * TR;
  constexpr int AP = BM + 16 / sizeof(T);
  constexpr unsigned STAGE_BYTES = (unsigned)(R * AP * sizeof(T));
  // sC padded to 128 bytes: TMA destinations start on 128-byte boundaries
  constexpr int CSZ = (BM * BK * (int)sizeof(T) + 127) / 128 * 128 / (int)sizeof(T);
  static_assert(S >= 2 && TX * TY == 256 && R <= 256, "bad tile shape");
  extern __shared__ __align__(128) unsigned char smem_raw[];
  T* sC = reinterpret_cast<T*>(smem_raw);  // [BM][BK]
  T* sA = sC + CSZ;                         // [S][R][AP]
  uint64_t* bar = reinterpret_cast<uint64_t*>(sA + S * R * AP);
  const int tid = threadIdx.x;
  const int ty = tid / TX, tx = tid - ty * TX;
  const bool inplace = (a.mode == RM_MVSDI);
  const int64_t ntiles = (a.n + R - 1) / R;

  if (tid == 0) {
    for (int st = 0; st < S; st++) mbar_init(&bar[st], 1);
    mbar_fence_init();
    tma_prefetch_desc(&mapA);
  }
  for (int q = tid; q < BM * BK; q += blockDim.x) sC[q] = T(0);
  __syncthreads();
  for (int q = tid; q < a.m * a.k; q += blockDim.x) {
    const int i = q % a.m, j = q / a.m;
    sC[i * BK + j] = a.C[i + j * a.ldc];
  }
  if (tid == 0) {
    for (int st = 0; st < S - 1; st++) {
      const int64_t tl = blockIdx.x + (int64_t)st * gridDim.x;
      if (tl < ntiles) {
        mbar_arrive_expect_tx(&bar[st], STAGE_BYTES);
        tma_load_2d(sA + st * R * AP, &mapA, 0, (int)(tl * R), &bar[st]);
      }
    }
  }
  __syncthreads();  // sC complete

  T out[TR][TC];
  bool ok = true;
  int stage = 0;
  int64_t it = 0;
  for (int64_t tile = blockIdx.x; tile < ntiles; tile += gridDim.x, it++) {
    if (tid == 0) {
      const int64_t nt = tile + (int64_t)(S - 1) * gridDim.x;
      const int ps = (stage + S - 1) % S;
      if (nt < ntiles) {
        mbar_arrive_expect_tx(&bar[ps], STAGE_BYTES);
        tma_load_2d(sA + ps * R * AP, &mapA, 0, (int)(nt * R), &bar[ps]);
      }
    }
    const bool landed = mbar_wait(&bar[stage], (unsigned)((it / S) & 1), err);
    ok = ok && landed;
    if (ok) {
      const T* a0 = sA + stage * R * AP;
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
    }
    __syncthreads();
    stage = (stage + 1) % S;
  }
}

}  // namespace pb
