// pb_block.cuh -- tall-skinny block products on row-major block vectors.
//
//  k_mvTmv   : C = alpha*V'W + beta*C  (mvecT_times_mvec, phist_kernels_decl.h:557)
//              split-n over a fixed grid, per-block partial Gram matrices,
//              deterministic second-level sum (pb_reduce.cuh).
//  k_rowgemm : per-row products, all in one pass over the rows:
//              mode MVSD  : W = alpha*V*C + beta*W            (:565)
//              mode MVSDI : W(:,0:k) = W(:,0:m)*C  in place   (:577)
//              mode VCWD  : W = V*C + W*D                     (:585)
//              optional fused Gram of the NEW W tile:
//              gram G_WW : G = W'W       (fused_mvsd_mvTmv,  fused_decl.h:92)
//              gram G_VW : G = alpha*V'W + beta*G (fused_mvsdi_mvTmv, :84)
//
// Both kernels stage a tile of R rows of every operand in shared memory
// (coalesced 16-byte loads of contiguous row segments), then each thread
// computes a register micro-tile; the small matrices C/D stay in shared
// memory for the whole launch.  Loop orders per output follow the builtin
// kernels (gemm_kernels_sC.F90:17-80, gemm_kernels_sB.F90:15-613).
#pragma once
#include "pb_core.hpp"
#include "pb_reduce.cuh"

namespace pb {

constexpr int BLK_BS = 256;

// ---------------------------------------------------------------- staging
// copy rows [r0, r0+R) x cols [0, ncols) of a row-major block vector into
// shared memory tile s[R][pitch] (zero-filled outside the matrix).
template <class T>
__device__ __forceinline__ void stage_rows(T* s, int pitch, const T* __restrict__ g, int64_t ldg,
                                           int64_t r0, int64_t n, int R, int ncols)
{
  const int tot = R * pitch;
  // rows stored back to back with the tile's own pitch and 16-byte aligned:
  // one flat vectorised copy (the common case of a full, unpadded mvec)
  constexpr int VW = 16 / sizeof(T);
  if (ldg == pitch && pitch == ncols && ((uintptr_t)(g + r0 * ldg) & 15u) == 0 &&
      ((uintptr_t)s & 15u) == 0 && (tot % VW) == 0) {
    const int64_t avail = (n - r0) * (int64_t)pitch;  // elements inside the matrix
    const T* src = g + r0 * ldg;
    const int nv = tot / VW;
    for (int t = threadIdx.x; t < nv; t += blockDim.x) {
      const int64_t e = (int64_t)t * VW;
      if (e + VW <= avail) {
        if (sizeof(T) == 8) {
          reinterpret_cast<double2*>(s)[t] = __ldcs(reinterpret_cast<const double2*>(src) + t);
        } else {
          reinterpret_cast<float4*>(s)[t] = __ldcs(reinterpret_cast<const float4*>(src) + t);
        }
      } else {
        for (int w = 0; w < VW; w++) s[e + w] = (e + w < avail) ? src[e + w] : T(0);
      }
    }
    return;
  }
  for (int t = threadIdx.x; t < tot; t += blockDim.x) {
    const int rr = t / pitch, c = t - rr * pitch;
    const int64_t row = r0 + rr;
    s[t] = (row < n && c < ncols) ? g[row * ldg + c] : T(0);
  }
}

// --------------------------------------------------------------- mvTmv
template <class T>
struct MvTmvArgs {
  int64_t n;
  int m, k;
  const T* V; int64_t ldv;
  const T* W; int64_t ldw;
  T alpha, beta;
  T* Cd; int64_t ldc;          // device result (col-major)
  T* part; unsigned int* counter;
  int R;                        // rows per tile
  int ext_reduce;               // k_mvtmv_async: leave the partials to k_reduce_partials
};

// thread (tm, tk, g): output micro-tile rows [tm*TM, +TM) of V' and columns
// [tk*TK, +TK) of W, rows of the tile with index = g (mod RG)
template <class T, int TM, int TK>
__global__ void __launch_bounds__(BLK_BS) k_mvTmv(MvTmvArgs<T> a)
{
  extern __shared__ __align__(16) unsigned char smem_raw[];
  T* sV = reinterpret_cast<T*>(smem_raw);
  const int mp = ((a.m + TM - 1) / TM) * TM, kp = ((a.k + TK - 1) / TK) * TK;
  T* sW = sV + a.R * mp;
  const int ntm = mp / TM, ntk = kp / TK, nt = ntm * ntk;
  const int RG = BLK_BS / nt;  // >= 1 by construction of the launch
  const int tid = threadIdx.x;
  const int g = tid / nt, tt = tid - g * nt;
  const int tm = tt % ntm, tk = tt / ntm;
  const bool active = g < RG;

  T acc[TM][TK];
#pragma unroll
  for (int p = 0; p < TM; p++)
#pragma unroll
    for (int q = 0; q < TK; q++) acc[p][q] = T(0);

  const int64_t ntiles = (a.n + a.R - 1) / a.R;
  for (int64_t t = blockIdx.x; t < ntiles; t += gridDim.x) {
    const int64_t r0 = t * a.R;
    __syncthreads();
    stage_rows(sV, mp, a.V, a.ldv, r0, a.n, a.R, a.m);
    stage_rows(sW, kp, a.W, a.ldw, r0, a.n, a.R, a.k);
    __syncthreads();
    if (active) {
      for (int rr = g; rr < a.R; rr += RG) {
        T v[TM], w[TK];
#pragma unroll
        for (int p = 0; p < TM; p++) v[p] = sV[rr * mp + tm * TM + p];
#pragma unroll
        for (int q = 0; q < TK; q++) w[q] = sW[rr * kp + tk * TK + q];
#pragma unroll
        for (int p = 0; p < TM; p++)
#pragma unroll
          for (int q = 0; q < TK; q++) acc[p][q] += v[p] * w[q];
      }
    }
  }
  // block reduction over the RG row groups in fixed order (reuse sV)
  __syncthreads();
  T* red = reinterpret_cast<T*>(smem_raw);  // [RG][mp*kp]
  const int mk = mp * kp;
  if (active) {
#pragma unroll
    for (int p = 0; p < TM; p++)
#pragma unroll
      for (int q = 0; q < TK; q++) red[g * mk + (tm * TM + p) + (tk * TK + q) * mp] = acc[p][q];
  }
  __syncthreads();
  const int nout = a.m * a.k;
  T* part = a.part + (int64_t)blockIdx.x * nout;
  for (int o = tid; o < nout; o += blockDim.x) {
    const int i = o % a.m, j = o / a.m;
    T s = T(0);
    for (int gg = 0; gg < RG; gg++) s += red[gg * mk + i + j * mp];
    part[o] = s;
  }
  last_block_reduce<T>(a.part, nout, gridDim.x, a.counter, a.Cd, 1, a.m, a.ldc, a.alpha, a.beta);
}

// -------------------------------------------------------------- rowgemm
enum RowMode { RM_MVSD = 0, RM_MVSDI = 1, RM_VCWD = 2 };
enum GramMode { GM_NONE = 0, GM_WW = 1, GM_VW = 2 };

template <class T>
struct RowGemmArgs {
  int64_t n;
  int m, k, mv;          // V (or in-place W) has m columns; W has k; V for G_VW has mv
  const T* V; int64_t ldv;
  T* W; int64_t ldw;
  const T* C; int64_t ldc;  // m x k (device, col-major)
  const T* D; int64_t ldd;  // k x k (device, col-major), VCWD only
  T alpha, beta;
  int mode, gram;
  const T* Vg; int64_t ldvg; // left operand of G_VW
  T galpha, gbeta;
  T* Gd; int64_t ldg;
  T* part; unsigned int* counter;
  int R;
};

// shared memory: sA[R][ap] (row operand: V, or W for MVSDI), sW[R][kp]
// (old W for beta/VCWD, then the new W tile), sC[ap][kp], sD[kp][kp],
// sVg[R][mvp] (G_VW only)
template <class T, int TR, int TK>
__global__ void __launch_bounds__(BLK_BS) k_rowgemm(RowGemmArgs<T> a)
{
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int acols = (a.mode == RM_MVSDI) ? a.m : a.m;
  const int ap = acols + (acols & 1);
  const int kp = ((a.k + TK - 1) / TK) * TK;
  const int mvp = a.mv + (a.mv & 1);
  T* sA = reinterpret_cast<T*>(smem_raw);
  T* sW = sA + a.R * ap;
  T* sC = sW + a.R * kp;
  T* sD = sC + ap * kp;
  T* sVg = sD + ((a.mode == RM_VCWD) ? kp * kp : 0);
  const int tid = threadIdx.x;

  // small matrices once per block
  for (int t = tid; t < ap * kp; t += blockDim.x) {
    const int i = t / kp, j = t - i * kp;
    sC[t] = (i < a.m && j < a.k) ? a.C[i + j * a.ldc] : T(0);
  }
  if (a.mode == RM_VCWD)
    for (int t = tid; t < kp * kp; t += blockDim.x) {
      const int i = t / kp, j = t - i * kp;
      sD[t] = (i < a.k && j < a.k) ? a.D[i + j * a.ldd] : T(0);
    }

  const int ntk = kp / TK;
  const int ntr = BLK_BS / ntk;         // thread rows; each covers TR tile rows
  const int tk = tid % ntk, trow = tid / ntk;
  const bool active = trow * TR < a.R;

  // fused Gram accumulators: thread owns output entries o = tid + q*BLK_BS
  const int gm = (a.gram == GM_WW) ? a.k : a.mv;
  const int gout = (a.gram == GM_NONE) ? 0 : gm * a.k;
  constexpr int GMAX = 16;  // up to 16*256 = 4096 = 64x64 Gram entries
  T gacc[GMAX];
#pragma unroll
  for (int q = 0; q < GMAX; q++) gacc[q] = T(0);

  const int64_t ntiles = (a.n + a.R - 1) / a.R;
  for (int64_t t = blockIdx.x; t < ntiles; t += gridDim.x) {
    const int64_t r0 = t * a.R;
    __syncthreads();
    if (a.mode == RM_MVSDI) {
      stage_rows(sA, ap, (const T*)a.W, a.ldw, r0, a.n, a.R, a.m);
    } else {
      stage_rows(sA, ap, a.V, a.ldv, r0, a.n, a.R, a.m);
      if (a.mode == RM_VCWD || a.beta != T(0)) stage_rows(sW, kp, (const T*)a.W, a.ldw, r0, a.n, a.R, a.k);
    }
    if (a.gram == GM_VW) stage_rows(sVg, mvp, a.Vg, a.ldvg, r0, a.n, a.R, a.mv);
    __syncthreads();

    T out[TR][TK];
    if (active) {
#pragma unroll
      for (int p = 0; p < TR; p++)
#pragma unroll
        for (int q = 0; q < TK; q++) out[p][q] = T(0);
      for (int j = 0; j < a.m; j++) {
        T b[TK];
#pragma unroll
        for (int q = 0; q < TK; q++) b[q] = sC[j * kp + tk * TK + q];
#pragma unroll
        for (int p = 0; p < TR; p++) {
          const T av = sA[(trow * TR + p) * ap + j];
#pragma unroll
          for (int q = 0; q < TK; q++) out[p][q] += av * b[q];
        }
      }
      if (a.mode == RM_VCWD) {
        for (int j = 0; j < a.k; j++) {
          T d[TK];
#pragma unroll
          for (int q = 0; q < TK; q++) d[q] = sD[j * kp + tk * TK + q];
#pragma unroll
          for (int p = 0; p < TR; p++) {
            const T wv = sW[(trow * TR + p) * kp + j];
#pragma unroll
            for (int q = 0; q < TK; q++) out[p][q] += wv * d[q];
          }
        }
      } else if (a.mode == RM_MVSD) {
#pragma unroll
        for (int p = 0; p < TR; p++)
#pragma unroll
          for (int q = 0; q < TK; q++) {
            const T o = a.alpha * out[p][q];
            out[p][q] = (a.beta != T(0)) ? o + a.beta * sW[(trow * TR + p) * kp + tk * TK + q] : o;
          }
      }
    }
    __syncthreads();  // everyone done reading sW before it is overwritten
    if (active) {
#pragma unroll
      for (int p = 0; p < TR; p++) {
        const int rr = trow * TR + p;
        const int64_t row = r0 + rr;
#pragma unroll
        for (int q = 0; q < TK; q++) {
          const int c = tk * TK + q;
          const T v = (row < a.n && c < a.k) ? out[p][q] : T(0);
          sW[rr * kp + c] = v;
          if (row < a.n && c < a.k) a.W[row * a.ldw + c] = v;
        }
      }
    }
    if (a.gram != GM_NONE) {
      __syncthreads();
      // Gram of the tile: entry o=(i,j) col-major in gm x k
#pragma unroll
      for (int q = 0; q < GMAX; q++) {
        const int o = tid + q * BLK_BS;
        if (o < gout) {
          const int i = o % gm, j = o / gm;
          T s = T(0);
          if (a.gram == GM_WW) {
            for (int rr = 0; rr < a.R; rr++) s += sW[rr * kp + i] * sW[rr * kp + j];
          } else {
            for (int rr = 0; rr < a.R; rr++) s += sVg[rr * mvp + i] * sW[rr * kp + j];
          }
          gacc[q] += s;
        }
      }
    }
  }
  if (a.gram == GM_NONE) return;
  T* part = a.part + (int64_t)blockIdx.x * gout;
#pragma unroll
  for (int q = 0; q < GMAX; q++) {
    const int o = tid + q * BLK_BS;
    if (o < gout) part[o] = gacc[q];
  }
  const T al = (a.gram == GM_WW) ? T(1) : a.galpha;
  const T be = (a.gram == GM_WW) ? T(0) : a.gbeta;
  last_block_reduce<T>(a.part, gout, gridDim.x, a.counter, a.Gd, 1, gm, a.ldg, al, be);
}

// ---------------------------------------------------- small widths (<= 8)
// One thread per row, everything in registers: the row of V (M values) and
// of W (K values) are loaded once, the M x K Gram contribution or the K new
// values of W are formed in registers.  Used when m, k (and mv) are <= 8,
// where the tiled kernels above would spend their time staging.

template <class T>
__device__ __forceinline__ void load_row(const T* __restrict__ p, int ncols, int NMAX, T* out)
{
  // NMAX compile-time at the call sites; columns >= ncols read as zero
#pragma unroll
  for (int c = 0; c < 8; c++)
    if (c < NMAX) out[c] = (c < ncols) ? __ldg(p + c) : T(0);
}

// sum the NOUT per-thread values of every thread of the block in a fixed
// order (warp butterfly, then warps in order) and write the block partial
template <class T, int NOUT>
__device__ __forceinline__ void block_partial(T* vals, T* part, int nout)
{
  __shared__ T red[8][NOUT];
#pragma unroll
  for (int off = 16; off >= 1; off >>= 1)
#pragma unroll
    for (int q = 0; q < NOUT; q++) vals[q] += __shfl_xor_sync(0xffffffffu, vals[q], off);
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  if (lane == 0)
#pragma unroll
    for (int q = 0; q < NOUT; q++) red[warp][q] = vals[q];
  __syncthreads();
  for (int q = threadIdx.x; q < nout; q += blockDim.x) {
    T s = T(0);
    for (int w = 0; w < (int)(blockDim.x >> 5); w++) s += red[w][q];
    part[(int64_t)blockIdx.x * nout + q] = s;
  }
}

// C(m x k) = alpha V'W + beta C, m <= M, k <= K
template <class T, int M, int K>
__global__ void __launch_bounds__(256) k_mvTmv_reg(MvTmvArgs<T> a)
{
  T acc[M * K];
#pragma unroll
  for (int q = 0; q < M * K; q++) acc[q] = T(0);
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < a.n;
       i += (int64_t)gridDim.x * blockDim.x) {
    T v[8], w[8];
    load_row(a.V + i * a.ldv, a.m, M, v);
    load_row(a.W + i * a.ldw, a.k, K, w);
#pragma unroll
    for (int q = 0; q < K; q++)
#pragma unroll
      for (int p = 0; p < M; p++) acc[p + q * M] += v[p] * w[q];
  }
  // compact to the m x k layout expected by the final reduction
  T vals[M * K];
#pragma unroll
  for (int q = 0; q < K; q++)
#pragma unroll
    for (int p = 0; p < M; p++) vals[p + q * M] = acc[p + q * M];
  block_partial<T, M * K>(vals, a.part, M * K);
  // outputs are laid out with row stride M in the partials: map to (m, k)
  last_block_reduce<T>(a.part, M * K, gridDim.x, a.counter, a.Cd, 1, M, a.ldc, a.alpha, a.beta, a.m, a.k);
}

// Thin blocks of exactly M and K columns (multiples of 4) whose rows start
// on 32-byte boundaries: one thread per row, each row of V and W read with
// 256-bit loads (ld.global.nc.v4.f64, 4 doubles), UNR rows of a thread in
// flight before their FMAs; the same fixed-order reductions as k_mvTmv_reg.
__device__ __forceinline__ void ld4_nc(const double* p, double* o)
{
  asm volatile("ld.global.nc.v4.f64 {%0, %1, %2, %3}, [%4];\n"
               : "=d"(o[0]), "=d"(o[1]), "=d"(o[2]), "=d"(o[3])
               : "l"(p));
}

template <int M, int K, int UNR>
__global__ void __launch_bounds__(256) k_mvTmv_v4(MvTmvArgs<double> a)
{
  double acc[M * K];
#pragma unroll
  for (int q = 0; q < M * K; q++) acc[q] = 0.0;
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  for (; i + (UNR - 1) * stride < a.n; i += UNR * stride) {
    double v[UNR][M], w[UNR][K];
#pragma unroll
    for (int u = 0; u < UNR; u++) {
#pragma unroll
      for (int c = 0; c < M; c += 4) ld4_nc(a.V + (i + u * stride) * a.ldv + c, &v[u][c]);
#pragma unroll
      for (int c = 0; c < K; c += 4) ld4_nc(a.W + (i + u * stride) * a.ldw + c, &w[u][c]);
    }
#pragma unroll
    for (int u = 0; u < UNR; u++)
#pragma unroll
      for (int q = 0; q < K; q++)
#pragma unroll
        for (int p = 0; p < M; p++) acc[p + q * M] += v[u][p] * w[u][q];
  }
  for (; i < a.n; i += stride) {
    double v[M], w[K];
#pragma unroll
    for (int c = 0; c < M; c += 4) ld4_nc(a.V + i * a.ldv + c, &v[c]);
#pragma unroll
    for (int c = 0; c < K; c += 4) ld4_nc(a.W + i * a.ldw + c, &w[c]);
#pragma unroll
    for (int q = 0; q < K; q++)
#pragma unroll
      for (int p = 0; p < M; p++) acc[p + q * M] += v[p] * w[q];
  }
  block_partial<double, M * K>(acc, a.part, M * K);
  last_block_reduce<double>(a.part, M * K, gridDim.x, a.counter, a.Cd, 1, M, a.ldc, a.alpha, a.beta, a.m, a.k);
}

// row-local products for m, k, mv <= 8 (modes and Gram as k_rowgemm)
template <class T, int M, int K, int MV>
__global__ void __launch_bounds__(256) k_rowgemm_reg(RowGemmArgs<T> a)
{
  __shared__ T sC[M * K];
  __shared__ T sD[K * K];
  for (int t = threadIdx.x; t < M * K; t += blockDim.x) {
    const int i = t % M, j = t / M;
    sC[t] = (i < a.m && j < a.k) ? a.C[i + j * a.ldc] : T(0);
  }
  if (a.mode == RM_VCWD)
    for (int t = threadIdx.x; t < K * K; t += blockDim.x) {
      const int i = t % K, j = t / K;
      sD[t] = (i < a.k && j < a.k) ? a.D[i + j * a.ldd] : T(0);
    }
  __syncthreads();
  constexpr int GM = (MV > K) ? MV : K;
  T gacc[GM * K];
#pragma unroll
  for (int q = 0; q < GM * K; q++) gacc[q] = T(0);
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < a.n;
       i += (int64_t)gridDim.x * blockDim.x) {
    T v[8], w[8], out[8];
    if (a.mode == RM_MVSDI) load_row((const T*)a.W + i * a.ldw, a.m, M, v);
    else load_row(a.V + i * a.ldv, a.m, M, v);
    if (a.mode == RM_VCWD || (a.mode == RM_MVSD && a.beta != T(0)))
      load_row((const T*)a.W + i * a.ldw, a.k, K, w);
#pragma unroll
    for (int q = 0; q < K; q++) {
      T s = T(0);
#pragma unroll
      for (int p = 0; p < M; p++) s += v[p] * sC[p + q * M];
      if (a.mode == RM_VCWD) {
#pragma unroll
        for (int p = 0; p < K; p++) s += w[p] * sD[p + q * K];
      } else if (a.mode == RM_MVSD) {
        s = (a.beta != T(0)) ? a.alpha * s + a.beta * w[q] : a.alpha * s;
      }
      out[q] = s;
    }
#pragma unroll
    for (int q = 0; q < K; q++)
      if (q < a.k) a.W[i * a.ldw + q] = out[q];
    if (a.gram == GM_WW) {
#pragma unroll
      for (int q = 0; q < K; q++)
#pragma unroll
        for (int p = 0; p < K; p++) gacc[p + q * K] += out[p] * out[q];
    } else if (a.gram == GM_VW) {
      T g[8];
      load_row(a.Vg + i * a.ldvg, a.mv, MV, g);
#pragma unroll
      for (int q = 0; q < K; q++)
#pragma unroll
        for (int p = 0; p < MV; p++) gacc[p + q * MV] += g[p] * out[q];
    }
  }
  if (a.gram == GM_NONE) return;
  const int gmax = (a.gram == GM_WW) ? K : MV;
  // partial layout: gmax rows (padded), K columns
  block_partial<T, GM * K>(gacc, a.part, gmax * K);
  const T al = (a.gram == GM_WW) ? T(1) : a.galpha;
  const T be = (a.gram == GM_WW) ? T(0) : a.gbeta;
  last_block_reduce<T>(a.part, gmax * K, gridDim.x, a.counter, a.Gd, 1, gmax, a.ldg, al, be,
                       (a.gram == GM_WW) ? a.k : a.mv, a.k);
}

}  // namespace pb
