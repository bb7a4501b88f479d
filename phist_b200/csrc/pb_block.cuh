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

}  // namespace pb
