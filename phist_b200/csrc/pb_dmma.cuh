// pb_dmma.cuh -- FP64 block products on the tensor cores (DMMA,
// mma.sync.m8n8k4.f64) with TMA-staged row tiles, for padded widths of 8 to
// 64 (multiples of 8).
//
//   k_mvtmv_dmma : C = alpha V'W + beta C      (Gram / projection matrices)
//   k_mvsd_dmma  : W = alpha V C + beta W, or W(:,0:k) = W(:,0:m) C in place
//
// Fragment layout of mma.m8n8k4.row.col.f64 (lane l, g = l/4, t = l%4):
//   A (8x4, row-major): a = A[g][t];  B (4x8, column-major): b = B[t][g];
//   C/D (8x8): d0 = D[g][2t], d1 = D[g][2t+1].
// One DMMA does 256 FMAs from one shared-memory value per lane and operand,
// so the narrow-width products that the scalar micro-tiles leave bound by
// shared-memory issue run at the HBM or FP64 rate instead.
//
// Shared rows are padded by 4 doubles (PV = BM + 4 etc.): the 4 (or 8) rows
// of one fragment then start 8 banks apart and each bank is hit exactly
// twice, the minimum for 256 bytes.  The TMA boxes are PV columns wide, the
// columns past m read as zero.
#pragma once
#include "pb_block.cuh"
#include "pb_tma.cuh"

namespace pb {

__device__ __forceinline__ void dmma_884(double& d0, double& d1, double a, double b)
{
  asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0, %1}, {%2}, {%3}, {%0, %1};\n"
               : "+d"(d0), "+d"(d1)
               : "d"(a), "d"(b));
}

// ------------------------------------------------------------------ V'W
// The k-dimension of the MMAs is the row index: warp w takes the 4-row steps
// ks = wq, wq + 8/WS, ... of every stage and accumulates its share of the
// BM x BK output (m-tiles [mh*MTW, (mh+1)*MTW) with mh = w % WS); WS = 2
// where one warp's full tile would not fit in registers.  Warps holding the
// same outputs are summed in warp order through shared memory.
template <int BM, int BK, int R, int S>
__global__ void __launch_bounds__(256) k_mvtmv_dmma(MvTmvArgs<double> a, const __grid_constant__ CUtensorMap mapV,
                                                    const __grid_constant__ CUtensorMap mapW, int* err)
{
  constexpr int MT = BM / 8, NT = BK / 8;
  constexpr int WS = (MT * NT > 32) ? 2 : 1;  // warps sharing the rows of one step
  constexpr int MTW = MT / WS;
  constexpr int PV = BM + 4, PW = BK + 4;
  constexpr int KSTEPS = R / 4, WQ = 8 / WS;  // 4-row steps per stage, warps per output slice
  constexpr unsigned STAGE_BYTES = (unsigned)(R * (PV + PW) * sizeof(double));
  static_assert(BM % 8 == 0 && BK % 8 == 0 && R % 32 == 0 && R <= 256 && S >= 2, "bad tile shape");
  extern __shared__ __align__(128) unsigned char smem_raw[];
  double* sV = reinterpret_cast<double*>(smem_raw);  // [S][R][PV]
  double* sW = sV + S * R * PV;                       // [S][R][PW]
  uint64_t* bar = reinterpret_cast<uint64_t*>(sW + S * R * PW);
  const int tid = threadIdx.x, lane = tid & 31, w = tid >> 5;
  const int g = lane >> 2, t = lane & 3;
  const int mh = w % WS, wq = w / WS;
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

  double acc[MTW][NT][2];
#pragma unroll
  for (int i = 0; i < MTW; i++)
#pragma unroll
    for (int j = 0; j < NT; j++) acc[i][j][0] = acc[i][j][1] = 0.0;

  bool ok = true;
  int stage = 0;
  int64_t it = 0;
  for (int64_t tile = blockIdx.x; tile < ntiles; tile += gridDim.x, it++) {
    if (tid == 0) {
      const int64_t nt = tile + (int64_t)(S - 1) * gridDim.x;
      const int ps = (stage + S - 1) % S;
      if (nt < ntiles) {
        mbar_arrive_expect_tx(&bar[ps], STAGE_BYTES);
        tma_load_2d(sV + ps * R * PV, &mapV, 0, (int)(nt * R), &bar[ps]);
        tma_load_2d(sW + ps * R * PW, &mapW, 0, (int)(nt * R), &bar[ps]);
      }
    }
    const bool landed = mbar_wait(&bar[stage], (unsigned)((it / S) & 1), err);
    ok = ok && landed;
    if (ok) {
      const double* v0 = sV + stage * R * PV;
      const double* w0 = sW + stage * R * PW;
#pragma unroll 2
      for (int ks = wq; ks < KSTEPS; ks += WQ) {
        const int r = ks * 4 + t;  // this lane's row of the step
        double av[MTW], bw[NT];
#pragma unroll
        for (int i = 0; i < MTW; i++) av[i] = v0[r * PV + (mh * MTW + i) * 8 + g];
#pragma unroll
        for (int j = 0; j < NT; j++) bw[j] = w0[r * PW + j * 8 + g];
#pragma unroll
        for (int i = 0; i < MTW; i++)
#pragma unroll
          for (int j = 0; j < NT; j++) dmma_884(acc[i][j][0], acc[i][j][1], av[i], bw[j]);
      }
    }
    __syncthreads();
    stage = (stage + 1) % S;
  }
  // sum the WQ warps of every output slice in warp order (reuses the staging)
  double* red = sV;  // [BM*BK], column-major i + j*BM
  for (int q = 0; q < WQ; q++) {
    if (wq == q) {
#pragma unroll
      for (int i = 0; i < MTW; i++)
#pragma unroll
        for (int j = 0; j < NT; j++)
#pragma unroll
          for (int e = 0; e < 2; e++) {
            const int row = (mh * MTW + i) * 8 + g, col = j * 8 + 2 * t + e;
            double* dst = red + row + col * BM;
            *dst = (q == 0) ? acc[i][j][e] : *dst + acc[i][j][e];
          }
    }
    __syncthreads();
  }
  const int nout = a.m * a.k;
  double* part = a.part + (int64_t)blockIdx.x * nout;
  for (int o = tid; o < nout; o += blockDim.x) part[o] = red[(o % a.m) + (o / a.m) * BM];
  if (a.ext_reduce) return;  // second pass: k_reduce_partials
  last_block_reduce<double>(a.part, nout, gridDim.x, a.counter, a.Cd, 1, a.m, a.ldc, a.alpha, a.beta);
}

// ------------------------------------------------------------------ V*C
// W tile (R x k) = A tile (R x m) * C (m x k).  Warp w owns rows
// [w*RW, (w+1)*RW) of the stage (RW = R/8, RW/8 row tiles) and all BK/8
// column tiles; the m-dimension is stepped 4 columns per DMMA.  C sits in
// shared memory row-major with pitch CP = BK + 4, zero-padded.
template <int BM, int BK, int R, int S>
__global__ void __launch_bounds__(256) k_mvsd_dmma(RowGemmArgs<double> a, const __grid_constant__ CUtensorMap mapA,
                                                   int* err)
{
  constexpr int NT = BK / 8, RW = R / 8, RT8 = RW / 8;
  constexpr int AP = BM + 4, CP = BK + 4;
  constexpr int CSZ = (BM * CP * 8 + 127) / 128 * 128 / 8;
  constexpr unsigned STAGE_BYTES = (unsigned)(R * AP * sizeof(double));
  static_assert(BM % 8 == 0 && BK % 8 == 0 && R % 64 == 0 && R <= 256 && S >= 2, "bad tile shape");
  extern __shared__ __align__(128) unsigned char smem_raw[];
  double* sC = reinterpret_cast<double*>(smem_raw);  // [BM][CP]
  double* sA = sC + CSZ;                              // [S][R][AP]
  uint64_t* bar = reinterpret_cast<uint64_t*>(sA + S * R * AP);
  const int tid = threadIdx.x, lane = tid & 31, w = tid >> 5;
  const int g = lane >> 2, t = lane & 3;
  const bool inplace = (a.mode == RM_MVSDI);
  const int64_t ntiles = (a.n + R - 1) / R;

  if (tid == 0) {
    for (int st = 0; st < S; st++) mbar_init(&bar[st], 1);
    mbar_fence_init();
    tma_prefetch_desc(&mapA);
  }
  for (int q = tid; q < BM * CP; q += blockDim.x) {
    const int i = q / CP, j = q - i * CP;
    sC[q] = (i < a.m && j < a.k) ? a.C[i + (int64_t)j * a.ldc] : 0.0;
  }
  __syncthreads();
  if (tid == 0) {
    for (int st = 0; st < S - 1; st++) {
      const int64_t tl = blockIdx.x + (int64_t)st * gridDim.x;
      if (tl < ntiles) {
        mbar_arrive_expect_tx(&bar[st], STAGE_BYTES);
        tma_load_2d(sA + st * R * AP, &mapA, 0, (int)(tl * R), &bar[st]);
      }
    }
  }

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
      const double* a0 = sA + stage * R * AP;
      double acc[RT8][NT][2];
#pragma unroll
      for (int r8 = 0; r8 < RT8; r8++)
#pragma unroll
        for (int j = 0; j < NT; j++) acc[r8][j][0] = acc[r8][j][1] = 0.0;
#pragma unroll 4
      for (int kk = 0; kk < BM; kk += 4) {
        double av[RT8], bc[NT];
#pragma unroll
        for (int r8 = 0; r8 < RT8; r8++) av[r8] = a0[(w * RW + r8 * 8 + g) * AP + kk + t];
#pragma unroll
        for (int j = 0; j < NT; j++) bc[j] = sC[(kk + t) * CP + j * 8 + g];
#pragma unroll
        for (int r8 = 0; r8 < RT8; r8++)
#pragma unroll
          for (int j = 0; j < NT; j++) dmma_884(acc[r8][j][0], acc[r8][j][1], av[r8], bc[j]);
      }
      const int64_t r0 = tile * R + w * RW;
#pragma unroll
      for (int r8 = 0; r8 < RT8; r8++) {
        const int64_t row = r0 + r8 * 8 + g;
        if (row >= a.n) continue;
        double* wr = a.W + row * a.ldw;
#pragma unroll
        for (int j = 0; j < NT; j++)
#pragma unroll
          for (int e = 0; e < 2; e++) {
            const int col = j * 8 + 2 * t + e;
            if (col < a.k) {
              const double v = acc[r8][j][e];
              if (inplace) wr[col] = v;
              else wr[col] = (a.beta != 0.0) ? a.alpha * v + a.beta * wr[col] : a.alpha * v;
            }
          }
      }
    }
    __syncthreads();
    stage = (stage + 1) % S;
  }
}

// ------------------------------------------------------- V*C fused with a Gram
// One pass for PHIST's fused_mvsd_mvTmv and fused_mvsdi_mvTmv
// (phist_kernels_fused_decl.h:84,92): the new W tile is computed as in
// k_mvsd_dmma, written to global memory and kept in shared memory (pitch
// PT = BK + 4), and the Gram product of the tile is accumulated right away
//   GM == GM_WW : G  = W'W              (GMR = BK rows)
//   GM == GM_VW : D  = galpha V'W + gbeta D, V staged by TMA with A (GMR = MV)
// with the warp split and fixed-order reduction of k_mvtmv_dmma.  W is not
// read back from HBM.
template <int BM, int BK, int MV, int R, int S, int GM>
__global__ void __launch_bounds__(256) k_mvsd_gram_dmma(RowGemmArgs<double> a,
                                                        const __grid_constant__ CUtensorMap mapA,
                                                        const __grid_constant__ CUtensorMap mapV, int* err)
{
  constexpr int NT = BK / 8, RW = R / 8, RT8 = RW / 8;
  constexpr int AP = BM + 4, CP = BK + 4, PT = BK + 4, PVG = MV + 4;
  constexpr int GMR = (GM == GM_WW) ? BK : MV;
  constexpr int MTG = GMR / 8, NTG = BK / 8;
  constexpr int WS = (MTG * NTG > 32) ? 2 : 1, MTW = MTG / WS, WQ = 8 / WS, KSTEPS = R / 4;
  constexpr int CSZ = (BM * CP * 8 + 127) / 128 * 128 / 8;
  constexpr int VSZ = (GM == GM_VW) ? R * PVG : 0;
  constexpr unsigned STAGE_BYTES = (unsigned)((R * AP + VSZ) * sizeof(double));
  static_assert(BM % 8 == 0 && BK % 8 == 0 && MV % 8 == 0 && R % 64 == 0 && R <= 256 && S >= 2, "bad shape");
  extern __shared__ __align__(128) unsigned char smem_raw[];
  double* sC = reinterpret_cast<double*>(smem_raw);  // [BM][CP]
  double* sA = sC + CSZ;                              // [S][R][AP]
  double* sV = sA + S * R * AP;                       // [S][R][PVG] (GM_VW)
  double* sT = sV + S * VSZ;                          // [R][PT] new W tile
  uint64_t* bar = reinterpret_cast<uint64_t*>(sT + R * PT);
  const int tid = threadIdx.x, lane = tid & 31, w = tid >> 5;
  const int g = lane >> 2, t = lane & 3;
  const int mh = w % WS, wq = w / WS;
  const bool inplace = (a.mode == RM_MVSDI);
  const int64_t ntiles = (a.n + R - 1) / R;

  if (tid == 0) {
    for (int st = 0; st < S; st++) mbar_init(&bar[st], 1);
    mbar_fence_init();
    tma_prefetch_desc(&mapA);
    if (GM == GM_VW) tma_prefetch_desc(&mapV);
  }
  for (int q = tid; q < BM * CP; q += blockDim.x) {
    const int i = q / CP, j = q - i * CP;
    sC[q] = (i < a.m && j < a.k) ? a.C[i + (int64_t)j * a.ldc] : 0.0;
  }
  __syncthreads();
  auto issue = [&](int st, int64_t tl) {
    mbar_arrive_expect_tx(&bar[st], STAGE_BYTES);
    tma_load_2d(sA + st * R * AP, &mapA, 0, (int)(tl * R), &bar[st]);
    if (GM == GM_VW) tma_load_2d(sV + st * VSZ, &mapV, 0, (int)(tl * R), &bar[st]);
  };
  if (tid == 0)
    for (int st = 0; st < S - 1; st++) {
      const int64_t tl = blockIdx.x + (int64_t)st * gridDim.x;
      if (tl < ntiles) issue(st, tl);
    }

  double gacc[MTW][NTG][2];
#pragma unroll
  for (int i = 0; i < MTW; i++)
#pragma unroll
    for (int j = 0; j < NTG; j++) gacc[i][j][0] = gacc[i][j][1] = 0.0;

  bool ok = true;
  int stage = 0;
  int64_t it = 0;
  for (int64_t tile = blockIdx.x; tile < ntiles; tile += gridDim.x, it++) {
    if (tid == 0) {
      const int64_t nt = tile + (int64_t)(S - 1) * gridDim.x;
      if (nt < ntiles) issue((stage + S - 1) % S, nt);
    }
    const bool landed = mbar_wait(&bar[stage], (unsigned)((it / S) & 1), err);
    ok = ok && landed;
    if (ok) {
      // ---- the new W tile: DMMA, written to HBM and to sT
      const double* a0 = sA + stage * R * AP;
      double acc[RT8][NT][2];
#pragma unroll
      for (int r8 = 0; r8 < RT8; r8++)
#pragma unroll
        for (int j = 0; j < NT; j++) acc[r8][j][0] = acc[r8][j][1] = 0.0;
#pragma unroll 4
      for (int kk = 0; kk < BM; kk += 4) {
        double av[RT8], bc[NT];
#pragma unroll
        for (int r8 = 0; r8 < RT8; r8++) av[r8] = a0[(w * RW + r8 * 8 + g) * AP + kk + t];
#pragma unroll
        for (int j = 0; j < NT; j++) bc[j] = sC[(kk + t) * CP + j * 8 + g];
#pragma unroll
        for (int r8 = 0; r8 < RT8; r8++)
#pragma unroll
          for (int j = 0; j < NT; j++) dmma_884(acc[r8][j][0], acc[r8][j][1], av[r8], bc[j]);
      }
      const int64_t r0 = tile * R;
#pragma unroll
      for (int r8 = 0; r8 < RT8; r8++) {
        const int lr = w * RW + r8 * 8 + g;  // row inside the tile
        const int64_t row = r0 + lr;
        double* wr = a.W + row * a.ldw;
#pragma unroll
        for (int j = 0; j < NT; j++)
#pragma unroll
          for (int e = 0; e < 2; e++) {
            const int col = j * 8 + 2 * t + e;
            double v = 0.0;
            if (row < a.n && col < a.k) {
              v = acc[r8][j][e];
              if (!inplace) v = (a.beta != 0.0) ? a.alpha * v + a.beta * wr[col] : a.alpha * v;
              wr[col] = v;
            }
            sT[lr * PT + col] = v;
          }
      }
    }
    __syncthreads();  // sT complete
    if (ok) {
      // ---- Gram of the tile: A operand rows from sT (W'W) or the V tile (V'W)
      const double* gl = (GM == GM_WW) ? sT : sV + stage * VSZ;
      constexpr int GP = (GM == GM_WW) ? PT : PVG;
#pragma unroll 2
      for (int ks = wq; ks < KSTEPS; ks += WQ) {
        const int r = ks * 4 + t;
        double av[MTW], bw[NTG];
#pragma unroll
        for (int i = 0; i < MTW; i++) av[i] = gl[r * GP + (mh * MTW + i) * 8 + g];
#pragma unroll
        for (int j = 0; j < NTG; j++) bw[j] = sT[r * PT + j * 8 + g];
#pragma unroll
        for (int i = 0; i < MTW; i++)
#pragma unroll
          for (int j = 0; j < NTG; j++) dmma_884(gacc[i][j][0], gacc[i][j][1], av[i], bw[j]);
      }
    }
    __syncthreads();  // stage and sT free for reuse
    stage = (stage + 1) % S;
  }
  // sum the WQ warps of every output slice in warp order
  double* red = reinterpret_cast<double*>(smem_raw);  // [GMR*BK], column-major
  for (int q = 0; q < WQ; q++) {
    if (wq == q) {
#pragma unroll
      for (int i = 0; i < MTW; i++)
#pragma unroll
        for (int j = 0; j < NTG; j++)
#pragma unroll
          for (int e = 0; e < 2; e++) {
            const int row = (mh * MTW + i) * 8 + g, col = j * 8 + 2 * t + e;
            double* dst = red + row + col * GMR;
            *dst = (q == 0) ? gacc[i][j][e] : *dst + gacc[i][j][e];
          }
    }
    __syncthreads();
  }
  const int gm = (GM == GM_WW) ? a.k : a.mv;
  const int nout = gm * a.k;
  double* part = a.part + (int64_t)blockIdx.x * nout;
  for (int o = tid; o < nout; o += blockDim.x) part[o] = red[(o % gm) + (o / gm) * GMR];
  if (a.R < 0) return;  // second pass: k_reduce_partials (launcher sets R = -1)
  last_block_reduce<double>(a.part, nout, gridDim.x, a.counter, a.Gd, 1, gm, a.ldg, a.galpha, a.gbeta);
}

}  // namespace pb
