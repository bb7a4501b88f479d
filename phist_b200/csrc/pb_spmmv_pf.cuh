// pb_spmmv_pf.cuh -- SpMMV with the next tile's matrix entries prefetched
// into shared memory while the current tile gathers X.
//
// In the one-tile-per-block kernel (pb_spmmv.cuh) every warp runs a chain
// of three dependent global loads: the chunk pointer, then the chunk's
// values and columns, then the X rows those columns name.  While the values
// and columns are in flight a warp has a few hundred bytes outstanding, and
// the SMs sit at 35-40 % of DRAM bandwidth with no unit saturated (ncu on the
// L=128 Anderson matrix at nvec = 32: DRAM 39 %, L2 37 %, L1 53 %, 34 cycles
// per issued instruction with 45 warps per SM).
//
// Here a resident grid walks the tiles in grid-stride order (so the GPU as a
// whole still sweeps the rows in order and X rows shared by neighbouring
// tiles are found in L2).  Per block and tile:
//   * the chunk pointers of the tile after next are loaded into registers,
//   * the values and columns of the next tile (one contiguous range of the
//     SELL arrays) are copied into a shared-memory buffer with cp.async,
//   * the current tile reads its entries from shared memory, gathers its X
//     rows and writes Y,
// so a tile costs one memory latency (the X gathers) instead of three, and
// the next tile's entries arrive meanwhile.
//
// The arithmetic is k_sell_spmmv's term for term: tmp = shift*x_i, the row's
// entries in stored order, y = alpha*tmp + beta*y (spmvm_kernels.F90:494-523);
// results are bitwise those of the one-tile kernel.
//
// With GRAM set, the kernel also forms W'W and V'W of the new W in the same
// pass (fused_spmv_mvTmv, phist_kernels_fused_decl.h:57-68): each tile's W
// rows (and its own X rows, for V'W) are kept in shared memory, every thread
// accumulates its share of the NV x NV products over the tile's rows, and
// each block leaves its partial sums for a fixed-order second pass.
//
// Preconditions (checked by the launcher): SELL chunk height 32, at most 8
// entries per row, no fused dot / axpby epilogue, the whole block vector as
// the column tile when GRAM is set.
#pragma once
#include "pb_spmmv.cuh"
#include "pb_tile.cuh"
#include "pb_dmma.cuh"
#include <type_traits>

namespace pb {

// Per-block accumulation of W'W and V'W over the tiles' rows kept in shared
// memory (ys: new W rows, xs: the rows' own X rows, row pitch PY), and the
// block's partial sums at the end: output o = c1 + NV*c2 (column-major
// NV x NV) at gram_w / gram_v + blockIdx.x*NV*NV.
//
// Scalar form (any width): each thread holds a TM x TM micro-tile of both
// products over one row group (rows g, g + RG, ... of every tile); NMT
// micro-tiles x RG groups = NT threads; the groups are added in group order.
template <class T, int NV, int NT, int RPB>
struct GramScalar {
  typedef typename Acc<T>::type GT;
  static constexpr int PY = NV + 1;
  static constexpr int TM = NV >= 4 ? 2 : 1;
  static constexpr int NB = NV / TM;
  static constexpr int NMT = NB * NB;
  static constexpr int RG = NMT >= NT ? 1 : NT / NMT;
  static_assert(NMT <= NT, "one micro-tile per thread at most");
  static_assert(RPB * PY >= NT * TM * TM, "group partials fit the row buffer");
  GT gw[TM][TM], gv[TM][TM];
  int c1, c2, g;
  __device__ __forceinline__ void init()
  {
    const int mt = (int)threadIdx.x % NMT;
    g = (int)threadIdx.x / NMT;
    c1 = (mt % NB) * TM;
    c2 = (mt / NB) * TM;
#pragma unroll
    for (int a = 0; a < TM; a++)
#pragma unroll
      for (int b = 0; b < TM; b++) { gw[a][b] = GT(0); gv[a][b] = GT(0); }
  }
  __device__ __forceinline__ void add_tile(const T* ys, const T* xs)
  {
    if (g >= RG) return;
#pragma unroll 2
    for (int rr = g; rr < RPB; rr += RG) {
      T y1[TM], y2[TM], x1[TM];
#pragma unroll
      for (int a = 0; a < TM; a++) {
        y1[a] = ys[rr * PY + c1 + a];
        y2[a] = ys[rr * PY + c2 + a];
        x1[a] = xs[rr * PY + c1 + a];
      }
#pragma unroll
      for (int a = 0; a < TM; a++)
#pragma unroll
        for (int b = 0; b < TM; b++) {
          gw[a][b] += GT(y1[a]) * GT(y2[b]);
          gv[a][b] += GT(x1[a]) * GT(y2[b]);
        }
    }
  }
  // buf: RPB*PY entries of shared memory, free on entry
  __device__ __forceinline__ void store(const SpmvArgs<T>& p, T* buf)
  {
    for (int which = 0; which < 2; which++) {
      T* out = which == 0 ? p.gram_w : p.gram_v;
      __syncthreads();
      if (out) {
#pragma unroll
        for (int a = 0; a < TM; a++)
#pragma unroll
          for (int b = 0; b < TM; b++)
            buf[(threadIdx.x * TM + a) * TM + b] = T(which == 0 ? gw[a][b] : gv[a][b]);
      }
      __syncthreads();
      if (out) {
        for (int o = threadIdx.x; o < NV * NV; o += NT) {
          const int i = o % NV, j = o / NV;
          const int mt = (i / TM) + NB * (j / TM), a = i % TM, b = j % TM;
          GT sum = GT(0);
          for (int q = 0; q < RG; q++) sum += GT(buf[((q * NMT + mt) * TM + a) * TM + b]);
          out[(int64_t)blockIdx.x * NV * NV + o] = T(sum);
        }
      }
    }
  }
};

// FP64 tensor-core form (NV a multiple of 16): the tile's Gram products as
// DMMA m8n8k4 steps with the row index as the k dimension (fragment layout
// as in pb_dmma.cuh: a = A[g][t], b = B[t][g], d = D[g][2t..2t+1]).  The
// MT x MT output tiles of 8 x 8 are spread over the warps; where there are
// fewer tiles than warps, warps with the same tile take interleaved 4-row
// steps (KG groups) and are added in group order at the end.  Row pitch
// NV + 4: the 4 rows of a fragment start 8 banks apart.
template <int NV, int NT, int RPB>
struct GramDmma {
  static constexpr int PY = NV + 4;
  static constexpr int MT = NV / 8;
  static constexpr int NW = NT / 32;
  static constexpr int TPW = MT * MT >= NW ? MT * MT / NW : 1;  // output tiles per warp
  static constexpr int KG = MT * MT >= NW ? 1 : NW / (MT * MT);  // k-step groups
  static constexpr int KS = RPB / 4;
  static_assert(NV % 8 == 0 && RPB % 4 == 0 && KS % KG == 0, "bad DMMA Gram shape");
  static_assert(RPB * PY >= KG * NV * NV, "group partials fit the row buffer");
  double dw[TPW][2], dv[TPW][2];
  int w, kg;
  __device__ __forceinline__ void init()
  {
    w = (int)threadIdx.x >> 5;
    kg = w / (MT * MT >= NW ? NW : MT * MT);
#pragma unroll
    for (int q = 0; q < TPW; q++) dw[q][0] = dw[q][1] = dv[q][0] = dv[q][1] = 0.0;
  }
  __device__ __forceinline__ int tile_of(int q) const
  {
    return MT * MT >= NW ? w * TPW + q : w % (MT * MT);
  }
  __device__ __forceinline__ void add_tile(const double* ys, const double* xs)
  {
    const int lane = threadIdx.x & 31, g8 = lane >> 2, t4 = lane & 3;
#pragma unroll 2
    for (int ks = kg; ks < KS; ks += KG) {
      const int r = ks * 4 + t4;
#pragma unroll
      for (int q = 0; q < TPW; q++) {
        const int tl = tile_of(q), i = tl % MT, j = tl / MT;
        const double a = ys[r * PY + i * 8 + g8];
        const double ax = xs[r * PY + i * 8 + g8];
        const double b = ys[r * PY + j * 8 + g8];
        dmma_884(dw[q][0], dw[q][1], a, b);
        dmma_884(dv[q][0], dv[q][1], ax, b);
      }
    }
  }
  __device__ __forceinline__ void store(const SpmvArgs<double>& p, double* buf)
  {
    const int lane = threadIdx.x & 31, g8 = lane >> 2, t4 = lane & 3;
    for (int which = 0; which < 2; which++) {
      double* out = which == 0 ? p.gram_w : p.gram_v;
      __syncthreads();
      if (out) {
#pragma unroll
        for (int q = 0; q < TPW; q++) {
          const int tl = tile_of(q), i = tl % MT, j = tl / MT;
          const int c1 = i * 8 + g8, c2 = j * 8 + 2 * t4;
          const double* d = which == 0 ? dw[q] : dv[q];
          buf[kg * NV * NV + c1 + NV * c2] = d[0];
          buf[kg * NV * NV + c1 + NV * (c2 + 1)] = d[1];
        }
      }
      __syncthreads();
      if (out) {
        for (int o = threadIdx.x; o < NV * NV; o += NT) {
          double sum = 0.0;
          for (int q = 0; q < KG; q++) sum += buf[q * NV * NV + o];
          out[(int64_t)blockIdx.x * NV * NV + o] = sum;
        }
      }
    }
  }
};

struct GramNone {
  static constexpr int PY = 1;
  __device__ __forceinline__ void init() {}
};

template <class T, int NV, int NT, int RPB>
struct GramPick {
  typedef GramScalar<T, NV, NT, RPB> type;
};
template <int NV, int NT, int RPB>
struct GramPick<double, NV, NT, RPB> {
  // widths 16 and 32 (at 8 the padded rows of the DMMA form exceed the
  // static shared memory next to the prefetch buffers)
  typedef typename std::conditional<NV % 16 == 0, GramDmma<NV, NT, RPB>, GramScalar<double, NV, NT, RPB>>::type type;
};

// VB: bytes per vector load and store of an X or Y row segment (16, or 32
// with the 256-bit forms when rows start on 32-byte boundaries)
template <class T, int NV, int TPR, int NT, bool GRAM, int VB>
__device__ __forceinline__ void sell_spmmv_pf(const SellDev<T>& A, const SpmvArgs<T>& p)
{
  constexpr int KMAX = 8, CC = 32;
  constexpr int VPT = NV / TPR;
  constexpr int VWMAX = VB / sizeof(T);
  constexpr int VW = VPT < VWMAX ? VPT : VWMAX;
  constexpr int NVV = VPT / VW;
  constexpr int RPB = NT / TPR;        // rows per tile
  constexpr int NCH = RPB / CC;        // chunks per tile
  constexpr int EPT = NCH * KMAX * CC; // entries per tile at most
  static_assert(RPB % CC == 0, "a tile is a whole number of chunks");
  typedef typename Acc<T>::type AT;
  __shared__ __align__(16) T sval[2][EPT];
  __shared__ __align__(16) int scol[2][EPT];
  __shared__ int64_t smeta[3][NCH + 1];  // chunk pointers of three tiles
  // GRAM: the tile's new W rows and X rows, and the block's accumulators
  typedef typename std::conditional<GRAM, typename GramPick<T, NV, NT, RPB>::type, GramNone>::type Gram;
  constexpr int PY = GRAM ? Gram::PY : 1;
  constexpr int GR = GRAM ? RPB : 1;
  __shared__ __align__(16) T gys[GR * PY];
  __shared__ __align__(16) T gxs[GR * PY];
  Gram gram;
  if constexpr (GRAM) gram.init();

  const int tid = threadIdx.x;
  const int s = tid % TPR, lr = tid / TPR;
  const int64_t nch = A.nchunks;
  const int64_t ntiles = (nch + NCH - 1) / NCH;
  const int64_t G = gridDim.x;
  const T* __restrict__ x = p.x + p.col0;

  // chunk pointer tid (0..NCH) of tile t, clamped to the end of the arrays
  auto meta_load = [&](int64_t t) -> int64_t {
    if (t >= ntiles || tid > NCH) return 0;
    int64_t c = t * NCH + tid;
    if (c > nch) c = nch;
    return A.chunk_ptr[c];
  };
  // values and columns of tile t (one contiguous range, a multiple of 32
  // entries, so of 128 bytes) into buffer buf, with its pointers in smeta[mb]
  auto copy_entries = [&](int64_t t, int buf, int mb) {
    if (t >= ntiles) return;
    const int64_t ncl = nch - t * NCH < NCH ? nch - t * NCH : NCH;
    const int64_t p0 = smeta[mb][0];
    const int64_t ne = smeta[mb][ncl] - p0;
    const int nv16 = (int)(ne * (int64_t)sizeof(T) / 16);
    const int nc16 = (int)(ne / 4);
    constexpr int EV = 16 / (int)sizeof(T);
    for (int q = tid; q < nv16 + nc16; q += NT) {
      if (q < nv16)
        cp_async16(&sval[buf][q * EV], A.val + p0 + (int64_t)q * EV, true);
      else
        cp_async16(&scol[buf][(q - nv16) * 4], A.col + p0 + (int64_t)(q - nv16) * 4, true);
    }
  };

  int64_t t = blockIdx.x;
  if (t >= ntiles) {
    if constexpr (GRAM) gram.store(p, gys);
    return;
  }
  {
    const int64_t m0 = meta_load(t);
    const int64_t m1 = meta_load(t + G);
    if (tid <= NCH) {
      smeta[0][tid] = m0;
      smeta[1][tid] = m1;
    }
    __syncthreads();
    copy_entries(t, 0, 0);
    cp_async_commit();
    cp_async_wait<0>();
    __syncthreads();
  }
  for (int it = 0; t < ntiles; t += G, it++) {
    const int buf = it & 1;
    const int mb = it % 3, mbn = (it + 1) % 3, mbnn = (it + 2) % 3;
    const int64_t mnext = meta_load(t + 2 * G);  // consumed after this tile
    copy_entries(t + G, buf ^ 1, mbn);
    cp_async_commit();

    const int64_t r = t * RPB + lr;  // SELL row
    if constexpr (GRAM) {
      // rows past the matrix add nothing to the products
#pragma unroll
      for (int v = 0; v < NVV; v++)
#pragma unroll
        for (int w = 0; w < VW; w++) {
          gys[lr * PY + spmv_col<TPR, VW>(s, v, w)] = T(0);
          gxs[lr * PY + spmv_col<TPR, VW>(s, v, w)] = T(0);
        }
    }
    if (r < nch * (int64_t)CC) {
      const int64_t i = (r < A.nrows) ? (A.perm ? (int64_t)A.perm[r] : r) : -1;
      AT acc[VPT];
#pragma unroll
      for (int q = 0; q < VPT; q++) acc[q] = AT(0);
      T xi[VPT];
      if constexpr (GRAM) {
        // the row's own X values: for the shift and for V'W
        if (i >= 0 && (p.has_shift || p.gram_v)) {
#pragma unroll
          for (int v = 0; v < NVV; v++) Vec<T, VW>::ld(x + i * p.ldx + spmv_col<TPR, VW>(s, v, 0), &xi[v * VW]);
        }
        if (i >= 0 && p.has_shift) {
#pragma unroll
          for (int v = 0; v < NVV; v++)
#pragma unroll
            for (int w = 0; w < VW; w++) {
              const int c = spmv_col<TPR, VW>(s, v, w);
              acc[v * VW + w] = AT(p.sh[c]) * AT(xi[v * VW + w]);
            }
        }
      } else {
        if (i >= 0 && p.has_shift) {
          T xs[VPT];
#pragma unroll
          for (int v = 0; v < NVV; v++) Vec<T, VW>::ld(x + i * p.ldx + spmv_col<TPR, VW>(s, v, 0), &xs[v * VW]);
#pragma unroll
          for (int v = 0; v < NVV; v++)
#pragma unroll
            for (int w = 0; w < VW; w++) {
              const int c = spmv_col<TPR, VW>(s, v, w);
              acc[v * VW + w] = AT(p.sh[c]) * AT(xs[v * VW + w]);
            }
        }
      }
      const int lc = lr / CC, l = lr % CC;
      const int cb = (int)(smeta[mb][lc] - smeta[mb][0]) + l;
      const int len = (int)((smeta[mb][lc + 1] - smeta[mb][lc]) / CC);
      T av[KMAX];
      int cv[KMAX];
#pragma unroll
      for (int k = 0; k < KMAX; k++) {
        av[k] = T(0);
        cv[k] = 0;
        if (k < len) {
          av[k] = sval[buf][cb + k * CC];
          cv[k] = scol[buf][cb + k * CC];
        }
      }
#pragma unroll
      for (int k = 1; k < KMAX; k++)
        if (k >= len) cv[k] = cv[0];
      T xv[KMAX][VPT];
#pragma unroll
      for (int k = 0; k < KMAX; k++) {
        const T* xr = x + (int64_t)cv[k] * p.ldx;
#pragma unroll
        for (int v = 0; v < NVV; v++) Vec<T, VW>::ld_ordered(xr + spmv_col<TPR, VW>(s, v, 0), &xv[k][v * VW]);
      }
#pragma unroll
      for (int k = 0; k < KMAX; k++)
#pragma unroll
        for (int q = 0; q < VPT; q++) reg_fence(xv[k][q]);
#pragma unroll
      for (int k = 0; k < KMAX; k++)
        if (k < len)
#pragma unroll
          for (int q = 0; q < VPT; q++) acc[q] += AT(av[k]) * AT(xv[k][q]);
      if (i >= 0) {
        T* yr = p.y + p.col0 + i * p.ldy;
#pragma unroll
        for (int v = 0; v < NVV; v++) {
          const int c = spmv_col<TPR, VW>(s, v, 0);
          T yv[VW];
          if (p.beta != T(0)) {
            Vec<T, VW>::ld_plain(yr + c, yv);
#pragma unroll
            for (int w = 0; w < VW; w++) yv[w] = T(AT(p.alpha) * acc[v * VW + w] + AT(p.beta) * AT(yv[w]));
          } else {
#pragma unroll
            for (int w = 0; w < VW; w++) yv[w] = T(AT(p.alpha) * acc[v * VW + w]);
          }
          if (!GRAM || !p.no_store) Vec<T, VW>::st(yr + c, yv);
          if constexpr (GRAM) {
#pragma unroll
            for (int w = 0; w < VW; w++) {
              gys[lr * PY + c + w] = yv[w];
              if (p.gram_v) gxs[lr * PY + c + w] = xi[v * VW + w];
            }
          }
        }
      }
    }
    if constexpr (GRAM) {
      // this tile's share of W'W and V'W
      __syncthreads();
      gram.add_tile(gys, gxs);
    }
    cp_async_wait<0>();
    if (tid <= NCH) smeta[mbnn][tid] = mnext;
    __syncthreads();
  }
  if constexpr (GRAM) gram.store(p, gys);
}

// The kernel comes in two entry points around the same body: with a minimum
// of resident blocks per SM handed to ptxas, which changes how it allocates
// registers and schedules the gathers, and without.  pf_min_blocks is the
// choice per form, measured on the L=128 Anderson matrix (FP64, 256-bit
// gathers; GB/s without -> with): plain SpMMV at width 4 (1 thread per row)
// 4,469 -> 4,748 with any minimum of 1..4, at 8 (2 per row) 4,728 -> 4,941
// and at 16 (4 per row) 4,358 -> 4,647 with 4, at 32 best without (4,575;
// 4,425 with 3 or 4); the single pass with W'W and V'W at widths 2 / 8 / 16
// 2,871 -> 3,015, 2,081 -> 2,206, 1,931 -> 2,081 with 4 / 3 / 4.  The FP32
// forms keep the plain entry point.
template <class T, int NV, int TPR, int NT, bool GRAM>
constexpr int pf_min_blocks()
{
  if (!std::is_same<T, double>::value) return 0;
  if (!GRAM) return ((NV == 4 && TPR == 1) || (NV == 8 && TPR == 2) || (NV == 16 && TPR == 4)) ? 4 : 0;
  return NV == 2 ? 4 : NV == 8 ? 3 : NV == 16 ? 4 : 0;
}

template <class T, int NV, int TPR, int NT, bool GRAM = false, int VB = 16>
__global__ void __launch_bounds__(NT) k_sell_spmmv_pf(SellDev<T> A, SpmvArgs<T> p)
{
  sell_spmmv_pf<T, NV, TPR, NT, GRAM, VB>(A, p);
}

template <class T, int NV, int TPR, int NT, bool GRAM, int VB, int MB>
__global__ void __launch_bounds__(NT, MB) k_sell_spmmv_pf_mb(SellDev<T> A, SpmvArgs<T> p)
{
  sell_spmmv_pf<T, NV, TPR, NT, GRAM, VB>(A, p);
}

// the entry point of a form
template <class T, int NV, int TPR, int NT, bool GRAM = false, int VB = 16>
constexpr auto pf_kernel()
{
  constexpr int mb = pf_min_blocks<T, NV, TPR, NT, GRAM>();
  if constexpr (mb > 0)
    return &k_sell_spmmv_pf_mb<T, NV, TPR, NT, GRAM, VB, mb>;
  else
    return &k_sell_spmmv_pf<T, NV, TPR, NT, GRAM, VB>;
}

}  // namespace pb
