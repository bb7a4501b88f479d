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

namespace pb {

// a block's partial W'W and V'W: output o = c1 + NV*c2 (column-major NV x NV)
template <class T, int NV, int NT, int NQ, class GT>
__device__ __forceinline__ void gram_store(const SpmvArgs<T>& p, const GT* gw, const GT* gv)
{
#pragma unroll
  for (int q = 0; q < NQ; q++) {
    const int o = threadIdx.x + q * NT;
    if (o < NV * NV) {
      if (p.gram_w) p.gram_w[(int64_t)blockIdx.x * NV * NV + o] = T(gw[q]);
      if (p.gram_v) p.gram_v[(int64_t)blockIdx.x * NV * NV + o] = T(gv[q]);
    }
  }
}

template <class T, int NV, int TPR, int NT, bool GRAM = false>
__global__ void __launch_bounds__(NT) k_sell_spmmv_pf(SellDev<T> A, SpmvArgs<T> p)
{
  constexpr int KMAX = 8, CC = 32;
  constexpr int VPT = NV / TPR;
  constexpr int VWMAX = 16 / sizeof(T);
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
  // GRAM: the tile's new W rows and X rows (padded rows: no bank conflicts)
  constexpr int GR = GRAM ? RPB : 1;
  constexpr int NQ = GRAM ? (NV * NV + NT - 1) / NT : 1;  // products per thread
  __shared__ T gys[GR][GRAM ? NV + 1 : 1];
  __shared__ T gxs[GR][GRAM ? NV + 1 : 1];
  typedef typename Acc<T>::type GT;
  GT gw[NQ], gv[NQ];
#pragma unroll
  for (int q = 0; q < NQ; q++) { gw[q] = GT(0); gv[q] = GT(0); }

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
    if (GRAM) gram_store<T, NV, NT, NQ>(p, gw, gv);
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
    if (GRAM) {
      // rows past the matrix add nothing to the products
#pragma unroll
      for (int v = 0; v < NVV; v++)
#pragma unroll
        for (int w = 0; w < VW; w++) {
          gys[lr][spmv_col<TPR, VW>(s, v, w)] = T(0);
          gxs[lr][spmv_col<TPR, VW>(s, v, w)] = T(0);
        }
    }
    if (r < nch * (int64_t)CC) {
      const int64_t i = (r < A.nrows) ? (A.perm ? (int64_t)A.perm[r] : r) : -1;
      AT acc[VPT];
#pragma unroll
      for (int q = 0; q < VPT; q++) acc[q] = AT(0);
      T xi[VPT];
      if (i >= 0 && (p.has_shift || (GRAM && p.gram_v))) {
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
          if (GRAM) {
#pragma unroll
            for (int w = 0; w < VW; w++) {
              gys[lr][c + w] = yv[w];
              if (p.gram_v) gxs[lr][c + w] = xi[v * VW + w];
            }
          }
        }
      }
    }
    if (GRAM) {
      // this tile's share of W'W and V'W, rows in tile order
      __syncthreads();
#pragma unroll
      for (int q = 0; q < NQ; q++) {
        const int o = tid + q * NT;
        if (o < NV * NV) {
          const int c1 = o % NV, c2 = o / NV;
#pragma unroll 4
          for (int rr = 0; rr < RPB; rr++) {
            const T y2 = gys[rr][c2];
            if (p.gram_w) gw[q] += GT(gys[rr][c1]) * GT(y2);
            if (p.gram_v) gv[q] += GT(gxs[rr][c1]) * GT(y2);
          }
        }
      }
    }
    cp_async_wait<0>();
    if (tid <= NCH) smeta[mbnn][tid] = mnext;
    __syncthreads();
  }
  if (GRAM) gram_store<T, NV, NT, NQ>(p, gw, gv);
}

}  // namespace pb
