// pb_spmmv_staged.cuh -- SpMMV for wide block vectors (nvec = 8..64) with
// the X rows staged in shared memory by cp.async.
//
// For wide vectors the gathers of X rows dominate, and when they are loaded
// into registers the bytes in flight per SM are capped by the register file.
// Here a block walks SELL chunks (C = 32 rows, at most 8 entries per row)
// with a software pipeline:
//   stage A(c+2): cp.async the chunk's col/val arrays into shared memory,
//   stage B(c+1): cp.async the X rows those columns address (up to
//                 8 x 32 rows of nvec values) into shared memory,
//   compute  (c): y = alpha*(shift*x_i + sum_k a_k x_{col_k}) + beta*y from
//                 shared memory, entries in stored (column) order.
// The copies for chunk c+1 are in flight while chunk c is computed.  Thread
// (row l, lane s) owns columns [s*VPT, s*VPT+VPT) of row l (8 threads per row).
#pragma once
#include "pb_spmmv.cuh"
#include "pb_tile.cuh"

namespace pb {

constexpr int ST_C = 32;     // chunk height
constexpr int ST_KMAX = 8;   // entries per row
constexpr int ST_TPR = 8;    // threads per row

template <class T, int NV>
struct StagedSmem {
  static constexpr int VW = 16 / sizeof(T);
  static constexpr int XP = NV + VW;  // padded X-row pitch in shared memory
  static constexpr size_t xbuf = (size_t)ST_KMAX * ST_C * XP;           // elements per X buffer
  static constexpr size_t bytes = sizeof(T) * 2 * xbuf                  // 2 X buffers
                                  + 3 * ST_KMAX * ST_C * (sizeof(T) + sizeof(int))  // 3 val/col
                                  + 16;
};

template <class T, int NV>
__global__ void __launch_bounds__(256) k_sell_spmmv_staged(SellDev<T> A, SpmvArgs<T> p)
{
  typedef StagedSmem<T, NV> SM;
  constexpr int VW = SM::VW, XP = SM::XP;
  constexpr int VPT = NV / ST_TPR;                 // values per thread
  constexpr int LW = VPT < VW ? VPT : VW;          // load width
  constexpr int NL = VPT / LW;                     // loads per thread per entry
  constexpr int CH = NV / VW;                      // 16-byte chunks per X row
  extern __shared__ __align__(16) unsigned char smem_raw[];
  T* xs = reinterpret_cast<T*>(smem_raw);                      // [2][KMAX][C][XP]
  T* vs = xs + 2 * SM::xbuf;                                    // [3][KMAX][C]
  int* cs = reinterpret_cast<int*>(vs + 3 * ST_KMAX * ST_C);    // [3][KMAX][C]

  const int tid = threadIdx.x;
  const int l = tid / ST_TPR, s = tid - l * ST_TPR;
  const T* __restrict__ x = p.x + p.col0;
  const int64_t nch = A.nchunks;

  // stage A: col/val of chunk ch into slot (16-byte copies, chunk arrays
  // are contiguous: len*32 entries from chunk_ptr)
  auto stage_a = [&](int64_t ch, int slot) {
    if (ch >= nch) return;
    const int len = A.chunk_len[ch];
    const int64_t base = A.chunk_ptr[ch];
    const int nvv = len * ST_C * (int)sizeof(T) / 16;   // val chunks
    const int ncc = len * ST_C * 4 / 16;                 // col chunks
    for (int q = tid; q < nvv + ncc; q += blockDim.x) {
      if (q < nvv)
        cp_async16(vs + slot * ST_KMAX * ST_C + q * (16 / sizeof(T)), A.val + base + q * (16 / sizeof(T)), true);
      else
        cp_async16(cs + slot * ST_KMAX * ST_C + (q - nvv) * 4, A.col + base + (q - nvv) * 4, true);
    }
  };
  // stage B: X rows addressed by chunk ch (its col slot is complete)
  auto stage_b = [&](int64_t ch, int slot, int buf) {
    if (ch >= nch) return;
    const int len = A.chunk_len[ch];
    const int* cc = cs + slot * ST_KMAX * ST_C;
    T* xb = xs + buf * SM::xbuf;
    const int tot = len * ST_C * CH;
    for (int q = tid; q < tot; q += blockDim.x) {
      const int e = q / CH, c = q - e * CH;          // e = k*C + lane
      const int64_t col = cc[e];
      cp_async16(xb + (size_t)e * XP + c * VW, x + col * p.ldx + c * VW, true);
    }
  };

  int64_t ch = blockIdx.x;
  const int64_t step = gridDim.x;
  stage_a(ch, 0);
  cp_async_commit();
  cp_async_wait<0>();
  __syncthreads();
  stage_b(ch, 0, 0);
  stage_a(ch + step, 1);
  cp_async_commit();
  int it = 0;
  for (; ch < nch; ch += step, it++) {
    const int slot = it % 3, buf = it & 1;
    cp_async_wait<0>();          // X rows of ch and col/val of ch+step are in
    __syncthreads();
    stage_b(ch + step, (it + 1) % 3, buf ^ 1);
    stage_a(ch + 2 * step, (it + 2) % 3);
    cp_async_commit();

    const int64_t r = ch * ST_C + l;
    const int64_t i = (r < A.nrows) ? (A.perm ? (int64_t)A.perm[r] : r) : -1;
    const int len = A.chunk_len[ch];
    typename Acc<T>::type acc[VPT];
#pragma unroll
    for (int q = 0; q < VPT; q++) acc[q] = 0;
    if (i >= 0 && p.has_shift) {
#pragma unroll
      for (int q = 0; q < VPT; q++) {
        const int c = s * VPT + q;
        acc[q] = p.sh[c] * x[i * p.ldx + c];
      }
    }
    const T* vv = vs + slot * ST_KMAX * ST_C;
    const T* xb = xs + buf * SM::xbuf;
#pragma unroll
    for (int k = 0; k < ST_KMAX; k++) {
      if (k < len) {
        const T a = vv[k * ST_C + l];
        const T* xr = xb + (size_t)(k * ST_C + l) * XP + s * VPT;
#pragma unroll
        for (int u = 0; u < NL; u++) {
          T xv[LW];
          Vec<T, LW>::ld_plain(xr + u * LW, xv);
#pragma unroll
          for (int w = 0; w < LW; w++) acc[u * LW + w] += a * xv[w];
        }
      }
    }
    if (i >= 0) {
      T* yr = p.y + p.col0 + i * p.ldy + s * VPT;
#pragma unroll
      for (int u = 0; u < NL; u++) {
        T yv[LW];
        if (p.beta != T(0)) {
          Vec<T, LW>::ld_plain(yr + u * LW, yv);
#pragma unroll
          for (int w = 0; w < LW; w++) yv[w] = p.alpha * acc[u * LW + w] + p.beta * yv[w];
        } else {
#pragma unroll
          for (int w = 0; w < LW; w++) yv[w] = p.alpha * acc[u * LW + w];
        }
        Vec<T, LW>::st(yr + u * LW, yv);
      }
    }
    __syncthreads();  // buffers of this chunk may be refilled next
  }
  cp_async_wait<0>();
}

}  // namespace pb
