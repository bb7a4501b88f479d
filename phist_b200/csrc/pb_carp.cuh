// pb_carp.cuh -- CARP: Kaczmarz forward/backward sweeps on (A - sigma_j I)
// (carp_setup/carp_sweep/carp_destroy, phist_kernels_carp_decl.h:35-106).
//
// The builtin sweep is row-sequential (kacz_loop_seq_def.h) or runs over the
// rows of a distance-2 colouring (kacz_loop_clr_def.h).  On the GPU every
// colour class is one launch: rows of one colour share no column, so their
// projections touch disjoint entries of X and may run concurrently; the
// result equals the sequential sweep over the rows in colour order.  The
// update formulae are those of kacz_sub_def.h:50-150:
//   tmp_j  = sum_k a_ik x_kj - sigma_j x_ij - b_ij
//   rn_j   = sum_k a_ik^2 - 2 a_ii sigma_j + sigma_j^2   (1 if zero)
//   tmp_j *= omega_j / rn_j
//   x_ij  += tmp_j sigma_j ;  x_kj -= tmp_j a_ik  for every entry k of row i
// The matrix is stored once more in colour order (CRS), so the rows of one
// launch are contiguous and their entries are read with coalesced loads.
//
// Block-coloured sweep (k_kacz_blocks, the default): a row colouring makes
// every colour launch touch rows of X all over the vector, so X is streamed
// once per colour.  Instead the rows are grouped into compact blocks whose
// footprints (columns of X they touch) are staged in shared memory, and the
// blocks are coloured (pb_carp_blocks.hpp); one launch per block colour, one
// thread block per row block.
#pragma once
#include <algorithm>

#include "pb_carp_blocks.hpp"
#include "pb_core.hpp"
#include "pb_tile.cuh"

namespace pb {

template <class T>
struct CarpWork {
  int nshifts = 0;
  std::vector<T> sigma_r, sigma_i;
  // sequential row order of the sweep and its distance-2 independent segments
  int ncolors = 0;
  std::vector<int64_t> h_color_ptr;
  std::vector<int32_t> h_rows;
  int64_t nrows = 0;
  // row-colour layout (blocks == false)
  int32_t* d_rows = nullptr;         // colour order -> original row
  int64_t* d_rp = nullptr;           // CRS in colour order
  int32_t* d_col = nullptr;
  T* d_val = nullptr;
  T* d_nrm = nullptr;                // sum_k a_ik^2 per colour-ordered row
  T* d_diag = nullptr;               // a_ii per colour-ordered row
  // block-coloured layout (blocks == true)
  bool blocks = false;
  int nbcolors = 0;
  std::vector<int64_t> h_bcolor_ptr;  // blocks [bcolor_ptr[c], bcolor_ptr[c+1]) have colour c
  int max_fp = 0, max_rows = 0, max_nnz = 0;
  CarpBlockDesc* d_desc = nullptr;
  int32_t* d_bfp = nullptr;
  T* d_bval = nullptr;
  uint16_t* d_blcol = nullptr;
  uint16_t* d_blrp = nullptr;
  T* d_bnd = nullptr;
  uint16_t* d_bstep = nullptr;
};

template <class T>
struct KaczArgs {
  const int32_t* __restrict__ rows;
  const int64_t* __restrict__ rp;
  const int32_t* __restrict__ col;
  const T* __restrict__ val;
  const T* __restrict__ nrm;
  const T* __restrict__ diag;
  int64_t q0, q1;       // colour-ordered row range of this launch
  int nvec;
  T sig_r[32];
  T sig_i[32];
  T omega[32];
  const T* b; int64_t ldb;   // may be nullptr (b = 0)
  T* xr; int64_t ldxr;
  T* xi; int64_t ldxi;       // rc variant only
};

// One thread per (row, column): TPR consecutive threads (TPR >= nvec, a power
// of two) share a row, thread j owns column j.  Within a colour class the
// (row, column) projections are independent of each other (distance-2
// colouring, and columns never mix), so no thread waits for another; the
// TPR threads of a row read and write each X row as one contiguous segment.
template <class T, int TPR, bool RC>
__global__ void __launch_bounds__(256) k_kacz_color_cols(KaczArgs<T> a)
{
  const int64_t q = a.q0 + (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) / TPR;
  const int j = threadIdx.x % TPR;
  if (q >= a.q1 || j >= a.nvec) return;
  const int64_t i = a.rows[q];
  const int64_t p0 = a.rp[q], p1 = a.rp[q + 1];
  const T sr = a.sig_r[j];
  const T si = RC ? a.sig_i[j] : T(0);
  T tr, ti = T(0);
  {
    const T xr = a.xr[i * a.ldxr + j];
    if (RC) {
      const T xi = a.xi[i * a.ldxi + j];
      tr = -sr * xr + si * xi;
      ti = -si * xr - sr * xi;
    } else {
      tr = -sr * xr;
    }
  }
#pragma unroll 4
  for (int64_t p = p0; p < p1; p++) {
    const T v = a.val[p];
    const int64_t c = a.col[p];
    tr += v * a.xr[c * a.ldxr + j];
    if (RC) ti += v * a.xi[c * a.ldxi + j];
  }
  if (a.b) tr -= a.b[i * a.ldb + j];
  const T nrm = a.nrm[q], d = a.diag[q];
  T rn = nrm - T(2) * d * sr + sr * sr;
  if (RC) rn += si * si;
  if (rn == T(0)) rn = T(1);
  const T f = a.omega[j] / rn;
  tr *= f;
  if (RC) {
    ti *= f;
    a.xr[i * a.ldxr + j] += tr * sr + ti * si;
    a.xi[i * a.ldxi + j] += ti * sr - tr * si;
  } else {
    a.xr[i * a.ldxr + j] += tr * sr;
  }
#pragma unroll 4
  for (int64_t p = p0; p < p1; p++) {
    const T v = a.val[p];
    const int64_t c = a.col[p];
    a.xr[c * a.ldxr + j] -= tr * v;
    if (RC) a.xi[c * a.ldxi + j] -= ti * v;
  }
}

template <class T>
struct KaczBlockArgs {
  const CarpBlockDesc* __restrict__ desc;
  const int32_t* __restrict__ fp;
  const T* __restrict__ val;
  const uint16_t* __restrict__ lcol;
  const uint16_t* __restrict__ lrp;
  const T* __restrict__ nd;
  const uint16_t* __restrict__ step;
  int64_t blk0;   // first block of this launch; thread block k takes block blk0 + k
  int dir;        // 1 forward, 2 backward, 3 forward then backward
  int nvec;
  int max_fp, max_rows, max_nnz;
  T sig_r[32];
  T sig_i[32];
  T omega[32];
  const T* b; int64_t ldb;   // may be nullptr (b = 0)
  T* xr; int64_t ldxr;
  T* xi; int64_t ldxi;       // rc variant only
};

constexpr int KB_NT = 256;

template <class T>
__device__ __forceinline__ void cp_async_elem(T* s, const T* g)
{
  const unsigned sa = (unsigned)__cvta_generic_to_shared(s);
  if constexpr (sizeof(T) == 8)
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(sa), "l"(g) : "memory");
  else
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4;\n" ::"r"(sa), "l"(g) : "memory");
}

// One thread block per row block.  (1) cp.async the block's segments (matrix
// entries with footprint-local columns, entry offsets, norms and diagonals,
// footprint rows, step starts), the footprint rows of X and the rows of B
// into shared memory; (2) run the steps, forward and/or backward: in a step
// thread (r, j), TPR threads per row, projects row r of the step for column
// j with the update formulae above, all in shared memory, the rows of one
// step touching disjoint footprint slots; a barrier separates the steps;
// (3) write the footprint rows of X back.  Blocks of one launch have
// disjoint footprints.
template <class T, int TPR, bool RC>
__global__ void __launch_bounds__(KB_NT) k_kacz_blocks(KaczBlockArgs<T> a)
{
  extern __shared__ __align__(16) unsigned char smem[];
  const CarpSmem L = carp_smem_layout(a.max_fp, a.max_rows, a.max_nnz, TPR, (int)sizeof(T), RC, a.b != nullptr);
  T* xs = (T*)(smem + L.xs);
  T* xis = (T*)(smem + L.xis);
  T* bs = (T*)(smem + L.bs);
  T* vs = (T*)(smem + L.val);
  T* nds = (T*)(smem + L.nd);
  int32_t* fps = (int32_t*)(smem + L.fp);
  uint16_t* lcs = (uint16_t*)(smem + L.lcol);
  uint16_t* lrs = (uint16_t*)(smem + L.lrp);
  uint16_t* sts = (uint16_t*)(smem + L.step);
  const int tid = threadIdx.x;
  const int nv = a.nvec;
  const CarpBlockDesc d = a.desc[a.blk0 + blockIdx.x];
  {
    // 16-byte chunks of the block's segments
    const int nval = carp_r8(d.nnz) * (int)sizeof(T) / 16;
    const int nlc = carp_r8(d.nnz) * 2 / 16;
    const int nlr = carp_r8(d.nrows + 1) * 2 / 16;
    const int nnd = carp_r8(d.nrows) * 2 * (int)sizeof(T) / 16;
    const int nfp = ((d.nfp + 3) & ~3) * 4 / 16;
    const int nst = carp_r8(d.nsteps + 1) * 2 / 16;
    const int tot = nval + nlc + nlr + nnd + nfp + nst;
    for (int c = tid; c < tot; c += KB_NT) {
      int k = c;
      const char* g;
      char* sp;
      if (k < nval) {
        g = (const char*)(a.val + d.ent);
        sp = (char*)vs;
      } else if ((k -= nval) < nlc) {
        g = (const char*)(a.lcol + d.ent);
        sp = (char*)lcs;
      } else if ((k -= nlc) < nlr) {
        g = (const char*)(a.lrp + d.row);
        sp = (char*)lrs;
      } else if ((k -= nlr) < nnd) {
        g = (const char*)(a.nd + 2 * d.row);
        sp = (char*)nds;
      } else if ((k -= nnd) < nfp) {
        g = (const char*)(a.fp + d.fp);
        sp = (char*)fps;
      } else {
        k -= nfp;
        g = (const char*)(a.step + d.step);
        sp = (char*)sts;
      }
      cp_async16(sp + 16 * k, g + 16 * k, true);
    }
    // footprint rows of X (own rows first) and the block's rows of B
    for (int e = tid; e < d.nfp * TPR; e += KB_NT) {
      const int u = e / TPR, j = e % TPR;
      if (j < nv) {
        const int64_t g = a.fp[d.fp + u];
        cp_async_elem(xs + e, a.xr + g * a.ldxr + j);
        if (RC) cp_async_elem(xis + e, a.xi + g * a.ldxi + j);
      }
    }
    if (a.b) {
      for (int e = tid; e < d.nrows * TPR; e += KB_NT) {
        const int r = e / TPR, j = e % TPR;
        if (j < nv) cp_async_elem(bs + e, a.b + (int64_t)a.fp[d.fp + r] * a.ldb + j);
      }
    }
    cp_async_commit();
    cp_async_wait<0>();
    __syncthreads();
  }
  auto project = [&](int r, int j) {
    const T sr = a.sig_r[j];
    const T si = RC ? a.sig_i[j] : T(0);
    const int e0 = lrs[r], e1 = lrs[r + 1];
    T tr, ti = T(0);
    {
      const T x0 = xs[r * TPR + j];
      if (RC) {
        const T y0 = xis[r * TPR + j];
        tr = -sr * x0 + si * y0;
        ti = -si * x0 - sr * y0;
      } else {
        tr = -sr * x0;
      }
    }
    for (int p = e0; p < e1; p++) {
      const T v = vs[p];
      const int c = lcs[p];
      tr += v * xs[c * TPR + j];
      if (RC) ti += v * xis[c * TPR + j];
    }
    if (a.b) tr -= bs[r * TPR + j];
    const T nrm = nds[2 * r], dg = nds[2 * r + 1];
    T rn = nrm - T(2) * dg * sr + sr * sr;
    if (RC) rn += si * si;
    if (rn == T(0)) rn = T(1);
    const T f = a.omega[j] / rn;
    tr *= f;
    if (RC) {
      ti *= f;
      xs[r * TPR + j] += tr * sr + ti * si;
      xis[r * TPR + j] += ti * sr - tr * si;
    } else {
      xs[r * TPR + j] += tr * sr;
    }
    for (int p = e0; p < e1; p++) {
      const T v = vs[p];
      const int c = lcs[p];
      xs[c * TPR + j] -= tr * v;
      if (RC) xis[c * TPR + j] -= ti * v;
    }
  };
  auto run_step = [&](int s) {
    const int lo = sts[s], hi = sts[s + 1];
    for (int e = tid; e < (hi - lo) * TPR; e += KB_NT) {
      const int j = e % TPR;
      if (j < nv) project(lo + e / TPR, j);
    }
    __syncthreads();
  };
  if (a.dir & 1)
    for (int s = 0; s < d.nsteps; s++) run_step(s);
  if (a.dir & 2)
    for (int s = d.nsteps - 1; s >= 0; s--) run_step(s);
  for (int e = tid; e < d.nfp * TPR; e += KB_NT) {
    const int u = e / TPR, j = e % TPR;
    if (j < nv) {
      const int64_t g = fps[u];
      a.xr[g * a.ldxr + j] = xs[e];
      if (RC) a.xi[g * a.ldxi + j] = xis[e];
    }
  }
}

// Distance-2 colouring: row i takes the smallest colour not used by any row
// that shares a column with it (greedy in a given row order), first in
// natural order, then a few rounds of iterated greedy (rows visited colour
// class by colour class, classes in reverse order; such a pass never needs
// more colours than the colouring it starts from, and often fewer).  Fewer
// colours mean fewer sweep launches and fewer passes over the vector block.
// colT is the column -> rows pattern (transpose).
inline int dist2_greedy(int64_t n, const std::vector<int64_t>& rp, const std::vector<int32_t>& col,
                        const std::vector<int64_t>& tp, const std::vector<int32_t>& trow,
                        const std::vector<int32_t>& order, std::vector<int32_t>& color)
{
  color.assign(n, -1);
  std::vector<int64_t> mark;  // mark[c] == i: colour c forbidden for row i
  int ncolor = 0;
  for (int64_t k = 0; k < n; k++) {
    const int64_t i = order.empty() ? k : order[k];
    for (int64_t p = rp[i]; p < rp[i + 1]; p++) {
      const int32_t c = col[p];
      for (int64_t t = tp[c]; t < tp[c + 1]; t++) {
        const int32_t r = trow[t];
        const int32_t cr = color[r];
        if (r != i && cr >= 0) {
          if ((int)mark.size() <= cr) mark.resize(cr + 1, -1);
          mark[cr] = i;
        }
      }
    }
    int c = 0;
    while (c < (int)mark.size() && mark[c] == i) c++;
    color[i] = c;
    if (c + 1 > ncolor) ncolor = c + 1;
  }
  return ncolor;
}

inline int dist2_color(int64_t n, int64_t ncols, const std::vector<int64_t>& rp,
                       const std::vector<int32_t>& col, std::vector<int32_t>& color, int rounds = 8)
{
  std::vector<int64_t> tp(ncols + 1, 0);
  for (int64_t p = 0; p < rp[n]; p++) tp[col[p] + 1]++;
  for (int64_t j = 0; j < ncols; j++) tp[j + 1] += tp[j];
  std::vector<int32_t> trow(rp[n]);
  {
    std::vector<int64_t> fill(tp.begin(), tp.end() - 1);
    for (int64_t i = 0; i < n; i++)
      for (int64_t p = rp[i]; p < rp[i + 1]; p++) trow[fill[col[p]]++] = (int32_t)i;
  }
  int ncolor = dist2_greedy(n, rp, col, tp, trow, std::vector<int32_t>(), color);
  std::vector<int32_t> cur(color), order(n), cand;
  int ncur = ncolor;
  for (int r = 0; r < rounds && ncur > 1; r++) {
    // visit the rows class by class (ascending inside a class): even rounds
    // in reverse class order, odd rounds largest class first
    std::vector<int64_t> size(ncur, 0);
    for (int64_t i = 0; i < n; i++) size[cur[i]]++;
    std::vector<int> cls(ncur);
    for (int c = 0; c < ncur; c++) cls[c] = ncur - 1 - c;
    if (r % 2) std::stable_sort(cls.begin(), cls.end(), [&](int a, int b) { return size[a] > size[b]; });
    std::vector<int> rank(ncur);
    for (int k = 0; k < ncur; k++) rank[cls[k]] = k;
    std::vector<int64_t> start(ncur + 1, 0);
    for (int64_t i = 0; i < n; i++) start[rank[cur[i]] + 1]++;
    for (int c = 0; c < ncur; c++) start[c + 1] += start[c];
    for (int64_t i = 0; i < n; i++) order[start[rank[cur[i]]]++] = (int32_t)i;
    ncur = dist2_greedy(n, rp, col, tp, trow, order, cand);
    cur.swap(cand);
    if (ncur < ncolor) {
      ncolor = ncur;
      color = cur;
    }
  }
  return ncolor;
}

}  // namespace pb
