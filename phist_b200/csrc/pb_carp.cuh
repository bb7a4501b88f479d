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
  int max_fp = 0, max_rows = 0, seg_stride = 0;
  bool distinct = false;               // no row holds a column twice
  unsigned char* d_bseg = nullptr;     // block segments, seg_stride bytes apart
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
  const unsigned char* __restrict__ seg;   // segment b at b * seg_stride
  int64_t blk0;          // first block of the launch; thread block k takes block blk0 + k
  int dir;              // 1 forward, 2 backward, 3 forward then backward
  int nvec;
  int max_fp, max_rows, seg_stride;
  int distinct;         // no row holds a column twice
  T sig_r[32];
  T sig_i[32];
  T omega[32];
  const T* b; int64_t ldb;   // may be nullptr (b = 0)
  T* xr; int64_t ldxr;
  T* xi; int64_t ldxi;       // rc variant only
};

constexpr int KB_NT = 128;  // threads per block of the block sweep

// cp.async of BYTES (4, 8 or 16) from global to shared memory
template <int BYTES>
__device__ __forceinline__ void cp_async_n(void* s, const void* g)
{
  const unsigned sa = (unsigned)__cvta_generic_to_shared(s);
  if constexpr (BYTES == 16)
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(sa), "l"(g) : "memory");
  else
    asm volatile("cp.async.ca.shared.global [%0], [%1], %2;\n" ::"r"(sa), "l"(g), "n"(BYTES) : "memory");
}

// CPT consecutive elements of T (CPT * sizeof(T) <= 16, aligned)
template <class T, int CPT>
struct CarpVec {
  T v[CPT];
};
template <class T, int CPT>
__device__ __forceinline__ CarpVec<T, CPT> cv_ld(const T* p)
{
  CarpVec<T, CPT> r;
  if constexpr (CPT * sizeof(T) == 16) {
    const double2 q = *(const double2*)p;
    memcpy(&r, &q, 16);
  } else if constexpr (CPT * sizeof(T) == 8) {
    const double q = *(const double*)p;
    memcpy(&r, &q, 8);
  } else {
    r.v[0] = p[0];
  }
  return r;
}
template <class T, int CPT>
__device__ __forceinline__ void cv_st(T* p, const CarpVec<T, CPT>& r)
{
  if constexpr (CPT * sizeof(T) == 16) {
    double2 q;
    memcpy(&q, &r, 16);
    *(double2*)p = q;
  } else if constexpr (CPT * sizeof(T) == 8) {
    double q;
    memcpy(&q, &r, 8);
    *(double*)p = q;
  } else {
    p[0] = r.v[0];
  }
}

// One thread block per row block of one colour (blocks blk0 + blockIdx.x;
// the blocks of a launch have disjoint footprints).  Two copy stages
// precede the steps:
//   H: cp.async the head of the block's segment (header, footprint rows)
//   X: cp.async the rest of the segment (entries with footprint-local
//      columns, norms and diagonals, entry offsets, step starts), the
//      footprint rows of X and the block's rows of B
// then the steps, forward and/or backward, and X written back.  Many
// thread blocks per SM overlap one another's copies and steps.
//
// X rows are copied in pieces of W elements (16 bytes when the caller's
// alignment allows, else one element).  In a step, thread (r, q) projects
// row r of the step for the CPT columns q*CPT.. (TPR/CPT threads per row):
// the row's entries are read once for its CPT columns and X is read and
// written CPT columns at a time; each column follows the update formulae
// above in the same order.  Rows of one step touch disjoint footprint slots
// and a barrier separates the steps.
template <class T, int TPR, bool RC, int NT, int W>
__global__ void __launch_bounds__(NT) k_kacz_blocks(KaczBlockArgs<T> a)
{
  constexpr int CPT = (TPR >= 16 / (int)sizeof(T)) ? 16 / (int)sizeof(T) : TPR;  // columns per thread
  constexpr int TPRC = TPR / CPT;                                                  // threads per row
  constexpr int RE = 4;  // row length of the register path
  static_assert(NT % TPRC == 0, "a thread keeps its columns in every step");
  using V = CarpVec<T, CPT>;
  extern __shared__ __align__(16) unsigned char smem[];
  const CarpSmem L = carp_smem_layout(a.max_fp, a.max_rows, a.seg_stride, TPR, (int)sizeof(T), RC, a.b != nullptr);
  const int head = carp_seg_head(a.max_fp);
  const int tid = threadIdx.x;
  const int nv = a.nvec;
  unsigned char* mb = smem + L.mbase;   // the block's segment
  unsigned char* xb = smem + L.xbase;   // its X and B rows
  const unsigned char* gseg = a.seg + (a.blk0 + blockIdx.x) * a.seg_stride;

  // the next launch may start its thread blocks as this one's finish: they
  // copy their segments (read-only) and then wait for this grid to complete
  // before they touch X or B (griddepcontrol.wait below; both are no-ops
  // without a programmatic dependency)
  asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
  // H: header and footprint rows
  for (int c = tid; c < head / 16; c += NT) cp_async_n<16>(mb + 16 * c, gseg + 16 * c);
  cp_async_commit();
  cp_async_wait<0>();
  __syncthreads();
  // X: the rest of the segment, footprint rows of X (own rows first), rows
  // of B
  {
    const int32_t* hdr = (const int32_t*)mb;
    const int nrows = hdr[0], nfp = hdr[1];
    const int bytes = carp_seg(hdr[0], hdr[1], hdr[2], hdr[3], (int)sizeof(T)).bytes;
    for (int c = head / 16 + tid; c < bytes / 16; c += NT) cp_async_n<16>(mb + 16 * c, gseg + 16 * c);
    asm volatile("griddepcontrol.wait;" ::: "memory");
    const int32_t* fps = (const int32_t*)(mb + 16);
    T* xs = (T*)(xb + L.xs);
    T* xis = (T*)(xb + L.xis);
    T* bs = (T*)(xb + L.bs);
    constexpr int PW = TPR / W;  // pieces per footprint row
    for (int e = tid; e < nfp * PW; e += NT) {
      const int u = e / PW, j = (e % PW) * W;
      if (j < nv) {
        const int64_t g = fps[u];
        cp_async_n<W * sizeof(T)>(xs + u * TPR + j, a.xr + g * a.ldxr + j);
        if (RC) cp_async_n<W * sizeof(T)>(xis + u * TPR + j, a.xi + g * a.ldxi + j);
      }
    }
    if (a.b) {
      for (int e = tid; e < nrows * PW; e += NT) {
        const int r = e / PW, j = (e % PW) * W;
        if (j < nv) cp_async_n<W * sizeof(T)>(bs + r * TPR + j, a.b + (int64_t)fps[r] * a.ldb + j);
      }
    }
    cp_async_commit();
    cp_async_wait<0>();
    __syncthreads();
  }

  // the steps and the write-back
  {
    const int32_t* hdr = (const int32_t*)mb;
    const CarpSeg sg = carp_seg(hdr[0], hdr[1], hdr[2], hdr[3], (int)sizeof(T));
    const int32_t* fps = (const int32_t*)(mb + sg.fp);
    const T* vs = (const T*)(mb + sg.val);
    const T* nds = (const T*)(mb + sg.nd);
    const uint16_t* lcs = (const uint16_t*)(mb + sg.lcol);
    const uint16_t* lrs = (const uint16_t*)(mb + sg.lrp);
    const uint16_t* sts = (const uint16_t*)(mb + sg.step);
    T* xs = (T*)(xb + L.xs);
    T* xis = (T*)(xb + L.xis);
    const T* bs = (const T*)(xb + L.bs);

    // this thread's columns: thread e of a step takes row e / TPRC and the
    // CPT columns from (e % TPRC) * CPT; NT is a multiple of TPRC, so a
    // thread keeps its columns, shifts and relaxation in every step
    const int j0 = (tid % TPRC) * CPT;
    T sr[CPT], si[CPT], om[CPT];
#pragma unroll
    for (int k = 0; k < CPT; k++) {
      sr[k] = a.sig_r[j0 + k];
      si[k] = RC ? a.sig_i[j0 + k] : T(0);
      om[k] = a.omega[j0 + k];
    }
    auto project = [&](int r) {
      const int e0 = lrs[r], e1 = lrs[r + 1];
      const T nrm = nds[2 * r], dg = nds[2 * r + 1];
      // the scaling does not depend on X: formed while the gathers are out
      T f[CPT];
#pragma unroll
      for (int k = 0; k < CPT; k++) {
        T rn = nrm - T(2) * dg * sr[k] + sr[k] * sr[k];
        if (RC) rn += si[k] * si[k];
        if (rn == T(0)) rn = T(1);
        f[k] = om[k] / rn;
      }
      T tr[CPT], ti[CPT];
      const V x0 = cv_ld<T, CPT>(xs + r * TPR + j0);
      V y0;
      if (RC) y0 = cv_ld<T, CPT>(xis + r * TPR + j0);
#pragma unroll
      for (int k = 0; k < CPT; k++) {
        if (RC) {
          tr[k] = -sr[k] * x0.v[k] + si[k] * y0.v[k];
          ti[k] = -si[k] * x0.v[k] - sr[k] * y0.v[k];
        } else {
          tr[k] = -sr[k] * x0.v[k];
          ti[k] = T(0);
        }
      }
      if (!RC && a.distinct && e1 - e0 == RE) {
        // RE distinct columns (every row of the honeycomb matrices): the
        // entries and gathered values stay in registers; x_i first takes the
        // shift term, then every entry in order (the diagonal one
        // continuing from x_i), and each slot is stored once -- no other
        // thread of the step touches these slots
        T v[RE];
        int c[RE];
        V xg[RE];
#pragma unroll
        for (int q = 0; q < RE; q++) {
          v[q] = vs[e0 + q];
          c[q] = lcs[e0 + q];
        }
#pragma unroll
        for (int q = 0; q < RE; q++) xg[q] = cv_ld<T, CPT>(xs + c[q] * TPR + j0);
#pragma unroll
        for (int q = 0; q < RE; q++)
#pragma unroll
          for (int k = 0; k < CPT; k++) tr[k] += v[q] * xg[q].v[k];
        if (a.b) {
          const V bb = cv_ld<T, CPT>(bs + r * TPR + j0);
#pragma unroll
          for (int k = 0; k < CPT; k++) tr[k] -= bb.v[k];
        }
        V xo = x0;
#pragma unroll
        for (int k = 0; k < CPT; k++) {
          tr[k] *= f[k];
          xo.v[k] += tr[k] * sr[k];
        }
#pragma unroll
        for (int q = 0; q < RE; q++) {
          const bool own = c[q] == r;
          V t = own ? xo : xg[q];
#pragma unroll
          for (int k = 0; k < CPT; k++) t.v[k] -= tr[k] * v[q];
          if (own) xo = t;
          else cv_st<T, CPT>(xs + c[q] * TPR + j0, t);
        }
        cv_st<T, CPT>(xs + r * TPR + j0, xo);
        return;
      }
      // any row: entries read from shared memory, every slot updated in place
      for (int p = e0; p < e1; p++) {
        const T vv = vs[p];
        const int cc = lcs[p];
        const V xx = cv_ld<T, CPT>(xs + cc * TPR + j0);
        V yy;
        if (RC) yy = cv_ld<T, CPT>(xis + cc * TPR + j0);
#pragma unroll
        for (int k = 0; k < CPT; k++) {
          tr[k] += vv * xx.v[k];
          if (RC) ti[k] += vv * yy.v[k];
        }
      }
      if (a.b) {
        const V bb = cv_ld<T, CPT>(bs + r * TPR + j0);
#pragma unroll
        for (int k = 0; k < CPT; k++) tr[k] -= bb.v[k];
      }
#pragma unroll
      for (int k = 0; k < CPT; k++) {
        tr[k] *= f[k];
        if (RC) ti[k] *= f[k];
      }
      {
        // x_i was not written since it was read above
        V xo = x0;
        if (RC) {
          V yo = y0;
#pragma unroll
          for (int k = 0; k < CPT; k++) {
            xo.v[k] += tr[k] * sr[k] + ti[k] * si[k];
            yo.v[k] += ti[k] * sr[k] - tr[k] * si[k];
          }
          cv_st<T, CPT>(xis + r * TPR + j0, yo);
        } else {
#pragma unroll
          for (int k = 0; k < CPT; k++) xo.v[k] += tr[k] * sr[k];
        }
        cv_st<T, CPT>(xs + r * TPR + j0, xo);
      }
      for (int p = e0; p < e1; p++) {
        const T vv = vs[p];
        const int cc = lcs[p];
        V xx = cv_ld<T, CPT>(xs + cc * TPR + j0);
#pragma unroll
        for (int k = 0; k < CPT; k++) xx.v[k] -= tr[k] * vv;
        cv_st<T, CPT>(xs + cc * TPR + j0, xx);
        if (RC) {
          V yy = cv_ld<T, CPT>(xis + cc * TPR + j0);
#pragma unroll
          for (int k = 0; k < CPT; k++) yy.v[k] -= ti[k] * vv;
          cv_st<T, CPT>(xis + cc * TPR + j0, yy);
        }
      }
    };
    auto run_step = [&](int st) {
      const int lo = sts[st], hi = sts[st + 1];
      if (j0 < nv)
        for (int e = tid; e < (hi - lo) * TPRC; e += NT) project(lo + e / TPRC);
      __syncthreads();
    };
    if (a.dir & 1)
      for (int st = 0; st < sg.nsteps; st++) run_step(st);
    if (a.dir & 2)
      for (int st = sg.nsteps - 1; st >= 0; st--) run_step(st);
    constexpr int PW = TPR / W;
    for (int e = tid; e < sg.nfp * PW; e += NT) {
      const int u = e / PW, j = (e % PW) * W;
      if (j < nv) {
        const int64_t g = fps[u];
        cv_st<T, W>(a.xr + g * a.ldxr + j, cv_ld<T, W>(xs + u * TPR + j));
        if (RC) cv_st<T, W>(a.xi + g * a.ldxi + j, cv_ld<T, W>(xis + u * TPR + j));
      }
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
