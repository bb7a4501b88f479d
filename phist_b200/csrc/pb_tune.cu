// pb_tune.cu -- autotuner for the SpMMV of one matrix.
//
// The SELL-C-sigma layout (chunk height C, sorting window sigma) and the
// SpMMV kernel variant per block width (threads per row, the fully unrolled
// short-row kernel, the shared-memory staged kernel for wide blocks) are
// chosen by timing Y = A X on the matrix itself, on the device, with CUDA
// events on the calling thread's stream and the L2 cache flushed before
// every timed call.  GHOST, the library PHIST uses for SELL-C-sigma, fixes
// C = 32 on CUDA and sigma by flag (src/kernels/ghost/kernels.cpp:69-134);
// here they are measured.  Every layout and variant computes the same bits:
// each row sums its entries in column order, and the permutation is internal
// to the matrix (vectors keep the original row order).
#include <algorithm>
#include <cmath>
#include <vector>

#include "pb_api.cuh"

namespace pb {
namespace {

struct SpmvVariant {
  int tpr, unroll, staged;
};

// width class of a block width: 1, 2, 4, 8, 16, 32 -> 0..5
int width_class(int w) { return w <= 1 ? 0 : w <= 2 ? 1 : w <= 4 ? 2 : w <= 8 ? 3 : w <= 16 ? 4 : 5; }

// the variants spmv_tile/launch_spmv_nv instantiate for one width class
std::vector<SpmvVariant> spmv_variants(int lg, bool short_rows)
{
  static const int tprs[6][3] = {{1, 0, 0}, {1, 0, 0}, {1, 2, 0}, {1, 2, 4}, {2, 4, 8}, {4, 8, 16}};
  std::vector<SpmvVariant> v;
  for (int t = 0; t < 3; t++) {
    const int tpr = tprs[lg][t];
    if (tpr == 0) continue;
    for (int unroll = 1; unroll >= 0; unroll--) {
      if (!short_rows && unroll == 0) continue;  // without short rows both are the general kernel
      const bool can_stage = short_rows && unroll && lg >= 3;
      for (int staged = 0; staged <= (can_stage ? 1 : 0); staged++) {
        // the staged kernel does not depend on tpr: try it with one tpr only
        if (staged && t > 0) continue;
        v.push_back({tpr, short_rows ? unroll : 1, staged});
      }
    }
  }
  return v;
}

template <class T>
void raw_block(Mvec<T>& m, T* d, int64_t n, int w)
{
  m.map = nullptr;
  m.nrows = (int32_t)n;
  m.nvec = w;
  m.lda = w;
  m.root = &m;
  m.col_off = 0;
  m.d_base = d;
  m.h_base = nullptr;
}

struct Timing {
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  void* flush = nullptr;
  size_t flush_bytes = 0;
  Timing()
  {
    PB_CUDA(cudaEventCreate(&e0));
    PB_CUDA(cudaEventCreate(&e1));
    flush_bytes = (size_t)(2 * rt().l2_bytes());
    flush = rt().dmalloc(flush_bytes);
  }
  ~Timing()
  {
    if (e0) cudaEventDestroy(e0);
    if (e1) cudaEventDestroy(e1);
    rt().dfree(flush);
  }
};

// median device time of reps calls of Y = A X, in microseconds
template <class T>
double time_spmv(const SparseMat<T>* A, const Mvec<T>* X, Mvec<T>* Y, int reps, Timing& tm)
{
  spmv_general<T>(T(1), A, nullptr, X, T(0), Y, nullptr, nullptr, T(0), T(0), nullptr);  // warm-up
  std::vector<float> ts;
  for (int r = 0; r < reps; r++) {
    PB_CUDA(cudaMemsetAsync(tm.flush, r & 0xff, tm.flush_bytes, stream()));
    PB_CUDA(cudaEventRecord(tm.e0, stream()));
    spmv_general<T>(T(1), A, nullptr, X, T(0), Y, nullptr, nullptr, T(0), T(0), nullptr);
    PB_CUDA(cudaEventRecord(tm.e1, stream()));
    PB_CUDA(cudaEventSynchronize(tm.e1));
    float ms = 0.0f;
    PB_CUDA(cudaEventElapsedTime(&ms, tm.e0, tm.e1));
    ts.push_back(ms);
  }
  std::sort(ts.begin(), ts.end());
  return 1e3 * (double)ts[ts.size() / 2];
}

struct Choice {
  int C = 32;
  int64_t sigma = 1;
  double total = INFINITY;
  SpmvVariant v[6] = {};
  bool set[6] = {};
  std::vector<double> per_width;
};

}  // namespace

// Candidate layouts: C in {32, 16, 8} x sigma in {1, 4C, 1024} (sigma = 1
// only when all rows have the same length, where sorting changes nothing).
// For each layout and each width class present in widths[], every kernel
// variant is timed on all requested widths of that class and the fastest sum
// is kept; the layout with the least total over the widths wins.  The
// matrix is left in the winning layout with the winning variant per class;
// best_us[i] is the time of widths[i] there.
template <class T>
void sparse_autotune(SparseMat<T>* A, int nw, const int* widths, int reps, double* best_us)
{
  PB_REQUIRE(A, PB_INVALID_INPUT, "matrix is NULL");
  PB_REQUIRE(nw >= 1 && nw <= 64 && widths, PB_INVALID_INPUT, "need 1..64 block widths");
  for (int i = 0; i < nw; i++)
    PB_REQUIRE(widths[i] >= 1 && widths[i] <= 32, PB_INVALID_INPUT, "block width %d not in 1..32", widths[i]);
  reps = std::max(1, std::min(reps, 1000));
  const int64_t nr = A->nrows, nc = A->ncols;
  bool uniform = true;
  for (int64_t i = 1; i < nr && uniform; i++)
    uniform = (A->h_row_ptr[i + 1] - A->h_row_ptr[i]) == (A->h_row_ptr[1] - A->h_row_ptr[0]);

  const int C0 = A->C;
  const int64_t S0 = A->sigma;
  int tpr0[6], unr0[6], stg0[6];
  std::copy(A->tune_tpr, A->tune_tpr + 6, tpr0);
  std::copy(A->tune_unroll, A->tune_unroll + 6, unr0);
  std::copy(A->tune_staged, A->tune_staged + 6, stg0);

  std::vector<std::pair<int, int64_t>> layouts;
  for (int C : {32, 16, 8}) {
    std::vector<int64_t> sig = {1};
    if (!uniform) {
      sig.push_back(4 * C);
      sig.push_back(1024);
    }
    for (int64_t s : sig) layouts.push_back({C, s});
  }
  int wmax = 1;
  for (int i = 0; i < nw; i++) wmax = std::max(wmax, widths[i]);

  Choice best;
  try {
    Timing tm;
    T* xd = (T*)rt().dmalloc(sizeof(T) * (size_t)std::max<int64_t>(nc, 1) * wmax);
    T* yd = (T*)rt().dmalloc(sizeof(T) * (size_t)std::max<int64_t>(nr, 1) * wmax);
    struct Free {
      void *a, *b;
      ~Free()
      {
        rt().dfree(a);
        rt().dfree(b);
      }
    } fr{xd, yd};
    for (const auto& L : layouts) {
      sell_layout(A, A->h_row_ptr, A->h_col, A->h_val, L.first, L.second);
      const bool short_rows = A->C == 32 && A->max_row_len <= 8;
      Choice cur;
      cur.C = L.first;
      cur.sigma = L.second;
      cur.total = 0.0;
      cur.per_width.assign(nw, 0.0);
      for (int lg = 0; lg < 6; lg++) {
        std::vector<int> members;
        for (int i = 0; i < nw; i++)
          if (width_class(widths[i]) == lg) members.push_back(i);
        if (members.empty()) continue;
        double best_sum = INFINITY;
        std::vector<double> best_t(members.size());
        for (const SpmvVariant& v : spmv_variants(lg, short_rows)) {
          A->tune_tpr[lg] = v.tpr;
          A->tune_unroll[lg] = v.unroll;
          A->tune_staged[lg] = v.staged;
          double sum = 0.0;
          std::vector<double> t(members.size());
          for (size_t k = 0; k < members.size(); k++) {
            const int w = widths[members[k]];
            Mvec<T> X, Y;
            raw_block(X, xd, nc, w);
            raw_block(Y, yd, nr, w);
            k_random<T><<<grid_for(nc * (int64_t)w), 256, 0, stream()>>>(xd, w, nc, w, w, 0, 12345);
            PB_LAUNCH_CHECK();
            t[k] = time_spmv<T>(A, &X, &Y, reps, tm);
            sum += t[k];
          }
          if (sum < best_sum) {
            best_sum = sum;
            best_t = t;
            cur.v[lg] = v;
            cur.set[lg] = true;
          }
        }
        for (size_t k = 0; k < members.size(); k++) cur.per_width[members[k]] = best_t[k];
        cur.total += best_sum;
      }
      if (cur.total < best.total) best = cur;
    }
    if (A->C != best.C || A->sigma != best.sigma)
      sell_layout(A, A->h_row_ptr, A->h_col, A->h_val, best.C, best.sigma);
    for (int lg = 0; lg < 6; lg++) {
      A->tune_tpr[lg] = best.set[lg] ? best.v[lg].tpr : tpr0[lg];
      A->tune_unroll[lg] = best.set[lg] ? best.v[lg].unroll : unr0[lg];
      A->tune_staged[lg] = best.set[lg] ? best.v[lg].staged : stg0[lg];
    }
  } catch (...) {
    // leave the matrix as it came
    std::copy(tpr0, tpr0 + 6, A->tune_tpr);
    std::copy(unr0, unr0 + 6, A->tune_unroll);
    std::copy(stg0, stg0 + 6, A->tune_staged);
    try {
      if (A->C != C0 || A->sigma != S0) sell_layout(A, A->h_row_ptr, A->h_col, A->h_val, C0, S0);
    } catch (...) {
    }
    throw;
  }
  if (best_us)
    for (int i = 0; i < nw; i++) best_us[i] = best.per_width[i];
}

template <class T>
void sparse_get_tuning(const SparseMat<T>* A, int* C, int64_t* sigma, int* tpr, int* unroll, int* staged)
{
  PB_REQUIRE(A, PB_INVALID_INPUT, "matrix is NULL");
  if (C) *C = A->C;
  if (sigma) *sigma = A->sigma;
  for (int lg = 0; lg < 6; lg++) {
    if (tpr) tpr[lg] = A->tune_tpr[lg] > 0 ? A->tune_tpr[lg] : rt().spmv_tpr[lg];
    if (unroll) unroll[lg] = A->tune_unroll[lg] >= 0 ? A->tune_unroll[lg] : (rt().spmv_unroll ? 1 : 0);
    if (staged)
      staged[lg] = A->tune_staged[lg] >= 0 ? A->tune_staged[lg]
                                           : ((lg >= 3 && (1 << lg) >= rt().spmv_staged_min_nvec) ? 1 : 0);
  }
}

}  // namespace pb

extern "C" {

void phist_b200_DsparseMat_autotune(void* A, int nw, const int* widths, int reps, double* best_us, int* iflag)
{
  PB_API_BEGIN(iflag);
  pb::sparse_autotune<double>(pb::SP<double>(A), nw, widths, reps, best_us);
  PB_API_END(iflag);
}

void phist_b200_SsparseMat_autotune(void* A, int nw, const int* widths, int reps, double* best_us, int* iflag)
{
  PB_API_BEGIN(iflag);
  pb::sparse_autotune<float>(pb::SP<float>(A), nw, widths, reps, best_us);
  PB_API_END(iflag);
}

void phist_b200_DsparseMat_get_tuning(const void* A, int* C, int64_t* sigma, int* tpr, int* unroll, int* staged,
                                      int* iflag)
{
  PB_API_BEGIN(iflag);
  pb::sparse_get_tuning<double>(pb::SP<double>(A), C, sigma, tpr, unroll, staged);
  PB_API_END(iflag);
}

void phist_b200_SsparseMat_get_tuning(const void* A, int* C, int64_t* sigma, int* tpr, int* unroll, int* staged,
                                      int* iflag)
{
  PB_API_BEGIN(iflag);
  pb::sparse_get_tuning<float>(pb::SP<float>(A), C, sigma, tpr, unroll, staged);
  PB_API_END(iflag);
}

}  // extern "C"
