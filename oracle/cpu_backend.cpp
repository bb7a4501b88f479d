// cpu_backend.cpp -- a CPU implementation of the part of PHIST's kernel API
// (phist_kernels_decl.h, phist_kernels_fused_decl.h, phist_kernels.h) that
// PHIST's FP64 solvers call (TEST INFRASTRUCTURE, never shipped).
//
// PHIST's builtin kernel library (Fortran 2008 + MPI, src/kernels/builtin/)
// cannot be built here.  This file restates it on the host so that PHIST's
// unchanged subspacejada, compiled from its sources, can run on the CPU cores:
// as the timed CPU baseline of the eigen-solves and as a solver-level check
// of the GPU library (same eigenvalues, iteration counts within 10 %).
// The data layout is the builtin's: CRS matrices with columns sorted inside
// each row (crsmat_module.F90:484-516), row-major block vectors with views
// that share the parent's storage and leading dimension
// (mvec_module.F90:98-106), column-major small matrices (sdmat_module.F90).
// Every loop is OpenMP-parallel over rows as in the builtin; reductions sum
// per-thread partials (the builtin's OpenMP reduction clauses).
//
// Only type D is provided.  Entry points that the FP64 eigen-solve never
// calls return PHIST_NOT_IMPLEMENTED (-99), as PHIST's own libraries do for
// what they lack.
#include <omp.h>

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

namespace {

constexpr int kNotImpl = -99, kInvalid = -55;

struct Map {
  int64_t n;
};
struct Mvec {
  const Map* map;
  int64_t n;
  int nvec;
  int64_t lda;
  double* v;   // element (i, j) at v[i*lda + j]
  bool owner;
};
struct Sd {
  int nr, nc;
  int64_t lda;
  double* v;   // element (i, j) at v[i + j*lda]
  bool owner;
};
struct Sp {
  int64_t n, m;
  std::vector<int64_t> rp;
  std::vector<int32_t> col;
  std::vector<double> val;
  Map* rmap;
  Map* dmap;
};

int g_comm_dummy = 0;

inline Mvec* MV(const void* p) { return (Mvec*)p; }
inline Sd* SD(const void* p) { return (Sd*)p; }
inline Sp* SP(const void* p) { return (Sp*)p; }
inline double& at(const Mvec* V, int64_t i, int j) { return V->v[i * V->lda + j]; }
inline double& at(const Sd* M, int i, int j) { return M->v[i + (int64_t)j * M->lda]; }

// per-thread partial sums of a k x m accumulation, combined in thread order
template <class F>
void reduce_rows(int64_t n, int nout, double* out, F body)
{
  const int nt = omp_get_max_threads();
  std::vector<double> part((size_t)nt * nout, 0.0);
#pragma omp parallel
  {
    double* mine = part.data() + (size_t)omp_get_thread_num() * nout;
#pragma omp for schedule(static)
    for (int64_t i = 0; i < n; i++) body(i, mine);
  }
  for (int o = 0; o < nout; o++) {
    double s = 0.0;
    for (int t = 0; t < nt; t++) s += part[(size_t)t * nout + o];
    out[o] = s;
  }
}

// SpMMV row loop of the builtin (spmvm_kernels.F90:494-523): tmp = shift*x_i,
// the row's entries in stored order, y = alpha*tmp + beta*y
void spmv(double alpha, const Sp* A, const double* sh, const Mvec* X, double beta, Mvec* Y)
{
  const int nv = X->nvec;
  if (alpha == 0.0 || A->rp[A->n] == 0) {
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < A->n; i++)
      for (int j = 0; j < nv; j++) at(Y, i, j) = beta * at(Y, i, j);
    return;
  }
#pragma omp parallel
  {
    std::vector<double> tmp(nv);
#pragma omp for schedule(static)
    for (int64_t i = 0; i < A->n; i++) {
      for (int j = 0; j < nv; j++) tmp[j] = (sh ? sh[j] : 0.0) * at(X, i, j);
      for (int64_t p = A->rp[i]; p < A->rp[i + 1]; p++) {
        const double a = A->val[p];
        const double* xr = X->v + (int64_t)A->col[p] * X->lda;
        for (int j = 0; j < nv; j++) tmp[j] += a * xr[j];
      }
      for (int j = 0; j < nv; j++)
        at(Y, i, j) = beta == 0.0 ? alpha * tmp[j] : alpha * tmp[j] + beta * at(Y, i, j);
    }
  }
}

// C = alpha V'W + beta C (mvec_module.F90:2421-2747)
void mvtmv(double alpha, const Mvec* V, const Mvec* W, double beta, Sd* C)
{
  const int m = V->nvec, k = W->nvec;
  std::vector<double> s((size_t)m * k);
  reduce_rows(V->n, m * k, s.data(), [&](int64_t i, double* acc) {
    const double* vr = V->v + i * V->lda;
    const double* wr = W->v + i * W->lda;
    for (int j = 0; j < k; j++)
      for (int r = 0; r < m; r++) acc[r + j * m] += vr[r] * wr[j];
  });
  for (int j = 0; j < k; j++)
    for (int r = 0; r < m; r++)
      at(C, r, j) = beta == 0.0 ? alpha * s[r + j * m] : alpha * s[r + j * m] + beta * at(C, r, j);
}

// W = alpha V C + beta W (gemm_kernels_sB.F90)
void mvsd(double alpha, const Mvec* V, const Sd* C, double beta, Mvec* W)
{
  const int m = V->nvec, k = W->nvec;
#pragma omp parallel for schedule(static)
  for (int64_t i = 0; i < V->n; i++)
    for (int c = 0; c < k; c++) {
      double acc = 0.0;
      for (int j = 0; j < m; j++) acc += at(V, i, j) * at(C, j, c);
      at(W, i, c) = beta == 0.0 ? alpha * acc : alpha * acc + beta * at(W, i, c);
    }
}

// V(:, 0:k) = V M in place, row by row (gemm_kernels_sB.F90:519-613)
void mvsdi(Mvec* V, const Sd* M)
{
  const int m = V->nvec, k = M->nc;
#pragma omp parallel
  {
    std::vector<double> row(m);
#pragma omp for schedule(static)
    for (int64_t i = 0; i < V->n; i++) {
      for (int j = 0; j < m; j++) row[j] = at(V, i, j);
      for (int c = 0; c < k; c++) {
        double acc = 0.0;
        for (int j = 0; j < m; j++) acc += row[j] * at(M, j, c);
        at(V, i, c) = acc;
      }
    }
  }
}

// uniform [-1,1) of the library's counter-based generator (splitmix64)
uint64_t mix64(uint64_t z)
{
  z += 0x9E3779B97F4A7C15ull;
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return z ^ (z >> 31);
}
double unif(uint64_t seed, uint64_t idx)
{
  const uint64_t h = mix64(seed * 0x632BE59BD9B4E019ull + mix64(idx));
  return (double)(h >> 11) * (1.0 / 9007199254740992.0) * 2.0 - 1.0;
}

// the 7-point stencil matrices of the benchmark problems (the same rows as
// phist_b200/generators.py:stencil3d): lexicographic order x fastest,
// columns sorted, diag0 + uniform[lo, hi) on the diagonal (seeded)
Sp* stencil3d(int64_t L, bool periodic, double diag0, double lo, double hi, uint64_t seed)
{
  Sp* A = new Sp();
  const int64_t n = L * L * L;
  A->n = A->m = n;
  A->rp.assign(n + 1, 0);
  A->col.reserve(n * 7);
  A->val.reserve(n * 7);
  for (int64_t i = 0; i < n; i++) {
    const int64_t x = i % L, y = (i / L) % L, z = i / (L * L);
    const int64_t co[3] = {x, y, z}, st[3] = {1, L, L * L};
    std::vector<std::pair<int64_t, double>> e;
    for (int d = 0; d < 3; d++)
      for (int s = -1; s <= 1; s += 2) {
        int64_t xn = co[d] + s;
        if (periodic) xn = (xn + L) % L;
        else if (xn < 0 || xn >= L) continue;
        if (xn == co[d]) continue;
        e.push_back({i + (xn - co[d]) * st[d], -1.0});
      }
    const double r = hi == lo ? lo : lo + (hi - lo) * (unif(seed, (uint64_t)i) + 1.0) * 0.5;
    e.push_back({i, diag0 + r});
    std::sort(e.begin(), e.end(), [](const std::pair<int64_t, double>& a, const std::pair<int64_t, double>& b) {
      return a.first < b.first;
    });
    for (auto& q : e) {
      A->col.push_back((int32_t)q.first);
      A->val.push_back(q.second);
    }
    A->rp[i + 1] = (int64_t)A->col.size();
  }
  A->rmap = new Map{n};
  A->dmap = A->rmap;
  return A;
}

}  // namespace

#define API extern "C"
#define OK (*iflag = 0)

// ------------------------------------------------------------ untyped API
API void phist_kernels_init(int*, char***, int* iflag) { OK; }
API void phist_kernels_finalize(int* iflag) { OK; }
API void phist_comm_create(void** comm, int* iflag) { *comm = &g_comm_dummy; OK; }
API void phist_comm_delete(void*, int* iflag) { OK; }
API void phist_map_get_comm(const void*, const void** comm, int* iflag) { *comm = &g_comm_dummy; OK; }
API void phist_map_get_local_length(const void* m, int32_t* n, int* iflag) { *n = (int32_t)((const Map*)m)->n; OK; }
API void phist_b200_set_sell_params(int, int64_t, int* iflag) { OK; }
API void phist_b200_synchronize(int* iflag) { OK; }
API void phist_b200_launch_count(uint64_t* c, int* iflag) { *c = 0; OK; }

// problems LAPLACE3D-L, LAPDIAG3D-L-S<seed>, ANDERSON3D-L-S<seed>[-W<w>]
API void phist_b200_Dcreate_problem(void** A, const void*, const char* problem, int* iflag)
{
  std::string s(problem);
  std::vector<std::string> parts;
  size_t a = 0;
  for (size_t b; (b = s.find('-', a)) != std::string::npos; a = b + 1) parts.push_back(s.substr(a, b - a));
  parts.push_back(s.substr(a));
  if (parts.size() < 2) { *iflag = kInvalid; return; }
  const int64_t L = atoll(parts[1].c_str());
  uint64_t seed = 0;
  double W = 16.5;
  for (size_t q = 2; q < parts.size(); q++) {
    if (parts[q][0] == 'S') seed = strtoull(parts[q].c_str() + 1, nullptr, 10);
    if (parts[q][0] == 'W') W = atof(parts[q].c_str() + 1);
  }
  if (L < 3) { *iflag = kInvalid; return; }
  if (parts[0] == "LAPLACE3D") *A = stencil3d(L, false, 6.0, 0.0, 0.0, 0);
  else if (parts[0] == "LAPDIAG3D") *A = stencil3d(L, false, 6.0, 0.0, 1.0, seed);
  else if (parts[0] == "ANDERSON3D") *A = stencil3d(L, true, 0.0, -W / 2, W / 2, seed);
  else { *iflag = kNotImpl; return; }
  OK;
}

// ------------------------------------------------------------ sparseMat
API void phist_DsparseMat_delete(void* A, int* iflag)
{
  if (A) { delete SP(A)->rmap; delete SP(A); }
  OK;
}
API void phist_DsparseMat_get_row_map(const void* A, const void** m, int* iflag) { *m = SP(A)->rmap; OK; }
API void phist_DsparseMat_get_range_map(const void* A, const void** m, int* iflag) { *m = SP(A)->rmap; OK; }
API void phist_DsparseMat_get_domain_map(const void* A, const void** m, int* iflag) { *m = SP(A)->dmap; OK; }
API void phist_DsparseMat_times_mvec(double alpha, const void* A, const void* X, double beta, void* Y, int* iflag)
{
  spmv(alpha, SP(A), nullptr, MV(X), beta, MV(Y));
  OK;
}
API void phist_DsparseMat_times_mvec_add_mvec(double alpha, const void* A, double shift, const void* X, double beta,
                                             void* Y, int* iflag)
{
  std::vector<double> sh(MV(X)->nvec, shift);
  spmv(alpha, SP(A), sh.data(), MV(X), beta, MV(Y));
  OK;
}
API void phist_DsparseMat_times_mvec_vadd_mvec(double alpha, const void* A, const double* shifts, const void* X,
                                              double beta, void* Y, int* iflag)
{
  spmv(alpha, SP(A), shifts, MV(X), beta, MV(Y));
  OK;
}
API void phist_DsparseMatT_times_mvec(double, const void*, const void*, double, void*, int* iflag)
{
  *iflag = kNotImpl;
}

// ------------------------------------------------------------ mvec
API void phist_Dmvec_create(void** V, const void* map, int nvec, int* iflag)
{
  const Map* m = (const Map*)map;
  Mvec* X = new Mvec{m, m->n, nvec, nvec, (double*)calloc((size_t)(m->n > 0 ? m->n : 1) * nvec, sizeof(double)), true};
  *V = X;
  OK;
}
API void phist_Dmvec_clone_shape(void** V, const void* W, int* iflag) { phist_Dmvec_create(V, MV(W)->map, MV(W)->nvec, iflag); }
API void phist_Dmvec_delete(void* V, int* iflag)
{
  if (V) {
    if (MV(V)->owner) free(MV(V)->v);
    delete MV(V);
  }
  OK;
}
API void phist_Dmvec_get_map(const void* V, const void** m, int* iflag) { *m = MV(V)->map; OK; }
API void phist_Dmvec_get_comm(const void*, const void** comm, int* iflag) { *comm = &g_comm_dummy; OK; }
API void phist_Dmvec_num_vectors(const void* V, int* nv, int* iflag) { *nv = MV(V)->nvec; OK; }
API void phist_Dmvec_extract_view(void* V, double** val, int32_t* lda, int* iflag)
{
  *val = MV(V)->v;
  *lda = (int32_t)MV(V)->lda;
  OK;
}
API void phist_Dmvec_from_device(void*, int* iflag) { OK; }
API void phist_Dmvec_to_device(void*, int* iflag) { OK; }
API void phist_Dmvec_set_data(void* V, const double* data, int32_t lda, int row_major, int* iflag)
{
  Mvec* X = MV(V);
  for (int64_t i = 0; i < X->n; i++)
    for (int j = 0; j < X->nvec; j++) at(X, i, j) = row_major ? data[i * lda + j] : data[i + (int64_t)j * lda];
  OK;
}
API void phist_Dmvec_view_block(void* V, void** Vb, int jmin, int jmax, int* iflag)
{
  Mvec* X = MV(V);
  if (jmin < 0 || jmax >= X->nvec || jmax < jmin) { *iflag = kInvalid; return; }
  Mvec* B = *Vb ? MV(*Vb) : new Mvec();
  if (*Vb && B->owner) free(B->v);
  *B = Mvec{X->map, X->n, jmax - jmin + 1, X->lda, X->v + jmin, false};
  *Vb = B;
  OK;
}
API void phist_Dmvec_get_block(const void* V, void* Vb, int jmin, int jmax, int* iflag)
{
  const Mvec* X = MV(V);
  Mvec* B = MV(Vb);
#pragma omp parallel for schedule(static)
  for (int64_t i = 0; i < X->n; i++)
    for (int j = jmin; j <= jmax; j++) at(B, i, j - jmin) = at(X, i, j);
  OK;
}
API void phist_Dmvec_set_block(void* V, const void* Vb, int jmin, int jmax, int* iflag)
{
  Mvec* X = MV(V);
  const Mvec* B = MV(Vb);
#pragma omp parallel for schedule(static)
  for (int64_t i = 0; i < X->n; i++)
    for (int j = jmin; j <= jmax; j++) at(X, i, j) = at(B, i, j - jmin);
  OK;
}
API void phist_Dmvec_put_value(void* V, double s, int* iflag)
{
  Mvec* X = MV(V);
#pragma omp parallel for schedule(static)
  for (int64_t i = 0; i < X->n; i++)
    for (int j = 0; j < X->nvec; j++) at(X, i, j) = s;
  OK;
}
// uniform [-1,1) from the counter-based generator of the GPU library (the
// builtin's KISS generator, phist_random.c, is not reproduced by either)
API void phist_Dmvec_random(void* V, int* iflag)
{
  static uint64_t calls = 0;
  Mvec* X = MV(V);
  const uint64_t seed = 0x5EED0000ull + calls++;
#pragma omp parallel for schedule(static)
  for (int64_t i = 0; i < X->n; i++)
    for (int j = 0; j < X->nvec; j++) at(X, i, j) = unif(seed, (uint64_t)(i * X->nvec + j));
  OK;
}
API void phist_Dmvec_scale(void* V, double s, int* iflag)
{
  Mvec* X = MV(V);
#pragma omp parallel for schedule(static)
  for (int64_t i = 0; i < X->n; i++)
    for (int j = 0; j < X->nvec; j++) at(X, i, j) *= s;
  OK;
}
API void phist_Dmvec_vscale(void* V, const double* s, int* iflag)
{
  Mvec* X = MV(V);
#pragma omp parallel for schedule(static)
  for (int64_t i = 0; i < X->n; i++)
    for (int j = 0; j < X->nvec; j++) at(X, i, j) *= s[j];
  OK;
}
API void phist_Dmvec_add_mvec(double a, const void* X, double b, void* Y, int* iflag)
{
  const Mvec* x = MV(X);
  Mvec* y = MV(Y);
#pragma omp parallel for schedule(static)
  for (int64_t i = 0; i < x->n; i++)
    for (int j = 0; j < x->nvec; j++) at(y, i, j) = b == 0.0 ? a * at(x, i, j) : a * at(x, i, j) + b * at(y, i, j);
  OK;
}
API void phist_Dmvec_vadd_mvec(const double* a, const void* X, double b, void* Y, int* iflag)
{
  const Mvec* x = MV(X);
  Mvec* y = MV(Y);
#pragma omp parallel for schedule(static)
  for (int64_t i = 0; i < x->n; i++)
    for (int j = 0; j < x->nvec; j++)
      at(y, i, j) = b == 0.0 ? a[j] * at(x, i, j) : a[j] * at(x, i, j) + b * at(y, i, j);
  OK;
}
API void phist_Dmvec_dot_mvec(const void* V, const void* W, double* d, int* iflag)
{
  const Mvec* v = MV(V);
  const Mvec* w = MV(W);
  reduce_rows(v->n, v->nvec, d, [&](int64_t i, double* acc) {
    for (int j = 0; j < v->nvec; j++) acc[j] += at(v, i, j) * at(w, i, j);
  });
  OK;
}
API void phist_Dmvec_norm2(const void* V, double* nrm, int* iflag)
{
  phist_Dmvec_dot_mvec(V, V, nrm, iflag);
  for (int j = 0; j < MV(V)->nvec; j++) nrm[j] = std::sqrt(nrm[j]);
}
API void phist_Dmvec_normalize(void* V, double* nrm, int* iflag)
{
  phist_Dmvec_norm2(V, nrm, iflag);
  std::vector<double> s(MV(V)->nvec);
  for (int j = 0; j < MV(V)->nvec; j++) s[j] = nrm[j] == 0.0 ? 1.0 : 1.0 / nrm[j];
  phist_Dmvec_vscale(V, s.data(), iflag);
}
API void phist_DmvecT_times_mvec(double alpha, const void* V, const void* W, double beta, void* C, int* iflag)
{
  mvtmv(alpha, MV(V), MV(W), beta, SD(C));
  OK;
}
API void phist_Dmvec_times_sdMat(double alpha, const void* V, const void* C, double beta, void* W, int* iflag)
{
  mvsd(alpha, MV(V), SD(C), beta, MV(W));
  OK;
}
API void phist_Dmvec_times_sdMat_inplace(void* V, const void* M, int* iflag)
{
  mvsdi(MV(V), SD(M));
  OK;
}
// W = V C + W D (gemm_kernels_sB_add_sD.F90)
API void phist_Dmvec_times_sdMat_add_mvec_times_sdMat(const void* V, const void* C, void* W, const void* D,
                                                     int* iflag)
{
  const Mvec* v = MV(V);
  Mvec* w = MV(W);
  const Sd* c = SD(C);
  const Sd* d = SD(D);
  const int m = v->nvec, k = w->nvec;
#pragma omp parallel
  {
    std::vector<double> row(k);
#pragma omp for schedule(static)
    for (int64_t i = 0; i < v->n; i++) {
      for (int j = 0; j < k; j++) row[j] = at(w, i, j);
      for (int q = 0; q < k; q++) {
        double acc = 0.0;
        for (int j = 0; j < m; j++) acc += at(v, i, j) * at(c, j, q);
        for (int j = 0; j < k; j++) acc += row[j] * at(d, j, q);
        at(w, i, q) = acc;
      }
    }
  }
  OK;
}
// W = alpha V C + beta W, WtW = W'W (gemm_kernels_sB_augmented.F90)
API void phist_Dfused_mvsd_mvTmv(double alpha, const void* V, const void* C, double beta, void* W, void* WtW,
                                 int* iflag)
{
  mvsd(alpha, MV(V), SD(C), beta, MV(W));
  if (WtW) mvtmv(1.0, MV(W), MV(W), 0.0, SD(WtW));
  OK;
}
// W = W C in place, D = alpha V'W + beta D, V read after the update when it
// is W itself (gemm_kernels_fused_sCD.F90)
API void phist_Dfused_mvsdi_mvTmv(double alpha, const void* V, void* W, const void* C, double beta, void* D,
                                  int* iflag)
{
  mvsdi(MV(W), SD(C));
  if (D) {
    Mvec Wk = *MV(W);
    Wk.nvec = SD(C)->nc;
    mvtmv(alpha, MV(V), &Wk, beta, SD(D));
  }
  OK;
}
API void phist_Dfused_spmv_mvTmv(double alpha, const void* A, const void* V, double beta, void* W, void* WtW,
                                 void* VtW, int* iflag)
{
  void* tmp = nullptr;
  if (!W) {
    phist_Dmvec_create(&tmp, SP(A)->rmap, MV(V)->nvec, iflag);
    W = tmp;
    beta = 0.0;
  }
  spmv(alpha, SP(A), nullptr, MV(V), beta, MV(W));
  if (WtW) mvtmv(1.0, MV(W), MV(W), 0.0, SD(WtW));
  if (VtW) mvtmv(1.0, MV(V), MV(W), 0.0, SD(VtW));
  if (tmp) phist_Dmvec_delete(tmp, iflag);
  OK;
}
API void phist_Dfused_spmv_pair(double, const double*, const void*, const double*, const void*, const void*,
                                double, void*, int* iflag)
{
  *iflag = kNotImpl;
}

// ------------------------------------------------------------ sdMat
API void phist_DsdMat_create(void** M, int nr, int nc, const void*, int* iflag)
{
  *M = new Sd{nr, nc, nr > 0 ? nr : 1, (double*)calloc((size_t)(nr > 0 ? nr : 1) * (nc > 0 ? nc : 1), sizeof(double)),
              true};
  OK;
}
API void phist_DsdMat_delete(void* M, int* iflag)
{
  if (M) {
    if (SD(M)->owner) free(SD(M)->v);
    delete SD(M);
  }
  OK;
}
API void phist_DsdMat_get_nrows(const void* M, int* n, int* iflag) { *n = SD(M)->nr; OK; }
API void phist_DsdMat_get_ncols(const void* M, int* n, int* iflag) { *n = SD(M)->nc; OK; }
API void phist_DsdMat_extract_view(void* M, double** val, int32_t* lda, int* iflag)
{
  *val = SD(M)->v;
  *lda = (int32_t)SD(M)->lda;
  OK;
}
API void phist_DsdMat_from_device(void*, int* iflag) { OK; }
API void phist_DsdMat_to_device(void*, int* iflag) { OK; }
API void phist_DsdMat_sync_values(void*, const void*, int* iflag) { OK; }
API void phist_DsdMat_put_value(void* M, double s, int* iflag)
{
  for (int j = 0; j < SD(M)->nc; j++)
    for (int i = 0; i < SD(M)->nr; i++) at(SD(M), i, j) = s;
  OK;
}
API void phist_DsdMat_identity(void* M, int* iflag)
{
  for (int j = 0; j < SD(M)->nc; j++)
    for (int i = 0; i < SD(M)->nr; i++) at(SD(M), i, j) = i == j ? 1.0 : 0.0;
  OK;
}
API void phist_DsdMat_view_block(void* M, void** Mb, int imin, int imax, int jmin, int jmax, int* iflag)
{
  Sd* A = SD(M);
  if (imin < 0 || jmin < 0 || imax >= A->nr || jmax >= A->nc) { *iflag = kInvalid; return; }
  Sd* B = *Mb ? SD(*Mb) : new Sd();
  if (*Mb && B->owner) free(B->v);
  *B = Sd{imax - imin + 1, jmax - jmin + 1, A->lda, A->v + imin + (int64_t)jmin * A->lda, false};
  *Mb = B;
  OK;
}
API void phist_DsdMat_get_block(const void* M, void* Mb, int imin, int imax, int jmin, int jmax, int* iflag)
{
  for (int j = jmin; j <= jmax; j++)
    for (int i = imin; i <= imax; i++) at(SD(Mb), i - imin, j - jmin) = at(SD(M), i, j);
  OK;
}
API void phist_DsdMat_set_block(void* M, const void* Mb, int imin, int imax, int jmin, int jmax, int* iflag)
{
  for (int j = jmin; j <= jmax; j++)
    for (int i = imin; i <= imax; i++) at(SD(M), i, j) = at(SD(Mb), i - imin, j - jmin);
  OK;
}
// B = alpha A + beta B
API void phist_DsdMat_add_sdMat(double a, const void* A, double b, void* B, int* iflag)
{
  for (int j = 0; j < SD(B)->nc; j++)
    for (int i = 0; i < SD(B)->nr; i++)
      at(SD(B), i, j) = b == 0.0 ? a * at(SD(A), i, j) : a * at(SD(A), i, j) + b * at(SD(B), i, j);
  OK;
}
// B = alpha A' + beta B
API void phist_DsdMatT_add_sdMat(double a, const void* A, double b, void* B, int* iflag)
{
  for (int j = 0; j < SD(B)->nc; j++)
    for (int i = 0; i < SD(B)->nr; i++)
      at(SD(B), i, j) = b == 0.0 ? a * at(SD(A), j, i) : a * at(SD(A), j, i) + b * at(SD(B), i, j);
  OK;
}
// C = alpha V W + beta C
API void phist_DsdMat_times_sdMat(double a, const void* V, const void* W, double b, void* C, int* iflag)
{
  const Sd* v = SD(V);
  const Sd* w = SD(W);
  Sd* c = SD(C);
  if (v->nc != w->nr || c->nr != v->nr || c->nc != w->nc) { *iflag = kInvalid; return; }
  std::vector<double> r((size_t)c->nr * c->nc);
  for (int j = 0; j < c->nc; j++)
    for (int i = 0; i < c->nr; i++) {
      double s = 0.0;
      for (int q = 0; q < v->nc; q++) s += at(v, i, q) * at(w, q, j);
      r[i + (size_t)j * c->nr] = s;
    }
  for (int j = 0; j < c->nc; j++)
    for (int i = 0; i < c->nr; i++)
      at(c, i, j) = b == 0.0 ? a * r[i + (size_t)j * c->nr] : a * r[i + (size_t)j * c->nr] + b * at(c, i, j);
  OK;
}
// C = alpha V' W + beta C
API void phist_DsdMatT_times_sdMat(double a, const void* V, const void* W, double b, void* C, int* iflag)
{
  const Sd* v = SD(V);
  const Sd* w = SD(W);
  Sd* c = SD(C);
  if (v->nr != w->nr || c->nr != v->nc || c->nc != w->nc) { *iflag = kInvalid; return; }
  std::vector<double> r((size_t)c->nr * c->nc);
  for (int j = 0; j < c->nc; j++)
    for (int i = 0; i < c->nr; i++) {
      double s = 0.0;
      for (int q = 0; q < v->nr; q++) s += at(v, q, i) * at(w, q, j);
      r[i + (size_t)j * c->nr] = s;
    }
  for (int j = 0; j < c->nc; j++)
    for (int i = 0; i < c->nr; i++)
      at(c, i, j) = b == 0.0 ? a * r[i + (size_t)j * c->nr] : a * r[i + (size_t)j * c->nr] + b * at(c, i, j);
  OK;
}

// ------------------------------------------------------------ CARP: not
// needed by the eigen-solves (PHIST's carp_cg runs on the GPU library only)
API void phist_Dcarp_setup(const void*, int, const double*, void**, int* iflag) { *iflag = kNotImpl; }
API void phist_Dcarp_destroy(const void*, void*, int* iflag) { *iflag = kNotImpl; }
