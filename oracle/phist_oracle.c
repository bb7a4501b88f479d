/*
 * phist_oracle.c -- CPU oracle for the PHIST kernel path (TEST INFRASTRUCTURE).
 *
 * Plain C restatement of PHIST's builtin kernels; see phist_oracle.h for the
 * contract and the reference lines each function follows.  Only tests/, the
 * smoke check and bench.py's CPU-baseline leg use this file.
 */
#include "phist_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

int orc_num_threads(void)
{
#ifdef _OPENMP
  return omp_get_max_threads();
#else
  return 1;
#endif
}

void orc_set_num_threads(int n)
{
#ifdef _OPENMP
  if (n > 0) omp_set_num_threads(n);
#else
  (void)n;
#endif
}

/* --------------------------------------------------------------- SpMMV */

void orc_spmmv(int64_t nrows, const int64_t* row_ptr, const int32_t* col,
               const double* val, int nvec, double alpha,
               const double* shifts, const double* x, int64_t ldx,
               double beta, double* y, int64_t ldy)
{
  const int64_t nnz = row_ptr[nrows] - row_ptr[0];
  if (alpha == 0.0 || nnz == 0) {
    /* crsmat_module.F90:1508-1511: only scale y (mvec_scale) */
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < nrows; i++)
      for (int j = 0; j < nvec; j++) y[i * ldy + j] = beta * y[i * ldy + j];
    return;
  }
#pragma omp parallel
  {
    double tmp_stack[64];
    double* tmp = nvec <= 64 ? tmp_stack : (double*)malloc(sizeof(double) * nvec);
#pragma omp for schedule(static)
    for (int64_t i = 0; i < nrows; i++) {
      /* tmp(:) = shifts*x(:,i) */
      for (int j = 0; j < nvec; j++)
        tmp[j] = (shifts ? shifts[j] : 0.0) * x[i * ldx + j];
      for (int64_t p = row_ptr[i]; p < row_ptr[i + 1]; p++) {
        const double a = val[p];
        const double* xr = x + (int64_t)col[p] * ldx;
        for (int j = 0; j < nvec; j++) tmp[j] += a * xr[j];
      }
      if (beta == 0.0) {
        for (int j = 0; j < nvec; j++) y[i * ldy + j] = alpha * tmp[j];
      } else {
        for (int j = 0; j < nvec; j++)
          y[i * ldy + j] = alpha * tmp[j] + beta * y[i * ldy + j];
      }
    }
    if (tmp != tmp_stack) free(tmp);
  }
}

void orc_sspmmv(int64_t nrows, const int64_t* row_ptr, const int32_t* col,
                const float* val, int nvec, float alpha, const float* shifts,
                const float* x, int64_t ldx, float beta, float* y, int64_t ldy)
{
  const int64_t nnz = row_ptr[nrows] - row_ptr[0];
  if (alpha == 0.0f || nnz == 0) {
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < nrows; i++)
      for (int j = 0; j < nvec; j++) y[i * ldy + j] = beta * y[i * ldy + j];
    return;
  }
#pragma omp parallel
  {
    float tmp_stack[64];
    float* tmp = nvec <= 64 ? tmp_stack : (float*)malloc(sizeof(float) * nvec);
#pragma omp for schedule(static)
    for (int64_t i = 0; i < nrows; i++) {
      for (int j = 0; j < nvec; j++)
        tmp[j] = (shifts ? shifts[j] : 0.0f) * x[i * ldx + j];
      for (int64_t p = row_ptr[i]; p < row_ptr[i + 1]; p++) {
        const float a = val[p];
        const float* xr = x + (int64_t)col[p] * ldx;
        for (int j = 0; j < nvec; j++) tmp[j] += a * xr[j];
      }
      if (beta == 0.0f) {
        for (int j = 0; j < nvec; j++) y[i * ldy + j] = alpha * tmp[j];
      } else {
        for (int j = 0; j < nvec; j++)
          y[i * ldy + j] = alpha * tmp[j] + beta * y[i * ldy + j];
      }
    }
    if (tmp != tmp_stack) free(tmp);
  }
}

/* ------------------------------------------------------- block products */

/* rows are summed in fixed blocks of ORC_BLK, blocks in order: the result
 * does not depend on the thread count */
#define ORC_BLK 8192

void orc_mvTmv(int64_t n, int m, int k, double alpha, const double* V,
               int64_t ldv, const double* W, int64_t ldw, double beta,
               double* C, int64_t ldc)
{
  const int64_t nblk = (n + ORC_BLK - 1) / ORC_BLK;
  const size_t mk = (size_t)m * k;
  double* P = (double*)calloc((size_t)(nblk > 0 ? nblk : 1) * mk, sizeof(double));
#pragma omp parallel for schedule(static)
  for (int64_t b = 0; b < nblk; b++) {
    double* Ml = P + (size_t)b * mk;
    const int64_t i1 = (b + 1) * ORC_BLK < n ? (b + 1) * ORC_BLK : n;
    for (int64_t i = b * ORC_BLK; i < i1; i++)
      for (int j = 0; j < k; j++) {
        const double w = W[i * ldw + j];
        for (int r = 0; r < m; r++) Ml[r + j * m] += V[i * ldv + r] * w;
      }
  }
  for (int j = 0; j < k; j++)
    for (int r = 0; r < m; r++) {
      double acc = 0.0;
      for (int64_t b = 0; b < nblk; b++) acc += P[(size_t)b * mk + r + j * m];
      double* c = &C[r + j * ldc];
      *c = (beta == 0.0) ? alpha * acc : alpha * acc + beta * (*c);
    }
  free(P);
}

/* error-free transformations (Knuth TwoSum, TwoProduct via fma) */
static inline void two_sum(double a, double b, double* s, double* e)
{
  double x = a + b;
  double z = x - a;
  *e = (a - (x - z)) + (b - z);
  *s = x;
}
static inline void two_prod(double a, double b, double* p, double* e)
{
  double x = a * b;
  *e = fma(a, b, -x);
  *p = x;
}
/* (s,c) += a*b, Dot2 step of Ogita/Rump/Oishi */
static inline void dot2_step(double a, double b, double* s, double* c)
{
  double p, ep, t, et;
  two_prod(a, b, &p, &ep);
  two_sum(*s, p, &t, &et);
  *s = t;
  *c += ep + et;
}

void orc_mvTmv_prec(int64_t n, int m, int k, double alpha, const double* V,
                    int64_t ldv, const double* W, int64_t ldw, double beta,
                    double* C, int64_t ldc)
{
  for (int j = 0; j < k; j++)
    for (int r = 0; r < m; r++) {
      double s = 0.0, c = 0.0;
      for (int64_t i = 0; i < n; i++) dot2_step(V[i * ldv + r], W[i * ldw + j], &s, &c);
      /* alpha*(s+c) + beta*C in double-double, rounded once */
      double p, ep, q, eq, t, et;
      two_prod(alpha, s, &p, &ep);
      ep += alpha * c;
      double cc = C[r + j * ldc];
      if (beta == 0.0) { q = 0.0; eq = 0.0; } else two_prod(beta, cc, &q, &eq);
      two_sum(p, q, &t, &et);
      C[r + j * ldc] = t + (et + ep + eq);
    }
}

void orc_mvsd(int64_t n, int m, int k, double alpha, const double* V,
              int64_t ldv, const double* C, int64_t ldc, double beta,
              double* W, int64_t ldw)
{
#pragma omp parallel for schedule(static)
  for (int64_t i = 0; i < n; i++)
    for (int c = 0; c < k; c++) {
      double acc = (beta == 0.0) ? 0.0 : beta * W[i * ldw + c];
      for (int j = 0; j < m; j++) acc += alpha * C[j + c * ldc] * V[i * ldv + j];
      W[i * ldw + c] = acc;
    }
}

void orc_mvsdi(int64_t n, int m, int k, double* V, int64_t ldv,
               const double* M, int64_t ldm)
{
#pragma omp parallel
  {
    double* row = (double*)malloc(sizeof(double) * (m > 0 ? m : 1));
#pragma omp for schedule(static)
    for (int64_t i = 0; i < n; i++) {
      for (int j = 0; j < m; j++) row[j] = V[i * ldv + j];
      for (int c = 0; c < k; c++) {
        double acc = 0.0;
        for (int j = 0; j < m; j++) acc += row[j] * M[j + c * ldm];
        V[i * ldv + c] = acc;
      }
    }
    free(row);
  }
}

void orc_mvsd_add_mvsd(int64_t n, int m, int k, const double* V, int64_t ldv,
                       const double* C, int64_t ldc, double* W, int64_t ldw,
                       const double* D, int64_t ldd)
{
#pragma omp parallel
  {
    double* wrow = (double*)malloc(sizeof(double) * (k > 0 ? k : 1));
#pragma omp for schedule(static)
    for (int64_t i = 0; i < n; i++) {
      for (int j = 0; j < k; j++) wrow[j] = W[i * ldw + j];
      for (int c = 0; c < k; c++) {
        double acc = 0.0;
        for (int j = 0; j < k; j++) acc += wrow[j] * D[j + c * ldd];
        for (int j = 0; j < m; j++) acc += V[i * ldv + j] * C[j + c * ldc];
        W[i * ldw + c] = acc;
      }
    }
    free(wrow);
  }
}

void orc_fused_mvsd_mvTmv(int64_t n, int m, int k, double alpha,
                          const double* V, int64_t ldv, const double* C,
                          int64_t ldc, double beta, double* W, int64_t ldw,
                          double* WtW, int64_t ldwtw)
{
  orc_mvsd(n, m, k, alpha, V, ldv, C, ldc, beta, W, ldw);
  if (WtW) orc_mvTmv(n, k, k, 1.0, W, ldw, W, ldw, 0.0, WtW, ldwtw);
}

void orc_fused_mvsdi_mvTmv(int64_t n, int mv, int m, int k, double alpha,
                           const double* V, int64_t ldv, double* W,
                           int64_t ldw, const double* C, int64_t ldc,
                           double beta, double* D, int64_t ldd)
{
  orc_mvsdi(n, m, k, W, ldw, C, ldc);
  if (D) orc_mvTmv(n, mv, k, alpha, V, ldv, W, ldw, beta, D, ldd);
}

/* ---------------------------------------------------------------- BLAS1 */

void orc_dot(int64_t n, int nvec, const double* V, int64_t ldv,
             const double* W, int64_t ldw, double* out)
{
  const int64_t nblk = (n + ORC_BLK - 1) / ORC_BLK;
  double* P = (double*)calloc((size_t)(nblk > 0 ? nblk : 1) * (nvec > 0 ? nvec : 1), sizeof(double));
#pragma omp parallel for schedule(static)
  for (int64_t b = 0; b < nblk; b++) {
    double* l = P + (size_t)b * nvec;
    const int64_t i1 = (b + 1) * ORC_BLK < n ? (b + 1) * ORC_BLK : n;
    for (int64_t i = b * ORC_BLK; i < i1; i++)
      for (int j = 0; j < nvec; j++) l[j] += V[i * ldv + j] * W[i * ldw + j];
  }
  for (int j = 0; j < nvec; j++) {
    double acc = 0.0;
    for (int64_t b = 0; b < nblk; b++) acc += P[(size_t)b * nvec + j];
    out[j] = acc;
  }
  free(P);
}

void orc_dot_prec(int64_t n, int nvec, const double* V, int64_t ldv,
                  const double* W, int64_t ldw, double* out)
{
  for (int j = 0; j < nvec; j++) {
    double s = 0.0, c = 0.0;
    for (int64_t i = 0; i < n; i++) dot2_step(V[i * ldv + j], W[i * ldw + j], &s, &c);
    out[j] = s + c;
  }
}

void orc_norm2(int64_t n, int nvec, const double* V, int64_t ldv, double* out)
{
  orc_dot(n, nvec, V, ldv, V, ldv, out);
  for (int j = 0; j < nvec; j++) out[j] = sqrt(out[j]);
}

void orc_vadd(int64_t n, int nvec, double alpha, const double* valpha,
              const double* X, int64_t ldx, double beta, double* Y, int64_t ldy)
{
#pragma omp parallel for schedule(static)
  for (int64_t i = 0; i < n; i++)
    for (int j = 0; j < nvec; j++) {
      const double a = valpha ? valpha[j] : alpha;
      Y[i * ldy + j] = (beta == 0.0) ? a * X[i * ldx + j]
                                     : a * X[i * ldx + j] + beta * Y[i * ldy + j];
    }
}

void orc_vscale(int64_t n, int nvec, double* V, int64_t ldv, const double* s)
{
#pragma omp parallel for schedule(static)
  for (int64_t i = 0; i < n; i++)
    for (int j = 0; j < nvec; j++) V[i * ldv + j] *= s[j];
}

/* ----------------------------------------------------------------- CARP */

void orc_kacz_sweep(int64_t nrows, const int64_t* row_ptr, const int32_t* col,
                    const double* val, int nvec, const double* shifts,
                    const double* b, int64_t ldb, double* x, int64_t ldx,
                    const double* omega, const int32_t* order, int64_t nord)
{
  double* tmp = (double*)malloc(sizeof(double) * (nvec > 0 ? nvec : 1));
  double* rn = (double*)malloc(sizeof(double) * (nvec > 0 ? nvec : 1));
  (void)nrows;
  for (int64_t q = 0; q < nord; q++) {
    const int64_t i = order ? order[q] : q;
    double d = 0.0, nrm = 0.0;
    for (int j = 0; j < nvec; j++) tmp[j] = -shifts[j] * x[i * ldx + j];
    for (int64_t p = row_ptr[i]; p < row_ptr[i + 1]; p++) {
      const double a = val[p];
      const double* xr = x + (int64_t)col[p] * ldx;
      for (int j = 0; j < nvec; j++) tmp[j] += a * xr[j];
      nrm += a * a;
      if (col[p] == i) d = a;
    }
    if (b)
      for (int j = 0; j < nvec; j++) tmp[j] -= b[i * ldb + j];
    for (int j = 0; j < nvec; j++) {
      rn[j] = nrm - 2.0 * d * shifts[j] + shifts[j] * shifts[j];
      if (rn[j] == 0.0) rn[j] = 1.0;
      tmp[j] = tmp[j] * omega[j] / rn[j];
      x[i * ldx + j] += tmp[j] * shifts[j];
    }
    for (int64_t p = row_ptr[i]; p < row_ptr[i + 1]; p++) {
      const double a = val[p];
      double* xr = x + (int64_t)col[p] * ldx;
      for (int j = 0; j < nvec; j++) xr[j] -= tmp[j] * a;
    }
  }
  free(tmp);
  free(rn);
}

void orc_carp_sweep(int64_t nrows, const int64_t* row_ptr, const int32_t* col,
                    const double* val, int nvec, const double* shifts,
                    const double* b, int64_t ldb, double* x, int64_t ldx,
                    const double* omega)
{
  int32_t* ord = (int32_t*)malloc(sizeof(int32_t) * (nrows > 0 ? nrows : 1));
  for (int64_t i = 0; i < nrows; i++) ord[i] = (int32_t)i;
  orc_kacz_sweep(nrows, row_ptr, col, val, nvec, shifts, b, ldb, x, ldx, omega, ord, nrows);
  for (int64_t i = 0; i < nrows; i++) ord[i] = (int32_t)(nrows - 1 - i);
  orc_kacz_sweep(nrows, row_ptr, col, val, nvec, shifts, b, ldb, x, ldx, omega, ord, nrows);
  free(ord);
}

/* ------------------------------------------------------------ SELL-C-sigma */

void orc_sell_perm(int64_t nrows, const int64_t* row_ptr, int64_t sigma,
                   int32_t* perm)
{
  for (int64_t i = 0; i < nrows; i++) perm[i] = (int32_t)i;
  if (sigma <= 1) return;
  for (int64_t w0 = 0; w0 < nrows; w0 += sigma) {
    int64_t w1 = w0 + sigma < nrows ? w0 + sigma : nrows;
    /* stable insertion sort by descending length inside the window */
    for (int64_t a = w0 + 1; a < w1; a++) {
      int32_t r = perm[a];
      int64_t len = row_ptr[r + 1] - row_ptr[r];
      int64_t q = a - 1;
      while (q >= w0 && (row_ptr[perm[q] + 1] - row_ptr[perm[q]]) < len) {
        perm[q + 1] = perm[q];
        q--;
      }
      perm[q + 1] = r;
    }
  }
}

int64_t orc_check_dist2(int64_t nrows, const int64_t* row_ptr,
                        const int32_t* col, int64_t ncols,
                        const int32_t* color)
{
  /* for every column, the set of colours of rows touching it must be unique */
  int32_t* seen_color = (int32_t*)malloc(sizeof(int32_t) * (ncols > 0 ? ncols : 1));
  int64_t* seen_row = (int64_t*)malloc(sizeof(int64_t) * (ncols > 0 ? ncols : 1));
  int64_t bad = 0;
  int32_t maxc = 0;
  for (int64_t i = 0; i < nrows; i++) if (color[i] > maxc) maxc = color[i];
  /* one pass per colour keeps memory O(ncols) */
  for (int32_t c = 0; c <= maxc && !bad; c++) {
    for (int64_t j = 0; j < ncols; j++) seen_row[j] = -1;
    for (int64_t i = 0; i < nrows && !bad; i++) {
      if (color[i] != c) continue;
      for (int64_t p = row_ptr[i]; p < row_ptr[i + 1]; p++) {
        int32_t j = col[p];
        if (seen_row[j] >= 0 && seen_row[j] != i) { bad = i + 1; break; }
        seen_row[j] = i;
      }
    }
  }
  (void)seen_color;
  free(seen_color);
  free(seen_row);
  return bad;
}
