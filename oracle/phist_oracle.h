/*
 * phist_oracle.h -- CPU oracle for the PHIST kernel path (TEST INFRASTRUCTURE).
 *
 * This library is the checker, not the product: only tests/, the smoke check
 * and bench.py's CPU-baseline leg load it.  The shipped library
 * (phist_b200/lib/libphist_kernels_b200.so) never links or calls it.
 *
 * Every function restates, in plain C with OpenMP, the algorithm of PHIST's
 * "builtin" CPU kernel library (Fortran 2008 + C, src/kernels/builtin/ in the
 * PHIST sources).  The loop order and update formulae follow the cited
 * reference lines so that results agree to rounding.  Data layout follows the
 * builtin library: CRS with 0-based int64 row offsets and int32 column
 * indices, row-major block vectors (element (i,j) at x[i*ldx+j]) and
 * column-major small dense matrices (element (i,j) at C[i+j*ldc]).
 *
 * Parity pins (tests/test_oracle.py): the reference's own C kernels
 * (spmvm_kernels_nt.c, dot_kernels_prec.c, gemm_kernels_sC_prec.c) compiled
 * from the PHIST sources into oracle/_ref/, and the golden result vectors of
 * test/kernels/SparseMatTest_def.hpp (A2_precalc_result) extracted into
 * tests/golden/.
 */
#ifndef PHIST_ORACLE_H
#define PHIST_ORACLE_H
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* number of OpenMP threads the oracle uses (1 without OpenMP) */
int orc_num_threads(void);
void orc_set_num_threads(int n);

/* ---------------------------------------------------------------- SpMMV */
/* Y = alpha*(A + diag(shifts))*X + beta*Y, column j uses shifts[j]
 * (shifts may be NULL: all zero).  alpha==0 or nnz==0: Y = beta*Y.
 * beta==0: Y is not read (non-temporal path of the reference).
 * Follows crsmat_module.F90:1476-1672 (dispatch, alpha==0 scale-only at
 * :1508-1511) and spmvm_kernels.F90:494-523 (dspmvm_generic: tmp=shift*x_i,
 * local columns in stored order, y=alpha*tmp+beta*y). */
void orc_spmmv(int64_t nrows, const int64_t* row_ptr, const int32_t* col,
               const double* val, int nvec, double alpha,
               const double* shifts, const double* x, int64_t ldx,
               double beta, double* y, int64_t ldy);

/* single-precision counterpart with FP32 accumulation (mixed-precision form;
 * the reference builtin has no S kernels, builtin/kernels.cpp:270-283) */
void orc_sspmmv(int64_t nrows, const int64_t* row_ptr, const int32_t* col,
                const float* val, int nvec, float alpha,
                const float* shifts, const float* x, int64_t ldx,
                float beta, float* y, int64_t ldy);

/* ------------------------------------------------------- block products */
/* C(m x k, col-major) = alpha * V' W + beta*C; V n x m (ldv), W n x k (ldw).
 * Per-entry sum over rows in row order, as gemm_kernels_sC.F90:17-80 with
 * the alpha/beta update of mvec_module.F90:2729-2743. */
void orc_mvTmv(int64_t n, int m, int k, double alpha, const double* V,
               int64_t ldv, const double* W, int64_t ldw, double beta,
               double* C, int64_t ldc);

/* compensated (double-double) variant: TwoSum/TwoProduct error-free
 * transformations (Ogita, Rump, Oishi 2005, "Dot2"), the algorithm of
 * gemm_kernels_sC_prec.c / phist_prec_helpers.h.  The result is rounded
 * once at the end. */
void orc_mvTmv_prec(int64_t n, int m, int k, double alpha, const double* V,
                    int64_t ldv, const double* W, int64_t ldw, double beta,
                    double* C, int64_t ldc);

/* W(n x k) = alpha * V(n x m) C(m x k) + beta * W; beta==0: W not read.
 * gemm_kernels_sB.F90:15-133 (C(:,i)=beta*C(:,i); += alpha*B(:,j)*A(j,i)). */
void orc_mvsd(int64_t n, int m, int k, double alpha, const double* V,
              int64_t ldv, const double* C, int64_t ldc, double beta,
              double* W, int64_t ldw);

/* V(:,0:k-1) <- V(:,0:m-1) * M(m x k), k <= m, row by row in place
 * (gemm_kernels_sB.F90:519-613). */
void orc_mvsdi(int64_t n, int m, int k, double* V, int64_t ldv,
               const double* M, int64_t ldm);

/* W(n x k) <- V(n x m) C(m x k) + W D(k x k)  (gemm_kernels_sB_add_sD.F90) */
void orc_mvsd_add_mvsd(int64_t n, int m, int k, const double* V, int64_t ldv,
                       const double* C, int64_t ldc, double* W, int64_t ldw,
                       const double* D, int64_t ldd);

/* W = alpha V C + beta W, then WtW(k x k) = W'W
 * (gemm_kernels_sB_augmented.F90, mvec_module.F90:1915-2151) */
void orc_fused_mvsd_mvTmv(int64_t n, int m, int k, double alpha,
                          const double* V, int64_t ldv, const double* C,
                          int64_t ldc, double beta, double* W, int64_t ldw,
                          double* WtW, int64_t ldwtw);

/* W(n x k) <- W(:,0:m-1)*C(m x k) in place, then D(mv x k) = alpha V'W + beta D
 * (gemm_kernels_fused_sCD.F90, mvec_module.F90:2748-3080) */
void orc_fused_mvsdi_mvTmv(int64_t n, int mv, int m, int k, double alpha,
                           const double* V, int64_t ldv, double* W,
                           int64_t ldw, const double* C, int64_t ldc,
                           double beta, double* D, int64_t ldd);

/* ---------------------------------------------------------------- BLAS1 */
void orc_dot(int64_t n, int nvec, const double* V, int64_t ldv,
             const double* W, int64_t ldw, double* out);
void orc_dot_prec(int64_t n, int nvec, const double* V, int64_t ldv,
                  const double* W, int64_t ldw, double* out);
void orc_norm2(int64_t n, int nvec, const double* V, int64_t ldv, double* out);
/* Y = alpha[j]*X + beta*Y (alpha scalar when valpha==NULL) */
void orc_vadd(int64_t n, int nvec, double alpha, const double* valpha,
              const double* X, int64_t ldx, double beta, double* Y,
              int64_t ldy);
void orc_vscale(int64_t n, int nvec, double* V, int64_t ldv,
                const double* s);

/* ----------------------------------------------------------------- CARP */
/* One Kaczmarz sweep for (A - shifts[j] I) x_j = b_j over the rows in
 * order[0..nord-1] (forward) -- call again with the reversed order for the
 * backward half.  b may be NULL (b = 0).  Update formulae of
 * kacz_sub_def.h:50-150 (row norm on the fly with shift correction at
 * :102-111, projection x_i += tmp*shift, x_col -= tmp*a) with the row loop
 * of kacz_loop_seq_def.h (order = 0..n-1) or kacz_loop_clr_def.h (order =
 * rows grouped by colour). */
void orc_kacz_sweep(int64_t nrows, const int64_t* row_ptr, const int32_t* col,
                    const double* val, int nvec, const double* shifts,
                    const double* b, int64_t ldb, double* x, int64_t ldx,
                    const double* omega, const int32_t* order, int64_t nord);

/* forward then backward sweep in natural row order
 * (crsmat_module.F90:2889-2946 with one process: no import/average) */
void orc_carp_sweep(int64_t nrows, const int64_t* row_ptr, const int32_t* col,
                    const double* val, int nvec, const double* shifts,
                    const double* b, int64_t ldb, double* x, int64_t ldx,
                    const double* omega);

/* ------------------------------------------------------------ SELL-C-sigma */
/* Row permutation of SELL-C-sigma: inside each window of sigma consecutive
 * rows, rows are stably sorted by descending length.  perm[new] = old.
 * sigma<=1 gives the identity.  (Layout semantics as chosen for GHOST in
 * ghost/kernels.cpp:69-134; the sort itself is this project's own
 * convention, pinned bit-exactly against the library.) */
void orc_sell_perm(int64_t nrows, const int64_t* row_ptr, int64_t sigma,
                   int32_t* perm);

/* distance-2 colouring check: returns 0 if no two rows of one colour share
 * a column index, else 1 + index of the first offending row */
int64_t orc_check_dist2(int64_t nrows, const int64_t* row_ptr,
                        const int32_t* col, int64_t ncols,
                        const int32_t* color);

#ifdef __cplusplus
}
#endif
#endif
