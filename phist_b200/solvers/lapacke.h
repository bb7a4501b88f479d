/* Minimal LAPACKE interface for compiling PHIST's solver layers without a
 * system lapacke.h.  Declares the real-valued LAPACKE routines PHIST's
 * src/tools/phist_lapack.h maps its macros to (standard LAPACKE signatures,
 * column/row-major layout argument first) and binds them, together with the
 * Fortran BLAS names, to the OpenBLAS build that ships with SciPy, whose
 * symbols carry a "scipy_" prefix. */
#ifndef PHIST_B200_LAPACKE_SHIM_H
#define PHIST_B200_LAPACKE_SHIM_H

#ifdef __cplusplus
extern "C" {
#endif

typedef int lapack_int;
typedef int lapack_logical;
typedef lapack_logical (*LAPACK_S_SELECT2)(const float*, const float*);
typedef lapack_logical (*LAPACK_D_SELECT2)(const double*, const double*);
typedef lapack_logical (*LAPACK_S_SELECT3)(const float*, const float*, const float*);
typedef lapack_logical (*LAPACK_D_SELECT3)(const double*, const double*, const double*);

#define LAPACK_ROW_MAJOR 101
#define LAPACK_COL_MAJOR 102
#define LAPACK_GLOBAL(lcname, UCNAME) lcname##_

/* name binding to the prefixed OpenBLAS symbols */
#define LAPACKE_sgees scipy_LAPACKE_sgees
#define LAPACKE_dgees scipy_LAPACKE_dgees
#define LAPACKE_sgemqrt scipy_LAPACKE_sgemqrt
#define LAPACKE_dgemqrt scipy_LAPACKE_dgemqrt
#define LAPACKE_sgeqrt scipy_LAPACKE_sgeqrt
#define LAPACKE_dgeqrt scipy_LAPACKE_dgeqrt
#define LAPACKE_sgesvd scipy_LAPACKE_sgesvd
#define LAPACKE_dgesvd scipy_LAPACKE_dgesvd
#define LAPACKE_sgges scipy_LAPACKE_sgges
#define LAPACKE_dgges scipy_LAPACKE_dgges
#define LAPACKE_slartgp scipy_LAPACKE_slartgp
#define LAPACKE_dlartgp scipy_LAPACKE_dlartgp
#define LAPACKE_ssteqr scipy_LAPACKE_ssteqr
#define LAPACKE_dsteqr scipy_LAPACKE_dsteqr
#define LAPACKE_stgexc scipy_LAPACKE_stgexc
#define LAPACKE_dtgexc scipy_LAPACKE_dtgexc
#define LAPACKE_stgsen scipy_LAPACKE_stgsen
#define LAPACKE_dtgsen scipy_LAPACKE_dtgsen
#define LAPACKE_strevc scipy_LAPACKE_strevc
#define LAPACKE_dtrevc scipy_LAPACKE_dtrevc
#define LAPACKE_strexc scipy_LAPACKE_strexc
#define LAPACKE_dtrexc scipy_LAPACKE_dtrexc
#define LAPACKE_strsen scipy_LAPACKE_strsen
#define LAPACKE_dtrsen scipy_LAPACKE_dtrsen
#define LAPACKE_strtrs scipy_LAPACKE_strtrs
#define LAPACKE_dtrtrs scipy_LAPACKE_dtrtrs
#define LAPACKE_strsen_work scipy_LAPACKE_strsen_work
#define LAPACKE_dtrsen_work scipy_LAPACKE_dtrsen_work
#define LAPACKE_ssyevd scipy_LAPACKE_ssyevd
#define LAPACKE_dsyevd scipy_LAPACKE_dsyevd
#define sgemm_ scipy_sgemm_
#define dgemm_ scipy_dgemm_
#define strsm_ scipy_strsm_
#define dtrsm_ scipy_dtrsm_
#define strsv_ scipy_strsv_
#define dtrsv_ scipy_dtrsv_
#define clartg_ scipy_clartg_
#define zlartg_ scipy_zlartg_

#define PB_LAPACKE_REAL(P, T, SEL2, SEL3)                                                          \
  lapack_int LAPACKE_##P##gees(int layout, char jobvs, char sort, SEL2 select, lapack_int n,      \
                               T* a, lapack_int lda, lapack_int* sdim, T* wr, T* wi, T* vs,       \
                               lapack_int ldvs);                                                  \
  lapack_int LAPACKE_##P##gemqrt(int layout, char side, char trans, lapack_int m, lapack_int n,   \
                                 lapack_int k, lapack_int nb, const T* v, lapack_int ldv,         \
                                 const T* t, lapack_int ldt, T* c, lapack_int ldc);               \
  lapack_int LAPACKE_##P##geqrt(int layout, lapack_int m, lapack_int n, lapack_int nb, T* a,      \
                                lapack_int lda, T* t, lapack_int ldt);                            \
  lapack_int LAPACKE_##P##gesvd(int layout, char jobu, char jobvt, lapack_int m, lapack_int n,    \
                                T* a, lapack_int lda, T* s, T* u, lapack_int ldu, T* vt,          \
                                lapack_int ldvt, T* superb);                                      \
  lapack_int LAPACKE_##P##gges(int layout, char jobvsl, char jobvsr, char sort, SEL3 selctg,      \
                               lapack_int n, T* a, lapack_int lda, T* b, lapack_int ldb,          \
                               lapack_int* sdim, T* alphar, T* alphai, T* beta, T* vsl,           \
                               lapack_int ldvsl, T* vsr, lapack_int ldvsr);                       \
  lapack_int LAPACKE_##P##lartgp(T f, T g, T* cs, T* sn, T* r);                                  \
  lapack_int LAPACKE_##P##steqr(int layout, char compz, lapack_int n, T* d, T* e, T* z,           \
                                lapack_int ldz);                                                  \
  lapack_int LAPACKE_##P##tgexc(int layout, lapack_logical wantq, lapack_logical wantz,           \
                                lapack_int n, T* a, lapack_int lda, T* b, lapack_int ldb, T* q,   \
                                lapack_int ldq, T* z, lapack_int ldz, lapack_int* ifst,           \
                                lapack_int* ilst);                                                \
  lapack_int LAPACKE_##P##tgsen(int layout, lapack_int ijob, lapack_logical wantq,                \
                                lapack_logical wantz, const lapack_logical* select, lapack_int n, \
                                T* a, lapack_int lda, T* b, lapack_int ldb, T* alphar, T* alphai, \
                                T* beta, T* q, lapack_int ldq, T* z, lapack_int ldz,              \
                                lapack_int* m, T* pl, T* pr, T* dif);                             \
  lapack_int LAPACKE_##P##trevc(int layout, char side, char howmny, lapack_logical* select,       \
                                lapack_int n, const T* t, lapack_int ldt, T* vl, lapack_int ldvl, \
                                T* vr, lapack_int ldvr, lapack_int mm, lapack_int* m);            \
  lapack_int LAPACKE_##P##trexc(int layout, char compq, lapack_int n, T* t, lapack_int ldt, T* q, \
                                lapack_int ldq, lapack_int* ifst, lapack_int* ilst);              \
  lapack_int LAPACKE_##P##trsen(int layout, char job, char compq, const lapack_logical* select,   \
                                lapack_int n, T* t, lapack_int ldt, T* q, lapack_int ldq, T* wr,  \
                                T* wi, lapack_int* m, T* s, T* sep);                              \
  lapack_int LAPACKE_##P##trtrs(int layout, char uplo, char trans, char diag, lapack_int n,       \
                                lapack_int nrhs, const T* a, lapack_int lda, T* b,                \
                                lapack_int ldb);                                                  \
  lapack_int LAPACKE_##P##trsen_work(int layout, char job, char compq,                            \
                                     const lapack_logical* select, lapack_int n, T* t,            \
                                     lapack_int ldt, T* q, lapack_int ldq, T* wr, T* wi,          \
                                     lapack_int* m, T* s, T* sep, T* work, lapack_int lwork,      \
                                     lapack_int* iwork, lapack_int liwork);                       \
  lapack_int LAPACKE_##P##syevd(int layout, char jobz, char uplo, lapack_int n, T* a,             \
                                lapack_int lda, T* w);

PB_LAPACKE_REAL(s, float, LAPACK_S_SELECT2, LAPACK_S_SELECT3)
PB_LAPACKE_REAL(d, double, LAPACK_D_SELECT2, LAPACK_D_SELECT3)
#undef PB_LAPACKE_REAL

#ifdef __cplusplus
}
#endif
#endif
