/*
 * phist_b200_kernels.h -- C ABI of libphist_kernels_b200.so, the B200 kernel
 * library behind PHIST's phist_kernels interface.
 *
 * The entry points are exactly those a PHIST kernel library exports
 * (CMake target phist_kernels_${PHIST_KERNEL_LIB}, CMakeLists.txt:629; the
 * Python binding loads libphist_kernels_<lib>.so with RTLD_GLOBAL,
 * python/phist_kernels.py:13-15).  Each group below cites the PHIST
 * declaration it implements (paths relative to the PHIST source tree).
 * Names expand as in src/tools/phist_gen_d.h:36 (SUBR(x) -> phist_D##x) and
 * src/tools/phist_gen_s.h (phist_S##x).
 *
 * Conventions (src/kernels/phist_kernels_decl.h:47-67):
 *  - every function returns void, *iflag last: input flags on entry, status
 *    on exit (0 ok, >0 warning, <0 error: -1 functional, -44 allocation,
 *    -55 invalid input, -77 exception, -88 bad cast/NULL, -99 not
 *    implemented; src/tools/phist_defs.h:53-71);
 *  - mvecs are row-major (PHIST_MVECS_ROW_MAJOR): element (i,j) of a view
 *    with leading dimension lda sits at val[i*lda+j];
 *  - sdMats are column-major with lda >= nrows;
 *  - handles are opaque pointers; phist_lidx is int32, phist_gidx int64
 *    (src/kernels/builtin/phist_typedefs.h).
 *
 * The library runs on one GPU per process: comm objects describe a single
 * rank (size 1).  Values returned through host arrays (dots, norms) and
 * sdMat results are synchronised before the call returns.
 */
#ifndef PHIST_B200_KERNELS_H
#define PHIST_B200_KERNELS_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef int32_t phist_lidx;
typedef int64_t phist_gidx;

#ifndef PHIST_B200_NO_HANDLE_TYPES
/* opaque handles: src/kernels/phist_void_aliases.h, phist_void_aliases_decl.h */
typedef void* phist_comm_ptr;
typedef const void* phist_const_comm_ptr;
typedef void* phist_map_ptr;
typedef const void* phist_const_map_ptr;
typedef void* phist_context_ptr;
typedef const void* phist_const_context_ptr;
#define PB_HANDLES(P)                                              \
  typedef struct phist_##P##mvec_s phist_##P##mvec;                \
  typedef phist_##P##mvec* phist_##P##mvec_ptr;                    \
  typedef const phist_##P##mvec* phist_##P##const_mvec_ptr;        \
  typedef struct phist_##P##sdMat_s phist_##P##sdMat;              \
  typedef phist_##P##sdMat* phist_##P##sdMat_ptr;                  \
  typedef const phist_##P##sdMat* phist_##P##const_sdMat_ptr;      \
  typedef struct phist_##P##sparseMat_s phist_##P##sparseMat;      \
  typedef phist_##P##sparseMat* phist_##P##sparseMat_ptr;          \
  typedef const phist_##P##sparseMat* phist_##P##const_sparseMat_ptr;
PB_HANDLES(D)
PB_HANDLES(S)
#undef PB_HANDLES
typedef int MPI_Comm_b200_stub; /* MPI_Comm without MPI: phist_mpi_kernels.h */

/* row function: src/kernels/phist_kernels.h (phist_sparseMat_rowFunc) */
typedef int (*phist_sparseMat_rowFunc)(phist_gidx row, phist_lidx* len,
                                       phist_gidx* cols, void* vals, void* arg);
typedef int (*phist_sparseMat_rowFuncConstructor)(void* arg, void** work);
typedef int (*phist_mvec_elemFunc)(phist_gidx row, phist_lidx col, void* val, void* arg);
#endif

/* ---------------------------------------------------------------------------
 * type-independent functions: src/kernels/phist_kernels.h:79-175
 * ------------------------------------------------------------------------- */
void phist_kernels_init(int* argc, char*** argv, int* iflag);          /* :79 */
void phist_kernels_finalize(int* iflag);                               /* :84 */
void phist_comm_create(phist_comm_ptr* comm, int* iflag);              /* :87 */
void phist_comm_delete(phist_comm_ptr comm, int* iflag);               /* :91 */
void phist_comm_get_rank(phist_const_comm_ptr comm, int* rank, int* iflag);
void phist_comm_get_size(phist_const_comm_ptr comm, int* size, int* iflag);
void phist_comm_get_mpi_comm(phist_const_comm_ptr comm, int* mpiComm, int* iflag);
void phist_map_create(phist_map_ptr* map, phist_const_comm_ptr comm,
                      phist_gidx nglob, int* iflag);                   /* :104 */
void phist_map_delete(phist_map_ptr map, int* iflag);
void phist_map_get_comm(phist_const_map_ptr map, phist_const_comm_ptr* comm, int* iflag);
void phist_map_get_local_length(phist_const_map_ptr map, phist_lidx* nloc, int* iflag);
void phist_map_get_global_length(phist_const_map_ptr map, phist_gidx* nglob, int* iflag);
void phist_map_get_ilower(phist_const_map_ptr map, phist_gidx* ilower, int* iflag);
void phist_map_get_iupper(phist_const_map_ptr map, phist_gidx* iupper, int* iflag);
void phist_maps_compatible(phist_const_map_ptr map1, phist_const_map_ptr map2, int* iflag); /* :132 */
void phist_context_create(phist_context_ptr* ctx, phist_const_map_ptr row_map,
                          phist_const_map_ptr col_map, phist_const_map_ptr range_map,
                          phist_const_map_ptr domain_map, int* iflag); /* :154 */
void phist_context_delete(phist_context_ptr vctx, int* iflag);
/* STREAM benchmarks (:167-175): device-memory bandwidth in Gbyte/s */
void phist_bench_stream_load(double* mean_bw, double* max_bw, int* iflag);
void phist_bench_stream_store(double* mean_bw, double* max_bw, int* iflag);
void phist_bench_stream_copy(double* mean_bw, double* max_bw, int* iflag);
void phist_bench_stream_triad(double* mean_bw, double* max_bw, int* iflag);
void phist_kernels_common_init(int* argc, char*** argv, int* iflag);
void phist_kernels_common_finalize(int* iflag);
/* src/tools/phist_tools.h:143 and src/kernels/phist_driver_utils: sizes and
 * library name used by the Python binding (python/phist_kernels.py:46-60) */
const char* phist_kernel_lib(void);
int phist_sizeof_lidx(void);
int phist_sizeof_gidx(void);

/* ---------------------------------------------------------------------------
 * typed functions, declared once per type prefix P with scalar ST (_ST_) and
 * magnitude MT (_MT_): D = double, S = float.
 * ------------------------------------------------------------------------- */
#define PB_DECLARE_TYPED(P, ST, MT)                                                          \
/* src/kernels/phist_kernels_decl.h */                                                       \
void phist_##P##type_avail(int* iflag);                                          /* :79 */   \
void phist_##P##sparseMat_read_mm(phist_##P##sparseMat_ptr* A, phist_const_comm_ptr comm,    \
        const char* filename, int* iflag);                                       /* :98 */   \
void phist_##P##sparseMat_read_mm_with_context(phist_##P##sparseMat_ptr* A,                  \
        phist_const_context_ptr ctx, const char* filename, int* iflag);          /* :110 */  \
void phist_##P##sparseMat_read_hb(phist_##P##sparseMat_ptr* A, phist_const_comm_ptr comm,    \
        const char* filename, int* iflag);                                       /* :102 */  \
void phist_##P##sparseMat_read_bin(phist_##P##sparseMat_ptr* A, phist_const_comm_ptr comm,   \
        const char* filename, int* iflag);                                       /* :106 */  \
void phist_##P##sparseMat_read_hb_with_context(phist_##P##sparseMat_ptr* A,                  \
        phist_const_context_ptr ctx, const char* filename, int* iflag);          /* :114 */  \
void phist_##P##sparseMat_read_bin_with_context(phist_##P##sparseMat_ptr* A,                 \
        phist_const_context_ptr ctx, const char* filename, int* iflag);          /* :118 */  \
void phist_##P##sparseMat_get_row_map(phist_##P##const_sparseMat_ptr A,                      \
        phist_const_map_ptr* map, int* iflag);                                   /* :127 */  \
void phist_##P##sparseMat_get_col_map(phist_##P##const_sparseMat_ptr A,                      \
        phist_const_map_ptr* map, int* iflag);                                   /* :131 */  \
void phist_##P##sparseMat_get_domain_map(phist_##P##const_sparseMat_ptr A,                   \
        phist_const_map_ptr* map, int* iflag);                                   /* :135 */  \
void phist_##P##sparseMat_get_range_map(phist_##P##const_sparseMat_ptr A,                    \
        phist_const_map_ptr* map, int* iflag);                                   /* :139 */  \
void phist_##P##sparseMat_get_context(phist_##P##const_sparseMat_ptr A,                      \
        phist_const_context_ptr* ctx, int* iflag);                               /* :143 */  \
void phist_##P##sparseMat_local_nnz(phist_##P##const_sparseMat_ptr A, int64_t* nnz, int* iflag); \
void phist_##P##sparseMat_global_nnz(phist_##P##const_sparseMat_ptr A, int64_t* nnz, int* iflag); \
void phist_##P##mvec_create(phist_##P##mvec_ptr* V, phist_const_map_ptr map, int nvec,       \
        int* iflag);                                                             /* :166 */  \
void phist_##P##sdMat_create(phist_##P##sdMat_ptr* M, int nrows, int ncols,                  \
        phist_const_comm_ptr comm, int* iflag);                                  /* :178 */  \
void phist_##P##sparseMat_delete(phist_##P##sparseMat_ptr A, int* iflag);        /* :184 */  \
void phist_##P##mvec_delete(phist_##P##mvec_ptr V, int* iflag);                  /* :187 */  \
void phist_##P##sdMat_delete(phist_##P##sdMat_ptr M, int* iflag);                /* :190 */  \
void phist_##P##mvec_get_map(phist_##P##const_mvec_ptr V, phist_const_map_ptr* map, int* iflag); \
void phist_##P##mvec_num_vectors(phist_##P##const_mvec_ptr V, int* nvec, int* iflag);        \
void phist_##P##mvec_get_data(phist_##P##const_mvec_ptr V, ST* data, phist_lidx lda,         \
        int output_row_major, int* iflag);                                       /* :221 */  \
void phist_##P##mvec_extract_view(phist_##P##mvec_ptr V, ST** V_raw, phist_lidx* lda,        \
        int* iflag);                                                             /* :244 */  \
void phist_##P##mvec_extract_const_view(phist_##P##const_mvec_ptr V, const ST** V_raw,       \
        phist_lidx* lda, int* iflag);                                            /* :248 */  \
void phist_##P##sdMat_get_nrows(phist_##P##const_sdMat_ptr M, int* nrows, int* iflag);       \
void phist_##P##sdMat_get_ncols(phist_##P##const_sdMat_ptr M, int* ncols, int* iflag);       \
void phist_##P##sdMat_extract_view(phist_##P##sdMat_ptr M, ST** M_raw, phist_lidx* lda,      \
        int* iflag);                                                             /* :266 */  \
void phist_##P##sdMat_extract_const_view(phist_##P##const_sdMat_ptr M, const ST** M_raw,     \
        phist_lidx* lda, int* iflag);                                            /* :270 */  \
void phist_##P##sdMat_extract_error(phist_##P##sdMat_ptr M, ST** MC_raw, int* iflag); /* :284 */ \
void phist_##P##mvec_to_device(phist_##P##mvec_ptr V, int* iflag);               /* :296 */  \
void phist_##P##mvec_from_device(phist_##P##mvec_ptr V, int* iflag);             /* :299 */  \
void phist_##P##sdMat_to_device(phist_##P##sdMat_ptr M, int* iflag);             /* :309 */  \
void phist_##P##sdMat_from_device(phist_##P##sdMat_ptr M, int* iflag);           /* :312 */  \
void phist_##P##mvec_write_bin(phist_##P##const_mvec_ptr V, const char* fn, int* iflag);     \
void phist_##P##mvec_read_bin(phist_##P##mvec_ptr V, const char* fn, int* iflag);            \
void phist_##P##sdMat_write_bin(phist_##P##const_sdMat_ptr M, const char* fn, int* iflag);   \
void phist_##P##sdMat_read_bin(phist_##P##sdMat_ptr M, const char* fn, int* iflag);          \
void phist_##P##mvec_to_mvec(phist_##P##const_mvec_ptr v_in, phist_##P##mvec_ptr v_out,      \
        int* iflag);                                                             /* :343 */  \
void phist_##P##mvec_view_block(phist_##P##mvec_ptr V, phist_##P##mvec_ptr* Vblock,          \
        int jmin, int jmax, int* iflag);                                         /* :368 */  \
void phist_##P##mvec_get_block(phist_##P##const_mvec_ptr V, phist_##P##mvec_ptr Vblock,      \
        int jmin, int jmax, int* iflag);                                         /* :378 */  \
void phist_##P##mvec_set_block(phist_##P##mvec_ptr V, phist_##P##const_mvec_ptr Vblock,      \
        int jmin, int jmax, int* iflag);                                         /* :384 */  \
/* V(:, off_i : off_i + n_i - 1) = W[i] for the blocks side by side, and back */              \
void phist_##P##mvec_gather_mvecs(phist_##P##mvec_ptr V, phist_##P##const_mvec_ptr W[],         \
        int nblocks, int* iflag);                                                /* :736 */   \
void phist_##P##mvec_scatter_mvecs(phist_##P##const_mvec_ptr V, phist_##P##mvec_ptr W[],        \
        int nblocks, int* iflag);                                                /* :737 */   \
void phist_##P##sdMat_view_block(phist_##P##sdMat_ptr M, phist_##P##sdMat_ptr* Mblock,       \
        int imin, int imax, int jmin, int jmax, int* iflag);                     /* :402 */  \
void phist_##P##sdMat_get_block(phist_##P##const_sdMat_ptr M, phist_##P##sdMat_ptr Mblock,   \
        int imin, int imax, int jmin, int jmax, int* iflag);                     /* :412 */  \
void phist_##P##sdMat_set_block(phist_##P##sdMat_ptr M, phist_##P##const_sdMat_ptr Mblock,   \
        int imin, int imax, int jmin, int jmax, int* iflag);                     /* :418 */  \
void phist_##P##sdMat_set_data(phist_##P##sdMat_ptr M, const ST* data, phist_lidx lda,       \
        int input_row_major, int* iflag);                                        /* :428 */  \
void phist_##P##sdMat_get_data(phist_##P##const_sdMat_ptr M, ST* data, phist_lidx lda,      \
        int output_row_major, int* iflag);                                       /* :438 */  \
void phist_##P##mvec_put_value(phist_##P##mvec_ptr V, ST value, int* iflag);     /* :448 */  \
void phist_##P##mvec_put_func(phist_##P##mvec_ptr V, phist_mvec_elemFunc f, void* arg,       \
        int* iflag);                                                             /* :455 */  \
void phist_##P##mvec_random(phist_##P##mvec_ptr V, int* iflag);                  /* :459 */  \
void phist_##P##sdMat_random(phist_##P##sdMat_ptr M, int* iflag);                /* :467 */  \
void phist_##P##sdMat_put_value(phist_##P##sdMat_ptr M, ST value, int* iflag);   /* :470 */  \
void phist_##P##sdMat_identity(phist_##P##sdMat_ptr M, int* iflag);              /* :478 */  \
void phist_##P##mvec_print(phist_##P##const_mvec_ptr V, int* iflag);             /* :483 */  \
void phist_##P##sdMat_print(phist_##P##const_sdMat_ptr M, int* iflag);           /* :486 */  \
void phist_##P##mvec_norm2(phist_##P##const_mvec_ptr V, MT* vnrm, int* iflag);   /* :496 */  \
void phist_##P##mvec_normalize(phist_##P##mvec_ptr V, MT* vnrm, int* iflag);     /* :504 */  \
void phist_##P##mvec_scale(phist_##P##mvec_ptr V, ST scalar, int* iflag);        /* :508 */  \
void phist_##P##mvec_vscale(phist_##P##mvec_ptr V, const ST* scalar, int* iflag); /* :512 */ \
void phist_##P##mvec_add_mvec(ST alpha, phist_##P##const_mvec_ptr X, ST beta,                \
        phist_##P##mvec_ptr Y, int* iflag);                                      /* :522 */  \
void phist_##P##mvec_vadd_mvec(const ST alpha[], phist_##P##const_mvec_ptr X, ST beta,       \
        phist_##P##mvec_ptr Y, int* iflag);                                      /* :527 */  \
void phist_##P##mvec_times_mvec_elemwise(ST alpha, phist_##P##const_mvec_ptr V,              \
        phist_##P##mvec_ptr W, int* iflag);                                      /* :544 */  \
void phist_##P##mvec_dot_mvec(phist_##P##const_mvec_ptr V, phist_##P##const_mvec_ptr W,      \
        ST* vw, int* iflag);                                                     /* :548 */  \
void phist_##P##mvecT_times_mvec(ST alpha, phist_##P##const_mvec_ptr V,                      \
        phist_##P##const_mvec_ptr W, ST beta, phist_##P##sdMat_ptr C, int* iflag); /* :557 */\
void phist_##P##mvec_times_sdMat(ST alpha, phist_##P##const_mvec_ptr V,                      \
        phist_##P##const_sdMat_ptr C, ST beta, phist_##P##mvec_ptr W, int* iflag); /* :565 */\
void phist_##P##mvec_times_sdMat_inplace(phist_##P##mvec_ptr V, phist_##P##const_sdMat_ptr M, \
        int* iflag);                                                             /* :577 */  \
void phist_##P##mvec_times_sdMat_add_mvec_times_sdMat(phist_##P##const_mvec_ptr V,           \
        phist_##P##const_sdMat_ptr C, phist_##P##mvec_ptr W,                                 \
        phist_##P##const_sdMat_ptr D, int* iflag);                               /* :585 */  \
void phist_##P##sdMat_add_sdMat(ST alpha, phist_##P##const_sdMat_ptr A, ST beta,             \
        phist_##P##sdMat_ptr B, int* iflag);                                     /* :597 */  \
void phist_##P##sdMatT_add_sdMat(ST alpha, phist_##P##const_sdMat_ptr A, ST beta,            \
        phist_##P##sdMat_ptr B, int* iflag);                                     /* :602 */  \
void phist_##P##sdMat_times_sdMat(ST alpha, phist_##P##const_sdMat_ptr V,                    \
        phist_##P##const_sdMat_ptr W, ST beta, phist_##P##sdMat_ptr C, int* iflag); /* :612 */\
void phist_##P##sdMatT_times_sdMat(ST alpha, phist_##P##const_sdMat_ptr V,                   \
        phist_##P##const_sdMat_ptr W, ST beta, phist_##P##sdMat_ptr C, int* iflag); /* :622 */\
void phist_##P##sdMat_times_sdMatT(ST alpha, phist_##P##const_sdMat_ptr V,                   \
        phist_##P##const_sdMat_ptr W, ST beta, phist_##P##sdMat_ptr C, int* iflag); /* :632 */\
void phist_##P##sparseMat_times_mvec_communicate(phist_##P##const_sparseMat_ptr A,           \
        phist_##P##const_mvec_ptr x, int* iflag);                                /* :644 */  \
void phist_##P##sparseMat_times_mvec(ST alpha, phist_##P##const_sparseMat_ptr A,             \
        phist_##P##const_mvec_ptr x, ST beta, phist_##P##mvec_ptr y, int* iflag); /* :651 */ \
void phist_##P##sparseMatT_times_mvec(ST alpha, phist_##P##const_sparseMat_ptr A,            \
        phist_##P##const_mvec_ptr x, ST beta, phist_##P##mvec_ptr y, int* iflag); /* :659 */ \
void phist_##P##sparseMat_times_mvec_add_mvec(ST alpha, phist_##P##const_sparseMat_ptr A,    \
        ST shift, phist_##P##const_mvec_ptr x, ST beta, phist_##P##mvec_ptr y,               \
        int* iflag);                                                             /* :663 */  \
void phist_##P##sparseMat_times_mvec_vadd_mvec(ST alpha, phist_##P##const_sparseMat_ptr A,   \
        const ST shifts[], phist_##P##const_mvec_ptr x, ST beta, phist_##P##mvec_ptr y,      \
        int* iflag);                                                             /* :667 */  \
void phist_##P##mvec_QR(phist_##P##mvec_ptr V, phist_##P##sdMat_ptr R, int* iflag); /* :686 */\
void phist_##P##sparseMat_create_fromRowFunc(phist_##P##sparseMat_ptr* A,                    \
        phist_const_comm_ptr comm, phist_gidx nrows, phist_gidx ncols, phist_lidx maxnne,    \
        phist_sparseMat_rowFunc rowFunPtr, void* last_arg, int* iflag);          /* :700 */  \
void phist_##P##sparseMat_create_fromRowFuncAndContext(phist_##P##sparseMat_ptr* A,          \
        phist_const_context_ptr ctx, phist_lidx maxnne, phist_sparseMat_rowFunc rowFunPtr,   \
        void* last_arg, int* iflag);                                             /* :708 */  \
void phist_##P##sparseMat_create_fromRowFuncWithConstructor(phist_##P##sparseMat_ptr* A,     \
        phist_const_comm_ptr comm, phist_gidx nrows, phist_gidx ncols, phist_lidx maxnne,    \
        phist_sparseMat_rowFunc rowFunPtr, phist_sparseMat_rowFuncConstructor ctor,          \
        void* last_arg, int* iflag);                                             /* :717 */  \
void phist_##P##sparseMat_create_fromRowFuncWithConstructorAndContext(                       \
        phist_##P##sparseMat_ptr* A, phist_const_context_ptr ctx, phist_lidx maxnne,         \
        phist_sparseMat_rowFunc rowFunPtr, phist_sparseMat_rowFuncConstructor ctor,          \
        void* last_arg, int* iflag);                                             /* :728 */  \
/* src/kernels/phist_kernels_common_decl.h */                                                \
void phist_##P##sparseMat_global_nrows(phist_##P##sparseMat_ptr A, phist_gidx* s, int* iflag); /* :29 */ \
void phist_##P##sparseMat_global_ncols(phist_##P##sparseMat_ptr A, phist_gidx* s, int* iflag); /* :32 */ \
void phist_##P##mvec_my_length(phist_##P##const_mvec_ptr V, phist_lidx* len, int* iflag); /* :40 */ \
void phist_##P##mvec_global_length(phist_##P##const_mvec_ptr V, phist_gidx* len, int* iflag);  \
void phist_##P##mvec_get_comm(phist_##P##const_mvec_ptr V, phist_const_comm_ptr* comm, int* iflag); \
void phist_##P##mvec_clone_shape(phist_##P##mvec_ptr* V, phist_##P##const_mvec_ptr V_in,     \
        int* iflag);                                                             /* :61 */   \
void phist_##P##mvec_set_data(phist_##P##mvec_ptr V, const ST* data, phist_lidx lda,         \
        int input_row_major, int* iflag);                                        /* :75 */   \
/* src/kernels/phist_kernels_fused_decl.h */                                                 \
void phist_##P##fused_spmv_pair(ST alpha, const ST shifts1[], phist_##P##const_sparseMat_ptr A1, \
        const ST shifts2[], phist_##P##const_sparseMat_ptr A2, phist_##P##const_mvec_ptr X,  \
        ST beta, phist_##P##mvec_ptr Y, int* iflag);                             /* :45 */   \
void phist_##P##fused_spmv_mvdot(ST alpha, phist_##P##const_sparseMat_ptr A,                 \
        phist_##P##const_mvec_ptr V, ST beta, phist_##P##mvec_ptr W, ST* WdotW, ST* VdotW,   \
        int* iflag);                                                             /* :57 */   \
void phist_##P##fused_spmv_mvTmv(ST alpha, phist_##P##const_sparseMat_ptr A,                 \
        phist_##P##const_mvec_ptr V, ST beta, phist_##P##mvec_ptr W,                         \
        phist_##P##sdMat_ptr WtW, phist_##P##sdMat_ptr VtW, int* iflag);         /* :68 */   \
void phist_##P##fused_spmv_mvdot_mvadd(ST alpha, phist_##P##const_sparseMat_ptr A,           \
        phist_##P##const_mvec_ptr V, ST beta, phist_##P##mvec_ptr W, ST gamma, ST delta,     \
        phist_##P##mvec_ptr U, ST* WdotW, ST* VdotW, int* iflag);                /* :77 */   \
void phist_##P##fused_mvsdi_mvTmv(ST alpha, phist_##P##const_mvec_ptr V,                     \
        phist_##P##mvec_ptr W, phist_##P##const_sdMat_ptr C, ST beta,                        \
        phist_##P##sdMat_ptr D, int* iflag);                                     /* :84 */   \
void phist_##P##fused_mvsd_mvTmv(ST alpha, phist_##P##const_mvec_ptr V,                      \
        phist_##P##const_sdMat_ptr C, ST beta, phist_##P##mvec_ptr W,                        \
        phist_##P##sdMat_ptr WtW, int* iflag);                                   /* :92 */   \
/* src/kernels/phist_kernels_carp_decl.h */                                                  \
void phist_##P##carp_setup(phist_##P##const_sparseMat_ptr A, int numShifts,                  \
        const ST sigma[], void** work, int* iflag);                              /* :35 */   \
void phist_##P##carp_sweep(phist_##P##const_sparseMat_ptr A, const ST sigma[],               \
        phist_##P##const_mvec_ptr Rhs, phist_##P##mvec_ptr X, void* const work,              \
        const MT* omega, int* iflag);                                            /* :44 */   \
void phist_##P##carp_sweep_aug(phist_##P##const_sparseMat_ptr A, const ST sigma[],           \
        phist_##P##const_mvec_ptr Q, phist_##P##const_mvec_ptr Rhs, phist_##P##mvec_ptr X,   \
        phist_##P##sdMat_ptr q, void* const work, const MT* omega, int* iflag);  /* :58 */   \
void phist_##P##carp_setup_rc(phist_##P##const_sparseMat_ptr A, int numShifts,               \
        const MT sigma_r[], const MT sigma_i[], void** work, int* iflag);        /* :74 */   \
void phist_##P##carp_sweep_rc(phist_##P##const_sparseMat_ptr A, const MT sigma_r[],          \
        const MT sigma_i[], phist_##P##const_mvec_ptr Rhs, phist_##P##mvec_ptr X_r,          \
        phist_##P##mvec_ptr X_i, void* const work, const MT* omega, int* iflag); /* :80 */   \
void phist_##P##carp_sweep_aug_rc(phist_##P##const_sparseMat_ptr A, const MT sigma_r[],      \
        const MT sigma_i[], phist_##P##const_mvec_ptr Q, phist_##P##const_mvec_ptr Rhs,      \
        phist_##P##mvec_ptr X_r, phist_##P##mvec_ptr X_i, phist_##P##sdMat_ptr q_r,          \
        phist_##P##sdMat_ptr q_i, void* const work, const MT* omega, int* iflag); /* :90 */  \
void phist_##P##carp_destroy(phist_##P##const_sparseMat_ptr A, void* work, int* iflag); /* :102 */ \
/* src/kernels/phist_mpi_kernels_decl.h (one rank: no-op / not implemented) */               \
void phist_##P##sdMat_sync_values(phist_##P##sdMat_ptr V, phist_const_comm_ptr comm,         \
        int* iflag);                                                             /* :29 */   \
/* ---- library extensions (no counterpart in PHIST; prefixed phist_b200_ or     */         \
/* ---- documented here) -------------------------------------------------------- */        \
/* build a sparseMat from host CRS arrays (0-based, int64 row offsets, int32      */         \
/* columns); same result as sparseMat_create_fromRowFunc with a row function    */          \
/* that returns these rows.  iflag input: PHIST_SPARSEMAT_* flags.              */          \
void phist_b200_##P##sparseMat_create_fromCRS(phist_##P##sparseMat_ptr* A,                   \
        phist_const_comm_ptr comm, phist_gidx nrows, phist_gidx ncols,                       \
        const int64_t* row_ptr, const int32_t* col, const ST* val, int* iflag);              \
/* SELL-C-sigma layout facts of A; perm (may be NULL) receives nrows entries,    */         \
/* perm[sell_row] = original row.                                                */         \
void phist_b200_##P##sparseMat_sell_info(phist_##P##const_sparseMat_ptr A, int* C,           \
        int64_t* sigma, int64_t* nchunks, int64_t* nnz_padded, int32_t* perm, int* iflag);   \
/* raw device pointers of an mvec / sdMat view (element (0,0)) and its lda       */         \
void phist_b200_##P##mvec_device_view(phist_##P##mvec_ptr V, ST** d_ptr, phist_lidx* lda,    \
        int* iflag);                                                                         \
/* row order of the CARP sweep set up by carp_setup: the forward sweep equals   */          \
/* the sequential Kaczmarz sweep over `rows`, the backward sweep the one over   */          \
/* its reverse; rows[color_ptr[k] .. color_ptr[k+1]) is a distance-2            */          \
/* independent set (ncolors sets, color_ptr has ncolors+1 entries; pass NULL    */          \
/* for outputs that are not wanted)                                              */          \
void phist_b200_##P##carp_color_order(void* const work, int32_t* rows, int* ncolors,         \
        int64_t* color_ptr, int* iflag);

PB_DECLARE_TYPED(D, double, double)
PB_DECLARE_TYPED(S, float, float)

/* mixed precision helpers (library extensions, no counterpart in PHIST):
 * copy a double mvec into a float mvec of the same shape and back, and build
 * an FP32 copy of a double sparseMat with the identical SELL layout. */
void phist_b200_mvec_DtoS(phist_Dconst_mvec_ptr X, phist_Smvec_ptr Y, int* iflag);
void phist_b200_mvec_StoD(phist_Sconst_mvec_ptr X, phist_Dmvec_ptr Y, int* iflag);
void phist_b200_sparseMat_DtoS(phist_Dconst_sparseMat_ptr A, phist_SsparseMat_ptr* As, int* iflag);

/* synthetic test problems as row functions (library extensions; the
 * counterpart of PHIST's driver utility create_matrix with problem strings,
 * src/kernels/phist_driver_utils_def.h:232-470).  Problem strings:
 *   "LAPLACE3D-<L>"                     7-point Laplacian on L^3, Dirichlet
 *   "LAPDIAG3D-<L>-S<seed>"             the same + uniform[0,1] diagonal
 *   "ANDERSON3D-<L>-S<seed>[-W<w>]"     periodic, hopping -1, on-site U[-w/2,w/2]
 *   "HONEYCOMB-<Lx>[x<Ly>]-S<seed>[-W<w>]"  2 sites/cell, periodic, on-site U[-w/2,w/2]
 * *iflag on input: PHIST_SPARSEMAT_* flags. */
void phist_b200_Dcreate_problem(phist_DsparseMat_ptr* A, phist_const_comm_ptr comm,
                                const char* problem, int* iflag);
void phist_b200_Screate_problem(phist_SsparseMat_ptr* A, phist_const_comm_ptr comm,
                                const char* problem, int* iflag);
/* row function and its argument for a problem string: returns a malloc'ed
 * argument (release with free) and the row count / max row length */
void* phist_b200_problem_create(const char* problem, int single, int64_t* nrows, int32_t* maxnne);
int phist_b200_problem_rowfunc(phist_gidx row, phist_lidx* len, phist_gidx* cols, void* vals, void* arg);

/* No counterpart in PHIST.  C = alpha*V'W + beta*C (as phist_DmvecT_times_mvec)
 * on raw DEVICE pointers, for callers that cannot allocate device memory
 * (a host that fixes the device-memory budget at start-up and owns every later
 * allocation, or that forbids cudaMalloc after initialisation).  It allocates
 * nothing: its scratch is a fixed 4 MiB file-scope device array.
 * V: n x m row-major (ldv >= m), W: n x k row-major (ldw >= k), C: m x k
 * column-major (ldc >= m); 1 <= m, k <= 64, larger widths give *iflag = -55.
 * stream: a cudaStream_t (NULL = legacy default stream).  The call is
 * asynchronous on that stream.  The first call on a device does a one-time
 * cudaGetSymbolAddress set-up; make it before any stream capture.  All calls
 * share the scratch array: calls that overlap on the GPU race. */
void phist_b200_DmvecT_times_mvec_noalloc(int64_t n, int m, int k, double alpha,
                                          const double* V, int64_t ldv,
                                          const double* W, int64_t ldw, double beta,
                                          double* C, int64_t ldc, void* stream, int* iflag);

/* Batched multi-shift CARP-CG (library extension; the solver behind PHIST's
 * carp_cg driver, drivers/carp_cg.c:286-320, with the CGMN recurrence of
 * src/krylov/phist_carp_cg_def.hpp:440-690 run on the GPU).  Solves
 * (A - sigma_j I) x_j = b_j for the nsys columns of B (n x nsys) into X
 * (n x nsys) through `block` (1..32) slots, or, for block <= 0, the slot
 * count phist_b200_DcarpCG_tune_block picks: each slot iterates one system;
 * every checkEvery iterations the explicit FP64 residuals are measured, and
 * a system that reached ||b_j - (A - sigma_j I) x_j|| <= tol ||b_j|| (or
 * maxIter iterations) leaves its slot to the next queued system.  All CG
 * scalars live on the device; an iteration synchronises with the host only
 * at the checks.  mixed = 1: FP32 sweeps and FP32 CG on an FP32 copy of A,
 * inside per-slot FP64 iterative refinement (inner relative tolerance
 * innerTol, <= 0 selects 1e-5).  On exit iters[j] holds the CG iterations
 * spent on system j and relres[j] its final FP64 relative residual;
 * *iflag >= 0 is the number of systems that did not reach tol. */
void phist_b200_DcarpCG_batch(phist_Dconst_sparseMat_ptr A, int nsys, const double sigma[],
                              phist_Dconst_mvec_ptr B, phist_Dmvec_ptr X, int block, double tol,
                              int maxIter, int checkEvery, int mixed, double innerTol, int iters[],
                              double relres[], int* iflag);
/* slot count for phist_b200_DcarpCG_batch: the w in {1, 2, 4, 8, 16, 32},
 * w <= max(nsys, 1), with the most system-iterations per second w / t(w),
 * t(w) the device time of one iteration (colour sweep and fused CG updates,
 * median of reps after a warm-up; FP32 when mixed).  iter_us[6] (may be
 * NULL) receives t(1), t(2), ... t(32) in microseconds, 0 where not tried. */
void phist_b200_DcarpCG_tune_block(phist_Dconst_sparseMat_ptr A, int nsys, int mixed, int reps, int* block,
                                   double iter_us[], int* iflag);

/* Device-resident GMRES for the Jacobi-Davidson correction equations
 *   (I - Q Q')(A - sigma_j I) t_j = res(:, resIndex[j]),  j < k <= 32
 * (the task of PHIST's jadaCorrectionSolver_run with GMRES,
 * src/jada/phist_jadaCorrectionSolver_def.hpp:141-583).  Q (n x nq, may be
 * NULL) has orthonormal columns; resIndex may be NULL (identity).  x_0 = 0;
 * restarted after maxBas steps (<= 63), at most maxIter steps; system j is
 * converged when its GMRES residual is below 1000 eps absolute or tol[j]
 * relative to ||res_j|| (phist_blockedgmres_def.hpp:604-606).  The
 * Hessenberg matrices, rotations and all dot products stay on the device;
 * Gram-Schmidt is classical, done twice, as block products.  t (n x k)
 * receives the solutions scaled to unit norm (as PHIST returns them);
 * *iflag >= 0 is the number of systems that did not converge.  The S form
 * runs in FP32 (the small dense part in FP64). */
void phist_b200_DjadaCorrection_gmres(phist_Dconst_sparseMat_ptr A, phist_Dconst_mvec_ptr Q,
                                      phist_Dconst_mvec_ptr res, const int resIndex[], int k,
                                      const double sigma[], const double tol[], int maxIter, int maxBas,
                                      phist_Dmvec_ptr t, int* iflag);
void phist_b200_SjadaCorrection_gmres(phist_Sconst_sparseMat_ptr A, phist_Sconst_mvec_ptr Q,
                                      phist_Sconst_mvec_ptr res, const int resIndex[], int k,
                                      const double sigma[], const double tol[], int maxIter, int maxBas,
                                      phist_Smvec_ptr t, int* iflag);
/* The same solve with PHIST's blocked MINRES step (the task of
 * jadaCorrectionSolver_run with MINRES, phist_jadaCorrectionSolver_def.hpp:
 * 499-503; src/krylov/phist_blockedminres_def.hpp): the Lanczos three-term
 * recurrence alpha = V_j'W, W -= alpha V_j + beta V_{j-1} in place of
 * Gram-Schmidt, so every step costs the same; rotations, least squares,
 * restarts and the returned t as above; converged below 100 eps absolute or
 * tol[j] relative.  For symmetric A (real shifts), as PHIST's MINRES. */
void phist_b200_DjadaCorrection_minres(phist_Dconst_sparseMat_ptr A, phist_Dconst_mvec_ptr Q,
                                       phist_Dconst_mvec_ptr res, const int resIndex[], int k,
                                       const double sigma[], const double tol[], int maxIter, int maxBas,
                                       phist_Dmvec_ptr t, int* iflag);
void phist_b200_SjadaCorrection_minres(phist_Sconst_sparseMat_ptr A, phist_Sconst_mvec_ptr Q,
                                       phist_Sconst_mvec_ptr res, const int resIndex[], int k,
                                       const double sigma[], const double tol[], int maxIter, int maxBas,
                                       phist_Smvec_ptr t, int* iflag);

/* runtime controls and statistics (library extensions) */
/* SELL chunk height C (1..32, power of two) and the sigma window used when a
 * matrix is built with PHIST_SPARSEMAT_PERM_LOCAL (<=1: no sorting) */
void phist_b200_set_sell_params(int C, int64_t sigma, int* iflag);
/* SpMMV launch shape (autotuning control): threads per matrix row for block
 * width nvec (1,2,4,8,16,32; allowed 1:1, 2:1, 4:1|2, 8:1|2|4, 16:2|4|8,
 * 32:4|8|16) and, when unroll >= 0, whether the fully unrolled kernel for
 * matrices whose rows have at most 8 entries may be used */
void phist_b200_set_spmv_config(int nvec, int tpr, int unroll, int* iflag);
/* block widths >= min_nvec (8..32) use the SpMMV kernel that stages the
 * gathered X rows in shared memory (values above 32 disable it) */
void phist_b200_set_spmv_staged(int min_nvec, int* iflag);
/* SpMMV on matrices whose rows have at most 8 entries: on = 1 (the default;
 * environment PHIST_B200_SPMV_PREFETCH) runs a resident grid that copies the
 * next tile's matrix entries into shared memory while the current tile
 * gathers its X rows; on = 0 runs one tile per thread block.  Results are
 * bitwise the same. */
void phist_b200_set_spmv_prefetch(int on, int* iflag);
/* batched CARP-CG: replay each iteration as a recorded CUDA graph (1, the
 * default; environment PHIST_B200_GRAPHS) or launch its kernels one by one
 * (0); both give bitwise identical results */
void phist_b200_set_graphs(int on, int* iflag);
/* kernel-path switches, all on by default (1) and each also read from the
 * environment at init: "tma" (TMA-staged block products, PHIST_B200_TMA),
 * "dmma" (FP64 tensor-core tiles, PHIST_B200_DMMA), "graphs" (as
 * phist_b200_set_graphs, PHIST_B200_GRAPHS), "carp_blocks" (CARP sweeps
 * over a block colouring with X staged in shared memory, else one launch per
 * row colour class; PHIST_B200_CARP_BLOCKS; applies to CARP work set up
 * afterwards), "spmv_v256" (SpMMV gathers X row segments of 32 bytes or
 * more with 256-bit loads when rows start on 32-byte boundaries,
 * PHIST_B200_SPMV_V256).  "graphs" and "spmv_v256" never change a result;
 * tma/dmma change the summation order of the block products; carp_blocks
 * changes the row order of the sweep (phist_b200_Dcarp_color_order reports
 * it).
 * Unknown names: PHIST_INVALID_INPUT. */
void phist_b200_set_option(const char* name, int value, int* iflag);
/* SpMMV autotuner (no PHIST counterpart: GHOST fixes C = 32 on CUDA and sigma
 * by flag, src/kernels/ghost/kernels.cpp:69-134).  Times Y = A X on A itself
 * for each block width in widths[nw] (1..32) over the SELL layouts C in
 * {32, 16, 8} x sigma in {1, 4C, 1024} (sigma 1 only if all rows have the
 * same length) and the SpMMV kernel variants of each width (threads per
 * row, fully unrolled short-row kernel, shared-memory staged kernel), each
 * the median of reps device-timed calls after an L2 flush.  A is left in the
 * layout with the least total time, with the fastest variant per width;
 * best_us[nw] (may be NULL) receives each width's time there.  Results of
 * every SpMMV are bitwise the same in every layout and variant; vectors keep
 * their row order. */
void phist_b200_DsparseMat_autotune(phist_DsparseMat_ptr A, int nw, const int* widths, int reps,
                                    double* best_us, int* iflag);
void phist_b200_SsparseMat_autotune(phist_SsparseMat_ptr A, int nw, const int* widths, int reps,
                                    double* best_us, int* iflag);
/* the configuration in effect: SELL chunk height and sorting window, and per
 * width class 1, 2, 4, 8, 16, 32 (arrays of 6, each may be NULL): threads
 * per row, unrolled short-row kernel (0/1), staged kernel (0/1) */
void phist_b200_DsparseMat_get_tuning(phist_Dconst_sparseMat_ptr A, int* C, int64_t* sigma, int* tpr,
                                      int* unroll, int* staged, int* iflag);
void phist_b200_SsparseMat_get_tuning(phist_Sconst_sparseMat_ptr A, int* C, int64_t* sigma, int* tpr,
                                      int* unroll, int* staged, int* iflag);
/* wait for all work this library enqueued */
void phist_b200_synchronize(int* iflag);
/* failure-path check of the bounded device waits: runs one kernel whose
 * mbarrier wait cannot complete; the wait gives up after about one second,
 * stores its code in the device error word and the kernel returns, so the
 * call ends with PHIST_FUNCTIONAL_ERROR (-1) and a message, as a real
 * timed-out copy would; the word is cleared and the context stays usable */
void phist_b200_selftest_bounded_wait(int* iflag);
/* Every host thread that calls the library works on its own lane: a CUDA
 * stream with its own scratch, counters, result mailbox and device-memory
 * cache, so solves driven from several threads overlap on the GPU.  Objects
 * are meant to be used by the thread that created them (read-only matrices
 * may be shared).  phist_b200_synchronize drains the calling thread's lane;
 * phist_b200_get_stream returns it.  Number of lanes created so far: */
void phist_b200_lane_count(int* nlanes, int* iflag);
/* free and total device memory in bytes (admission control of a server) */
void phist_b200_device_memory(uint64_t* free_bytes, uint64_t* total_bytes, int* iflag);
/* number of kernel launches this library has issued since init */
void phist_b200_launch_count(uint64_t* count, int* iflag);
/* the CUDA stream all kernels are enqueued on (cudaStream_t) */
void phist_b200_get_stream(void** stream, int* iflag);

#ifdef __cplusplus
}
#endif
#endif /* PHIST_B200_KERNELS_H */
