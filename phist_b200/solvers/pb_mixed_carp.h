/* pb_mixed_carp.h -- multi-shift CARP-CG with FP32 sweeps and FP64
 * iterative refinement on the b200 kernel library.
 *
 * Solves (A - sigma_j I) x_j = b_j, one shift and right-hand side per column,
 * to a relative FP64 residual tol:
 *
 *   repeat
 *     r_j = b_j - (A - sigma_j I) x_j             FP64 SpMMV (vadd form)
 *     stop when ||r_j|| <= tol ||b_j|| for all j  FP64 norms
 *     solve (A - sigma_j I) d_j = r_j/||r_j||      PHIST's CARP-CG in FP32,
 *                                                  to innerTol
 *     x_j += ||r_j|| d_j                           FP64
 *
 * The inner solver is PHIST's own carp_cgState (src/krylov/phist_carp_cg_def.hpp)
 * instantiated for float, running on an FP32 SELL copy of A: every Kaczmarz
 * sweep, dot product and update reads and accumulates FP32.  The FP64 residual
 * of the outer loop removes the FP32 rounding of the corrections, so the
 * final relative residual is an FP64 one.
 *
 * Safeguards for shifts where FP32 CG stops converging: every FP32 inner
 * solve is capped (min(maxInnerIter, 1000) iterations at first, halved
 * whenever a correction made a column's FP64 residual larger -- such a
 * correction is taken back and that cap is not reached again -- and doubled
 * after one that cut every corrected residual by 10%), and converged columns
 * and non-finite corrections are not applied.  Where a shifted system is too
 * ill-conditioned for FP32 (two corrections in a row that halve no residual),
 * the remaining corrections are solved with PHIST's FP64 carp_cgState; the
 * loop stops after 3 FP64 corrections in a row that cut no residual by 10%.
 * PB_MIXED_CARP_VERBOSE=1 prints the relative residuals of every refinement
 * step to stderr.
 */
#ifndef PB_MIXED_CARP_H
#define PB_MIXED_CARP_H

#ifdef __cplusplus
extern "C" {
#endif

typedef struct pb_mixed_carp pb_mixed_carp;

/* A: phist_DsparseMat_ptr (kept by reference, must outlive the object);
 * nsys systems with real shifts sigma[nsys]. */
void phist_b200_mixed_carp_create(pb_mixed_carp** me, void const* A, int nsys, const double sigma[], int* iflag);

/* B, X: phist_Dmvec_ptr with nsys columns on A's row map; X holds the start
 * guess on entry.  omega[nsys] relaxation parameters (NULL: 1).  On exit
 * *refinements is the number of FP64 residual corrections; *iflag > 0 counts
 * the systems that did not reach tol within maxRefine corrections. */
void phist_b200_mixed_carp_solve(pb_mixed_carp* me, void const* B, void* X, const double omega[], double tol,
                                 double innerTol, int maxInnerIter, int maxRefine, int* refinements,
                                 int* iflag);

/* corrections of the last solve: inner solves in FP32 and in FP64 */
void phist_b200_mixed_carp_stats(pb_mixed_carp const* me, int* fp32_steps, int* fp64_steps, int* iflag);

void phist_b200_mixed_carp_delete(pb_mixed_carp* me, int* iflag);

#ifdef __cplusplus
}
#endif
#endif
