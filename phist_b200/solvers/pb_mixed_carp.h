/* pb_mixed_carp.h -- multi-shift CARP-CG with FP32 sweeps and FP64
 * iterative refinement on the b200 kernel library.
 *
 * Solves (A - sigma_j I) x_j = b_j, one shift and right-hand side per column,
 * to a relative FP64 residual tol:
 *
 *   repeat
 *     r_j = b_j - (A - sigma_j I) x_j             FP64 SpMMV (vadd form)
 *     stop when ||r_j|| <= tol ||b_j|| for all j  FP64 norms
 *     solve (A - sigma_j I) d_j = r_j to innerTol  PHIST's CARP-CG in FP32
 *     x_j += d_j                                   FP64
 *
 * The inner solver is PHIST's own carp_cgState (src/krylov/phist_carp_cg_def.hpp)
 * instantiated for float, running on an FP32 SELL copy of A: every Kaczmarz
 * sweep, dot product and update reads and accumulates FP32.  The FP64 residual
 * of the outer loop removes the FP32 rounding of the corrections, so the
 * final relative residual is an FP64 one.
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

void phist_b200_mixed_carp_delete(pb_mixed_carp* me, int* iflag);

#ifdef __cplusplus
}
#endif
#endif
