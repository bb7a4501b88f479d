/* pb_mixed_jada.h -- FP32 correction-equation solver for PHIST's block
 * Jacobi-Davidson eigensolver (phist_Dsubspacejada) on the b200 kernel
 * library: the mixed-precision form.
 *
 * The outer Jacobi-Davidson iteration stays PHIST's FP64 code: Rayleigh-Ritz
 * projection, Schur decomposition, orthogonalisation (CholQR/SVQB with the
 * library's compensated reductions when requested) and the residuals.  Only
 * the correction equations
 *
 *     (I - Q Q')(A - sigma_j I)(I - Q Q') t_j = -r_j
 *
 * are solved in FP32: the residual block, the projection block Q and the
 * shifts are rounded to FP32, PHIST's own GMRES correction solver
 * (phist_SjadaCorrectionSolver_run, src/jada/phist_jadaCorrectionSolver_def.hpp:141)
 * runs on an FP32 SELL copy of A with FP32 accumulation in every kernel, and
 * the corrections are widened back to FP64.  A correction only has to point
 * the search space in a useful direction, so its FP32 rounding (about 1e-7
 * relative) does not limit the attainable FP64 residual of the eigenpairs.
 *
 * The hook is PHIST's user-defined inner solver: innerSolvType =
 * phist_USER_LINSOLV with jadaOpts.customSolver / customSolver_run
 * (src/jada/phist_jadaOpts.h:150-179; dispatch at
 * src/jada/phist_jadaCorrectionSolver_def.hpp:166-225).  No PHIST source
 * changes.
 */
#ifndef PB_MIXED_JADA_H
#define PB_MIXED_JADA_H

#include "phist_jadaOpts.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct pb_mixed_jada pb_mixed_jada;

/* Builds the FP32 copy of the FP64 matrix A (phist_DsparseMat_ptr) and an FP32
 * GMRES correction solver configured from *opts (innerSolvBlockSize,
 * innerSolvMaxBas, innerSolvRobust as PHIST reads them; the inner solver type
 * must be GMRES or MINRES).  Only standard problems (B = I) with real shifts
 * are handled; run() answers anything else with -99 (PHIST_NOT_IMPLEMENTED). */
void phist_b200_mixed_jada_create(pb_mixed_jada** me, void const* A, const phist_jadaOpts* opts, int* iflag);

/* The general form: fp32 = 1 solves the correction equations in FP32 (on
 * the FP32 copy of A), fp32 = 0 in FP64 (on A itself); devgmres = 1 uses the
 * library's device-resident GMRES (phist_b200_{D,S}jadaCorrection_gmres:
 * Hessenberg matrix, rotations and every dot product on the GPU, CGS2 as
 * block products, no host synchronisation per step) instead of PHIST's
 * blocked GMRES.  fp32 = 0 always means the device GMRES (PHIST's own FP64
 * GMRES is what subspacejada runs without this hook).  With innerSolvType
 * MINRES the device solver runs MINRES instead
 * (phist_b200_{D,S}jadaCorrection_minres: the Lanczos three-term recurrence
 * of PHIST's blocked MINRES, for symmetric A).  Basis size:
 * innerSolvMaxBas, or innerSolvMaxIters when that is < 0 (PHIST's rule,
 * src/jada/phist_jadaCorrectionSolver_def.hpp:37-38). */
void phist_b200_jada_inner_create(pb_mixed_jada** me, void const* A, const phist_jadaOpts* opts, int fp32,
                                  int devgmres, int* iflag);

/* Points opts at this solver: innerSolvType = phist_USER_LINSOLV,
 * customSolver = me, customSolver_run = the FP32 solve. */
void phist_b200_mixed_jada_install(pb_mixed_jada* me, phist_jadaOpts* opts, int* iflag);

/* Number of correction solves, of systems solved and of systems that did not
 * reach their tolerance since create. */
void phist_b200_mixed_jada_stats(const pb_mixed_jada* me, long* calls, long* systems, long* unconverged, int* iflag);

void phist_b200_mixed_jada_delete(pb_mixed_jada* me, int* iflag);

#ifdef __cplusplus
}
#endif
#endif
