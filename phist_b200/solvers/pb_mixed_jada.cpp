// pb_mixed_jada.cpp -- FP32 correction-equation solver behind PHIST's
// user-defined inner-solver hook (declarations and the numerical argument in
// pb_mixed_jada.h).
//
// Per correction solve (one call of customSolver_run):
//   1. Qtil (n x nq, FP64) -> Qs, res (n x nres, FP64) -> Rs    [DtoS kernels]
//   2. phist_SjadaCorrectionSolver_run on the FP32 operator A32 - sigma_j I,
//      projected against Qs: PHIST's blocked GMRES, every SpMMV, dot, axpy
//      and orthogonalisation step an FP32 kernel of the b200 library
//   3. Ts (n x k, FP32) -> t (FP64)                             [StoD kernel]
// The FP32 blocks live in capacity-sized work mvecs that are created once
// and viewed at the width of each call.
#include <cstdio>
#include <cstring>
#include <new>
#include <vector>

#include "phist_config.h"
#include "phist_kernels.h"
#include "phist_core.h"
#include "phist_jada.h"
#include "pb_mixed_jada.h"

extern "C" {
void phist_b200_DjadaCorrection_gmres(phist_Dconst_sparseMat_ptr A, phist_Dconst_mvec_ptr Q,
                                      phist_Dconst_mvec_ptr res, const int resIndex[], int k, const double sigma[],
                                      const double tol[], int maxIter, int maxBas, phist_Dmvec_ptr t, int* iflag);
void phist_b200_SjadaCorrection_gmres(phist_Sconst_sparseMat_ptr A, phist_Sconst_mvec_ptr Q,
                                      phist_Sconst_mvec_ptr res, const int resIndex[], int k, const double sigma[],
                                      const double tol[], int maxIter, int maxBas, phist_Smvec_ptr t, int* iflag);
void phist_b200_DjadaCorrection_minres(phist_Dconst_sparseMat_ptr A, phist_Dconst_mvec_ptr Q,
                                       phist_Dconst_mvec_ptr res, const int resIndex[], int k, const double sigma[],
                                       const double tol[], int maxIter, int maxBas, phist_Dmvec_ptr t, int* iflag);
void phist_b200_SjadaCorrection_minres(phist_Sconst_sparseMat_ptr A, phist_Sconst_mvec_ptr Q,
                                       phist_Sconst_mvec_ptr res, const int resIndex[], int k, const double sigma[],
                                       const double tol[], int maxIter, int maxBas, phist_Smvec_ptr t, int* iflag);
void phist_b200_mvec_DtoS(phist_Dconst_mvec_ptr X, phist_Smvec_ptr Y, int* iflag);
void phist_b200_mvec_StoD(phist_Sconst_mvec_ptr X, phist_Dmvec_ptr Y, int* iflag);
void phist_b200_sparseMat_DtoS(phist_Dconst_sparseMat_ptr A, phist_SsparseMat_ptr* As, int* iflag);
}

namespace {

// an FP32 work block of fixed row map whose width grows on demand; view()
// returns a view of its first ncols columns
struct WorkBlock {
  phist_Smvec_ptr full = nullptr;
  phist_Smvec_ptr v = nullptr;
  int cap = 0;
  void view(phist_const_map_ptr map, int ncols, int* iflag)
  {
    *iflag = 0;
    if (ncols > cap) {
      if (v) { phist_Smvec_delete(v, iflag); v = nullptr; if (*iflag) return; }
      if (full) { phist_Smvec_delete(full, iflag); full = nullptr; if (*iflag) return; }
      phist_Smvec_create(&full, map, ncols, iflag);
      if (*iflag) return;
      cap = ncols;
    }
    phist_Smvec_view_block(full, &v, 0, ncols - 1, iflag);
  }
  void release(int* iflag)
  {
    *iflag = 0;
    if (v) phist_Smvec_delete(v, iflag);
    if (full) phist_Smvec_delete(full, iflag);
    v = full = nullptr;
    cap = 0;
  }
};

}  // namespace

struct pb_mixed_jada {
  int fp32 = 1;         // correction equations in FP32 (else FP64)
  int devgmres = 0;     // the library's device-resident GMRES (else PHIST's blocked GMRES)
  int minres = 0;       // innerSolvType MINRES: the device solver runs MINRES
  int maxBas = 20;      // GMRES basis size of the device solver
  phist_Dconst_sparseMat_ptr A = nullptr;
  phist_SsparseMat_ptr As = nullptr;
  phist_SlinearOp opAs;
  phist_SjadaCorrectionSolver_ptr inner = nullptr;
  phist_const_map_ptr map = nullptr;
  WorkBlock Q, R, T;
  long calls = 0, systems = 0, unconverged = 0;
};

#define PB_CHK(call)          \
  do {                        \
    *iflag = 0;               \
    call;                     \
    if (*iflag < 0) return;   \
  } while (0)

static void pb_mixed_jada_run(void* data, void const* A_op, void const* B_op, void const* Qtil,
                              void const* BQtil, const double sigma_r[], const double sigma_i[],
                              void const* res, const int resIndex[], const double tol[], int maxIter,
                              void* t, int robust, int abortAfterFirstConvergedInBlock, int* iflag)
{
  (void)A_op;
  (void)BQtil;
  pb_mixed_jada* me = (pb_mixed_jada*)data;
  *iflag = 0;
  if (!me || B_op != nullptr) {
    *iflag = PHIST_NOT_IMPLEMENTED;  // generalized problems: the FP32 copy is of A alone
    return;
  }
  int k = 0, nres = 0, nq = 0;
  PB_CHK(phist_Dmvec_num_vectors((phist_Dconst_mvec_ptr)t, &k, iflag));
  PB_CHK(phist_Dmvec_num_vectors((phist_Dconst_mvec_ptr)res, &nres, iflag));
  PB_CHK(phist_Dmvec_num_vectors((phist_Dconst_mvec_ptr)Qtil, &nq, iflag));
  for (int j = 0; j < k; j++)
    if (sigma_i && sigma_i[j] != 0.0) {
      *iflag = PHIST_NOT_IMPLEMENTED;  // complex shifts need the complex FP32 path
      return;
    }
  if (k > 64) {
    *iflag = PHIST_INVALID_INPUT;
    return;
  }
  if (!me->fp32) {
    // FP64 on the device-resident GMRES: no conversions
    *iflag = 0;
    (me->minres ? phist_b200_DjadaCorrection_minres : phist_b200_DjadaCorrection_gmres)(
        me->A, (phist_Dconst_mvec_ptr)Qtil, (phist_Dconst_mvec_ptr)res, resIndex, k, sigma_r, tol, maxIter,
        me->maxBas, (phist_Dmvec_ptr)t, iflag);
    if (*iflag < 0) return;
    me->calls++;
    me->systems += k;
    me->unconverged += *iflag;
    return;
  }

  PB_CHK(me->Q.view(me->map, nq, iflag));
  PB_CHK(me->R.view(me->map, nres, iflag));
  PB_CHK(me->T.view(me->map, k, iflag));
  PB_CHK(phist_b200_mvec_DtoS((phist_Dconst_mvec_ptr)Qtil, me->Q.v, iflag));
  PB_CHK(phist_b200_mvec_DtoS((phist_Dconst_mvec_ptr)res, me->R.v, iflag));
  // Scale every right-hand side to norm 1024.  PHIST's blocked GMRES counts a
  // system as converged once its residual is below 1000 eps of the type in
  // absolute terms (phist_blockedgmres_def.hpp:606,970), i.e. 1.2e-4 in FP32:
  // late Jacobi-Davidson residuals are smaller than that and would return
  // t = 0.  The correction equation is linear in r and the solver returns
  // t normalised (phist_jadaCorrectionSolver_def.hpp:583, end of the GMRES
  // branch), so the scaling changes nothing else.
  {
    std::vector<double> nr(nres);
    std::vector<float> sc(nres);
    PB_CHK(phist_Dmvec_norm2((phist_Dconst_mvec_ptr)res, nr.data(), iflag));
    for (int j = 0; j < nres; j++) sc[j] = nr[j] > 0.0 ? (float)(1024.0 / nr[j]) : 1.0f;
    PB_CHK(phist_Smvec_vscale(me->R.v, sc.data(), iflag));
  }

  *iflag = 0;
  if (me->devgmres) {
    (me->minres ? phist_b200_SjadaCorrection_minres : phist_b200_SjadaCorrection_gmres)(
        me->As, me->Q.v, me->R.v, resIndex, k, sigma_r, tol, maxIter, me->maxBas, me->T.v, iflag);
  } else {
    float s[64], tl[64];
    for (int j = 0; j < k; j++) {
      s[j] = (float)sigma_r[j];
      tl[j] = (float)tol[j];
    }
    phist_SjadaCorrectionSolver_run(me->inner, &me->opAs, nullptr, me->Q.v, nullptr, s, me->R.v, resIndex, tl,
                                    maxIter, me->T.v, robust, abortAfterFirstConvergedInBlock, 0, iflag);
  }
  if (*iflag < 0) return;
  const int notConverged = *iflag;
  PB_CHK(phist_b200_mvec_StoD(me->T.v, (phist_Dmvec_ptr)t, iflag));
  me->calls++;
  me->systems += k;
  me->unconverged += notConverged;
  *iflag = notConverged;
}

extern "C" void phist_b200_mixed_jada_create(pb_mixed_jada** out, void const* A, const phist_jadaOpts* opts,
                                             int* iflag)
{
  phist_b200_jada_inner_create(out, A, opts, 1, 0, iflag);
}

extern "C" void phist_b200_jada_inner_create(pb_mixed_jada** out, void const* A, const phist_jadaOpts* opts,
                                             int fp32, int devgmres, int* iflag)
{
  *iflag = 0;
  if (!out || !A || !opts) {
    *iflag = PHIST_INVALID_INPUT;
    return;
  }
  if (opts->innerSolvType != phist_GMRES && opts->innerSolvType != phist_MINRES) {
    *iflag = PHIST_NOT_IMPLEMENTED;
    return;
  }
  pb_mixed_jada* me = new (std::nothrow) pb_mixed_jada();
  if (!me) {
    *iflag = PHIST_MEM_ALLOC_FAILED;
    return;
  }
  me->fp32 = fp32 ? 1 : 0;
  me->devgmres = (devgmres || !fp32) ? 1 : 0;  // FP64 here means the device GMRES
  me->minres = opts->innerSolvType == phist_MINRES ? 1 : 0;
  me->maxBas = opts->innerSolvMaxBas > 0 ? opts->innerSolvMaxBas : opts->innerSolvMaxIters;
  me->A = (phist_Dconst_sparseMat_ptr)A;
  if (!me->fp32) {
    *out = me;
    return;
  }
  phist_b200_sparseMat_DtoS((phist_Dconst_sparseMat_ptr)A, &me->As, iflag);
  if (*iflag == 0) phist_SlinearOp_wrap_sparseMat(&me->opAs, me->As, iflag);
  if (*iflag == 0) phist_SsparseMat_get_domain_map(me->As, &me->map, iflag);
  if (*iflag == 0 && !me->devgmres) {
    phist_jadaOpts o = *opts;
    o.customSolver = nullptr;
    o.customSolver_run = nullptr;
    o.customSolver_run1 = nullptr;
    phist_SjadaCorrectionSolver_create(&me->inner, o, me->map, iflag);
  }
  if (*iflag != 0) {
    int e = *iflag, i2 = 0;
    if (me->As) phist_SsparseMat_delete(me->As, &i2);
    delete me;
    *iflag = e;
    return;
  }
  *out = me;
}

extern "C" void phist_b200_mixed_jada_install(pb_mixed_jada* me, phist_jadaOpts* opts, int* iflag)
{
  *iflag = 0;
  if (!me || !opts) {
    *iflag = PHIST_INVALID_INPUT;
    return;
  }
  opts->innerSolvType = phist_USER_LINSOLV;
  opts->customSolver = me;
  opts->customSolver_run = &pb_mixed_jada_run;
  opts->customSolver_run1 = nullptr;
}

extern "C" void phist_b200_mixed_jada_stats(const pb_mixed_jada* me, long* calls, long* systems,
                                            long* unconverged, int* iflag)
{
  *iflag = me ? 0 : PHIST_INVALID_INPUT;
  if (!me) return;
  if (calls) *calls = me->calls;
  if (systems) *systems = me->systems;
  if (unconverged) *unconverged = me->unconverged;
}

extern "C" void phist_b200_mixed_jada_delete(pb_mixed_jada* me, int* iflag)
{
  *iflag = 0;
  if (!me) return;
  int e = 0;
  me->Q.release(&e);
  me->R.release(&e);
  me->T.release(&e);
  if (me->inner) phist_SjadaCorrectionSolver_delete(me->inner, &e);
  if (me->opAs.destroy) me->opAs.destroy(&me->opAs, &e);
  if (me->As) phist_SsparseMat_delete(me->As, &e);
  delete me;
}
