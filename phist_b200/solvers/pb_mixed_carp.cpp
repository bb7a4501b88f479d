// pb_mixed_carp.cpp -- FP32 CARP-CG inside an FP64 refinement loop
// (algorithm and argument conventions in pb_mixed_carp.h).
#include <cmath>
#include <new>
#include <vector>

#include "phist_config.h"
#include "phist_kernels.h"
#include "phist_core.h"
#include "phist_krylov.h"
#include "pb_mixed_carp.h"

extern "C" {
void phist_b200_mvec_DtoS(phist_Dconst_mvec_ptr X, phist_Smvec_ptr Y, int* iflag);
void phist_b200_mvec_StoD(phist_Sconst_mvec_ptr X, phist_Dmvec_ptr Y, int* iflag);
void phist_b200_sparseMat_DtoS(phist_Dconst_sparseMat_ptr A, phist_SsparseMat_ptr* As, int* iflag);
}

struct pb_mixed_carp {
  phist_Dconst_sparseMat_ptr A = nullptr;
  phist_SsparseMat_ptr As = nullptr;
  int nsys = 0;
  std::vector<double> sigma, negSigma;
  std::vector<float> sigmaS, zerosS;
  phist_Scarp_cgState_ptr S = nullptr;
  phist_Dmvec_ptr R = nullptr, D = nullptr;
  phist_Smvec_ptr Rs = nullptr, Ds = nullptr;
};

#define PB_CHK(call)          \
  do {                        \
    *iflag = 0;               \
    call;                     \
    if (*iflag < 0) return;   \
  } while (0)

static void release(pb_mixed_carp* me)
{
  int e = 0;
  if (me->S) phist_Scarp_cgState_delete(me->S, &e);
  if (me->Rs) phist_Smvec_delete(me->Rs, &e);
  if (me->Ds) phist_Smvec_delete(me->Ds, &e);
  if (me->R) phist_Dmvec_delete(me->R, &e);
  if (me->D) phist_Dmvec_delete(me->D, &e);
  if (me->As) phist_SsparseMat_delete(me->As, &e);
  delete me;
}

extern "C" void phist_b200_mixed_carp_create(pb_mixed_carp** out, void const* A, int nsys, const double sigma[],
                                             int* iflag)
{
  *iflag = 0;
  if (!out || !A || nsys < 1 || !sigma) {
    *iflag = PHIST_INVALID_INPUT;
    return;
  }
  pb_mixed_carp* me = new (std::nothrow) pb_mixed_carp();
  if (!me) {
    *iflag = PHIST_MEM_ALLOC_FAILED;
    return;
  }
  me->A = (phist_Dconst_sparseMat_ptr)A;
  me->nsys = nsys;
  me->sigma.assign(sigma, sigma + nsys);
  me->negSigma.resize(nsys);
  me->sigmaS.resize(nsys);
  me->zerosS.assign(nsys, 0.0f);  // carp_cgState_create reads sigma_i[j] for every j
  for (int j = 0; j < nsys; j++) {
    me->negSigma[j] = -sigma[j];
    me->sigmaS[j] = (float)sigma[j];
  }
  phist_const_map_ptr mapD = nullptr, mapS = nullptr;
  phist_b200_sparseMat_DtoS(me->A, &me->As, iflag);
  if (*iflag == 0) phist_DsparseMat_get_row_map(me->A, &mapD, iflag);
  if (*iflag == 0) phist_SsparseMat_get_row_map(me->As, &mapS, iflag);
  if (*iflag == 0) phist_Dmvec_create(&me->R, mapD, nsys, iflag);
  if (*iflag == 0) phist_Dmvec_create(&me->D, mapD, nsys, iflag);
  if (*iflag == 0) phist_Smvec_create(&me->Rs, mapS, nsys, iflag);
  if (*iflag == 0) phist_Smvec_create(&me->Ds, mapS, nsys, iflag);
  if (*iflag == 0) phist_Scarp_cgState_create(&me->S, me->As, nullptr, nsys, me->sigmaS.data(), me->zerosS.data(), iflag);
  if (*iflag != 0) {
    const int e = *iflag;
    release(me);
    *iflag = e;
    return;
  }
  *out = me;
}

extern "C" void phist_b200_mixed_carp_solve(pb_mixed_carp* me, void const* B, void* X, const double omega[],
                                            double tol, double innerTol, int maxInnerIter, int maxRefine,
                                            int* refinements, int* iflag)
{
  *iflag = 0;
  if (!me || !B || !X) {
    *iflag = PHIST_INVALID_INPUT;
    return;
  }
  const int ns = me->nsys;
  for (int j = 0; j < ns; j++) me->S->omega_[j] = omega ? (float)omega[j] : 1.0f;
  std::vector<double> nb(ns), nr(ns);
  PB_CHK(phist_Dmvec_norm2((phist_Dconst_mvec_ptr)B, nb.data(), iflag));
  int k = 0, unconverged = ns;
  for (;; k++) {
    // r = b - (A - sigma I) x in FP64
    PB_CHK(phist_Dmvec_add_mvec(1.0, (phist_Dconst_mvec_ptr)B, 0.0, me->R, iflag));
    PB_CHK(phist_DsparseMat_times_mvec_vadd_mvec(-1.0, me->A, me->negSigma.data(), (phist_Dconst_mvec_ptr)X, 1.0,
                                                  me->R, iflag));
    PB_CHK(phist_Dmvec_norm2(me->R, nr.data(), iflag));
    unconverged = 0;
    for (int j = 0; j < ns; j++) unconverged += !(nr[j] <= tol * nb[j]);
    if (unconverged == 0 || k >= maxRefine) break;
    // d = (A - sigma I)^{-1} r to innerTol, FP32
    PB_CHK(phist_b200_mvec_DtoS(me->R, me->Rs, iflag));
    PB_CHK(phist_Smvec_put_value(me->Ds, 0.0f, iflag));
    PB_CHK(phist_Scarp_cgState_reset(me->S, me->Rs, nullptr, iflag));
    *iflag = 0;
    phist_Scarp_cgState_iterate(me->S, me->Ds, nullptr, (float)innerTol, maxInnerIter, 0, iflag);
    if (*iflag < 0) return;
    // x += d in FP64
    PB_CHK(phist_b200_mvec_StoD(me->Ds, me->D, iflag));
    PB_CHK(phist_Dmvec_add_mvec(1.0, me->D, 1.0, (phist_Dmvec_ptr)X, iflag));
  }
  if (refinements) *refinements = k;
  *iflag = unconverged;
}

extern "C" void phist_b200_mixed_carp_delete(pb_mixed_carp* me, int* iflag)
{
  *iflag = 0;
  if (me) release(me);
}
