// pb_mixed_carp.cpp -- FP32 CARP-CG inside an FP64 refinement loop
// (algorithm and argument conventions in pb_mixed_carp.h).
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
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
  std::vector<double> zerosD;
  phist_Scarp_cgState_ptr S = nullptr;
  phist_Dcarp_cgState_ptr SD = nullptr;  // FP64 inner solver, created when first needed
  int fp32_steps = 0, fp64_steps = 0;   // corrections of the last solve
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
  if (me->SD) phist_Dcarp_cgState_delete(me->SD, &e);
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
  me->zerosD.assign(nsys, 0.0);
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
  const char* verb = getenv("PB_MIXED_CARP_VERBOSE");
  const bool verbose = verb && atoi(verb) > 0;
  std::vector<double> nb(ns), nr(ns), nr_prev(ns), scale(ns), unscale(ns), last(ns, 0.0), undo(ns), nd(ns);
  PB_CHK(phist_Dmvec_norm2((phist_Dconst_mvec_ptr)B, nb.data(), iflag));
  auto residual = [&](int* iflag) {
    // r = b - (A - sigma I) x and its column norms, FP64
    PB_CHK(phist_Dmvec_add_mvec(1.0, (phist_Dconst_mvec_ptr)B, 0.0, me->R, iflag));
    PB_CHK(phist_DsparseMat_times_mvec_vadd_mvec(-1.0, me->A, me->negSigma.data(), (phist_Dconst_mvec_ptr)X, 1.0,
                                                  me->R, iflag));
    PB_CHK(phist_Dmvec_norm2(me->R, nr.data(), iflag));
  };
  // FP32 CG on an ill-conditioned shift can stop converging and then drift
  // far from the solution if it runs long enough, so each FP32 inner solve is
  // capped: the cap starts at min(maxInnerIter, 1000), halves whenever a
  // correction made some column's FP64 residual larger (that correction is
  // taken back; caps from that one up are not tried again) and doubles after
  // a correction that reduced every corrected column's residual by at least
  // 10%.  Where the shifted system is too ill-conditioned for FP32 (cond *
  // eps_float near 1) a correction gains little: after 2 corrections in a row
  // that cut no residual by half, the remaining corrections are solved with
  // PHIST's FP64 carp_cgState to innerTol.  The loop ends when every column
  // has converged, after maxRefine corrections, or after 3 FP64 corrections
  // in a row that cut no residual by 10%.
  int cap = std::min(maxInnerIter, 1000), ceiling = maxInnerIter, slow = 0, stalled = 0;
  bool use64 = false;
  me->fp32_steps = me->fp64_steps = 0;
  int k = 0, unconverged = ns;
  for (;; k++) {
    PB_CHK(residual(iflag));
    if (k > 0) {
      bool worse = false, better = false, all_better = true, halved = false;
      for (int j = 0; j < ns; j++) {
        undo[j] = 0.0;
        if (last[j] == 0.0) continue;
        if (!(nr[j] < nr_prev[j])) {
          undo[j] = -last[j];
          worse = true;
        }
        if (nr[j] <= 0.9 * nr_prev[j]) better = true;
        else all_better = false;
        if (nr[j] <= 0.5 * nr_prev[j]) halved = true;
      }
      if (worse) {
        PB_CHK(phist_Dmvec_vadd_mvec(undo.data(), me->D, 1.0, (phist_Dmvec_ptr)X, iflag));
        PB_CHK(residual(iflag));
        ceiling = std::max(cap / 2, 16);
        cap = ceiling;
      } else if (all_better) {
        cap = (int)std::min<int64_t>(2 * (int64_t)cap, ceiling);
      }
      if (use64) {
        stalled = better ? 0 : stalled + 1;
      } else {
        slow = halved ? 0 : slow + 1;
        if (slow >= 2) use64 = true;
      }
    }
    unconverged = 0;
    for (int j = 0; j < ns; j++) unconverged += !(nr[j] <= tol * nb[j]);
    if (verbose) {
      fprintf(stderr, "mixed_carp refinement %d (%s, inner cap %d): relres", k, use64 ? "FP64" : "FP32",
              use64 ? maxInnerIter : cap);
      for (int j = 0; j < ns; j++) fprintf(stderr, " %.3e", nr[j] / nb[j]);
      fprintf(stderr, "\n");
    }
    if (unconverged == 0 || k >= maxRefine || stalled >= 3) break;
    // d = (A - sigma I)^{-1} r.  Each column of r is scaled to norm 1 first,
    // so the FP32 recurrence works on quantities of order one however small
    // the FP64 residual has become (no underflow of r'r or p'q); the
    // correction is scaled back when it is added.  Converged columns and
    // columns with a non-finite correction are left unchanged.
    for (int j = 0; j < ns; j++) {
      const bool ok = std::isfinite(nr[j]) && nr[j] > 0.0;
      scale[j] = ok ? 1.0 / nr[j] : 1.0;
      unscale[j] = (ok && !(nr[j] <= tol * nb[j])) ? nr[j] : 0.0;
    }
    PB_CHK(phist_Dmvec_vscale(me->R, scale.data(), iflag));
    if (use64) {
      if (!me->SD) {
        PB_CHK(phist_Dcarp_cgState_create(&me->SD, me->A, nullptr, ns, me->sigma.data(), me->zerosD.data(), iflag));
        for (int j = 0; j < ns; j++) me->SD->omega_[j] = omega ? omega[j] : 1.0;
      }
      PB_CHK(phist_Dmvec_put_value(me->D, 0.0, iflag));
      PB_CHK(phist_Dcarp_cgState_reset(me->SD, me->R, nullptr, iflag));
      *iflag = 0;
      phist_Dcarp_cgState_iterate(me->SD, me->D, nullptr, innerTol, maxInnerIter, 0, iflag);
      if (*iflag < 0) return;
      me->fp64_steps++;
    } else {
      PB_CHK(phist_b200_mvec_DtoS(me->R, me->Rs, iflag));
      PB_CHK(phist_Smvec_put_value(me->Ds, 0.0f, iflag));
      PB_CHK(phist_Scarp_cgState_reset(me->S, me->Rs, nullptr, iflag));
      *iflag = 0;
      phist_Scarp_cgState_iterate(me->S, me->Ds, nullptr, (float)innerTol, cap, 0, iflag);
      if (*iflag < 0) return;
      PB_CHK(phist_b200_mvec_StoD(me->Ds, me->D, iflag));
      me->fp32_steps++;
    }
    PB_CHK(phist_Dmvec_norm2(me->D, nd.data(), iflag));
    for (int j = 0; j < ns; j++) {
      if (!std::isfinite(nd[j])) unscale[j] = 0.0;
      last[j] = unscale[j];
      nr_prev[j] = nr[j];
    }
    // x += ||r_j|| d_j in FP64
    PB_CHK(phist_Dmvec_vadd_mvec(unscale.data(), me->D, 1.0, (phist_Dmvec_ptr)X, iflag));
  }
  if (refinements) *refinements = k;
  *iflag = unconverged;
}

extern "C" void phist_b200_mixed_carp_stats(pb_mixed_carp const* me, int* fp32_steps, int* fp64_steps, int* iflag)
{
  *iflag = 0;
  if (!me) {
    *iflag = PHIST_INVALID_INPUT;
    return;
  }
  if (fp32_steps) *fp32_steps = me->fp32_steps;
  if (fp64_steps) *fp64_steps = me->fp64_steps;
}

extern "C" void phist_b200_mixed_carp_delete(pb_mixed_carp* me, int* iflag)
{
  *iflag = 0;
  if (me) release(me);
}
