// carp_run.cpp -- runs PHIST's unchanged CARP-CG solver
// (phist_Dcarp_cgState_iterate, src/krylov/phist_carp_cg_def.hpp:304) for a
// queue of real shifts on the b200 kernel library and prints one JSON line
// with explicit relative residuals (null where not finite), launch counts and
// wall times.
//
// The call sequence follows PHIST's driver drivers/carp_cg.c:286-320: one
// carp_cgState per block of shifts (create, reset with the right-hand sides,
// iterate, delete).  Here each column of a block carries its own shift and
// right-hand side, so a block of width w solves w different systems
// (A - sigma_j I) x_j = b_j at once; the solver state, the CARP sweeps
// (carp_setup/carp_sweep, phist_kernels_carp_decl.h:35,44) and all vector
// operations run on the GPU through libphist_kernels_b200.so.
//
//   carp_run <problem> [key=value ...]
//   keys: nshifts (32) block (8) tol (1e-10) maxIter (20000) seed (4)
//         omega (1.0) sigma (SELL sigma, 1) reps (1)
//         out (file receiving the solutions X, n x nshifts row-major float64)
//         mixed=1: FP32 CARP-CG inside FP64 iterative refinement
//         (pb_mixed_carp.h) with innerTol (1e-5) and maxRefine (20); maxIter
//         then bounds the FP32 iterations of each refinement step
//         batch=1: the library's batched solver phist_b200_DcarpCG_batch
//         instead of PHIST's carp_cgState (block = slots, converged systems
//         refilled from the queue, checks every checkEvery (10) iterations;
//         mixed=1 there means FP32 inner solves with FP64 refinement;
//         block=0 there: slot count from phist_b200_DcarpCG_tune_block)
//   shifts sigma_j = 2.5 * u(seed, j), right-hand sides b_ij = u(seed + 1 + j, i)
//   with u uniform [-1,1) from a splitmix64 hash (the library's pb_unif).
#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "phist_config.h"
#include "phist_kernels.h"
#include "phist_core.h"
#include "phist_krylov.h"
#include "phist_enums.h"
#include "pb_mixed_carp.h"

extern "C" {
void phist_b200_Dcreate_problem(phist_DsparseMat_ptr* A, phist_const_comm_ptr comm,
                                const char* problem, int* iflag);
void phist_b200_set_sell_params(int C, int64_t sigma, int* iflag);
void phist_b200_synchronize(int* iflag);
void phist_b200_launch_count(uint64_t* count, int* iflag);
void phist_b200_DcarpCG_batch(phist_Dconst_sparseMat_ptr A, int nsys, const double sigma[],
                              phist_Dconst_mvec_ptr B, phist_Dmvec_ptr X, int block, double tol,
                              int maxIter, int checkEvery, int mixed, double innerTol, int iters[],
                              double relres[], int* iflag);
void phist_b200_DcarpCG_tune_block(phist_Dconst_sparseMat_ptr A, int nsys, int mixed, int reps, int* block,
                                   double iter_us[], int* iflag);
}

#define CHK(call)                                                              \
  do {                                                                         \
    iflag = 0;                                                                 \
    call;                                                                      \
    if (iflag < 0) {                                                           \
      fprintf(stderr, "error %d in %s (line %d)\n", iflag, #call, __LINE__); \
      return 1;                                                                \
    }                                                                          \
  } while (0)

static uint64_t mix64(uint64_t z)
{
  z += 0x9E3779B97F4A7C15ull;
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return z ^ (z >> 31);
}
// JSON number, null where not finite
static void jnum(const char* sep, double v, const char* fmt)
{
  if (std::isfinite(v)) { printf("%s", sep); printf(fmt, v); }
  else printf("%snull", sep);
}

static double unif(uint64_t seed, uint64_t idx)
{
  const uint64_t h = mix64(seed * 0x632BE59BD9B4E019ull + mix64(idx));
  return (double)(h >> 11) * (1.0 / 9007199254740992.0) * 2.0 - 1.0;
}

int main(int argc, char** argv)
{
  if (argc < 2) {
    fprintf(stderr, "usage: %s <problem> [key=value ...]\n", argv[0]);
    return 2;
  }
  int iflag = 0;
  const char* problem = argv[1];
  int nshifts = 32, block = 8, maxIter = 20000, reps = 1;
  double tol = 1e-10, omega = 1.0;
  uint64_t seed = 4;
  int64_t sigma = 1;
  std::string out;
  int mixed = 0, maxRefine = 20, batch = 0, checkEvery = 10;
  double innerTol = 1e-5;
  for (int a = 2; a < argc; a++) {
    const char* kv = argv[a];
    const char* eq = strchr(kv, '=');
    if (!eq) continue;
    std::string k(kv, eq - kv);
    const char* v = eq + 1;
    if (k == "nshifts") nshifts = atoi(v);
    else if (k == "block") block = atoi(v);
    else if (k == "tol") tol = atof(v);
    else if (k == "maxIter") maxIter = atoi(v);
    else if (k == "seed") seed = strtoull(v, nullptr, 10);
    else if (k == "omega") omega = atof(v);
    else if (k == "sigma") sigma = atoll(v);
    else if (k == "reps") reps = atoi(v);
    else if (k == "out") out = v;
    else if (k == "mixed") mixed = atoi(v);
    else if (k == "innerTol") innerTol = atof(v);
    else if (k == "maxRefine") maxRefine = atoi(v);
    else if (k == "batch") batch = atoi(v);
    else if (k == "checkEvery") checkEvery = atoi(v);
  }
  if (block < (batch ? 0 : 1) || nshifts < 1) return 2;

  CHK(phist_kernels_init(&argc, &argv, &iflag));
  phist_comm_ptr comm = NULL;
  CHK(phist_comm_create(&comm, &iflag));
  CHK(phist_b200_set_sell_params(32, sigma, &iflag));
  phist_DsparseMat_ptr A = NULL;
  iflag = (sigma > 1 ? PHIST_SPARSEMAT_PERM_LOCAL : 0) | PHIST_SPARSEMAT_OPT_CARP;
  phist_b200_Dcreate_problem(&A, comm, problem, &iflag);
  if (iflag < 0) { fprintf(stderr, "cannot create %s\n", problem); return 1; }
  phist_const_map_ptr map = NULL;
  CHK(phist_DsparseMat_get_domain_map(A, &map, &iflag));
  phist_lidx nloc = 0;
  CHK(phist_map_get_local_length(map, &nloc, &iflag));

  std::vector<double> shifts(nshifts);
  for (int j = 0; j < nshifts; j++) shifts[j] = 2.5 * unif(seed, (uint64_t)j);
  phist_Dmvec_ptr B = NULL, X = NULL, R = NULL;
  CHK(phist_Dmvec_create(&B, map, nshifts, &iflag));
  CHK(phist_Dmvec_create(&X, map, nshifts, &iflag));
  CHK(phist_Dmvec_create(&R, map, nshifts, &iflag));
  {
    std::vector<double> h((size_t)nloc * nshifts);
    for (phist_lidx i = 0; i < nloc; i++)
      for (int j = 0; j < nshifts; j++) h[(size_t)i * nshifts + j] = unif(seed + 1 + j, (uint64_t)i);
    CHK(phist_Dmvec_set_data(B, h.data(), nshifts, 1, &iflag));
  }

  std::vector<double> iter_us(6, 0.0);
  if (block == 0) {
    CHK(phist_b200_DcarpCG_tune_block(A, nshifts, mixed, 3, &block, iter_us.data(), &iflag));
  }

  std::vector<double> walls, relres(nshifts, 0.0);
  std::vector<int> refines, fp64_steps, conv(nshifts, 0), batch_iters;
  uint64_t launches = 0;
  for (int rep = 0; rep < reps; rep++) {
    CHK(phist_Dmvec_put_value(X, 0.0, &iflag));
    refines.clear();
    fp64_steps.clear();
    uint64_t l0 = 0, l1 = 0;
    CHK(phist_b200_launch_count(&l0, &iflag));
    CHK(phist_b200_synchronize(&iflag));
    auto t0 = std::chrono::steady_clock::now();
    if (batch) {
      std::vector<double> brel(nshifts, 0.0);
      batch_iters.assign(nshifts, 0);
      iflag = 0;
      phist_b200_DcarpCG_batch(A, nshifts, shifts.data(), B, X, block, tol, maxIter, checkEvery, mixed, innerTol,
                               batch_iters.data(), brel.data(), &iflag);
      if (iflag < 0) {
        fprintf(stderr, "DcarpCG_batch returned %d\n", iflag);
        return 1;
      }
    }
    for (int j0 = 0; j0 < nshifts && !batch; j0 += block) {
      const int w = std::min(block, nshifts - j0);
      phist_Dmvec_ptr Bj = NULL, Xj = NULL;
      CHK(phist_Dmvec_view_block(B, &Bj, j0, j0 + w - 1, &iflag));
      CHK(phist_Dmvec_view_block(X, &Xj, j0, j0 + w - 1, &iflag));
      if (mixed) {
        pb_mixed_carp* M = NULL;
        std::vector<double> om(w, omega);
        CHK(phist_b200_mixed_carp_create(&M, A, w, &shifts[j0], &iflag));
        int nref = 0;
        iflag = 0;
        phist_b200_mixed_carp_solve(M, Bj, Xj, om.data(), tol, innerTol, maxIter, maxRefine, &nref, &iflag);
        if (iflag < 0) {
          fprintf(stderr, "mixed_carp_solve returned %d\n", iflag);
          return 1;
        }
        refines.push_back(nref);
        int s32 = 0, s64 = 0;
        CHK(phist_b200_mixed_carp_stats(M, &s32, &s64, &iflag));
        fp64_steps.push_back(s64);
        CHK(phist_b200_mixed_carp_delete(M, &iflag));
      } else {
        phist_Dcarp_cgState_ptr S = NULL;
        // carp_cgState_create reads sigma_i[j] for every j (phist_carp_cg_def.hpp:131-135)
        std::vector<double> zeros(w, 0.0);
        CHK(phist_Dcarp_cgState_create(&S, A, NULL, w, &shifts[j0], zeros.data(), &iflag));
        for (int j = 0; j < w; j++) S->omega_[j] = omega;
        CHK(phist_Dcarp_cgState_reset(S, Bj, NULL, &iflag));
        iflag = 0;
        phist_Dcarp_cgState_iterate(S, Xj, NULL, tol, maxIter, 0, &iflag);
        if (iflag < 0) {
          fprintf(stderr, "carp_cgState_iterate returned %d\n", iflag);
          return 1;
        }
        for (int j = 0; j < w; j++) conv[j0 + j] = S->conv[j];
        CHK(phist_Dcarp_cgState_delete(S, &iflag));
      }
      CHK(phist_Dmvec_delete(Xj, &iflag));
      CHK(phist_Dmvec_delete(Bj, &iflag));
    }
    CHK(phist_b200_synchronize(&iflag));
    walls.push_back(std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count());
    CHK(phist_b200_launch_count(&l1, &iflag));
    launches = l1 - l0;
    // explicit residuals r_j = b_j - (A - sigma_j I) x_j, relative to ||b_j||
    std::vector<double> negs(nshifts), nb(nshifts), nr(nshifts);
    for (int j = 0; j < nshifts; j++) negs[j] = -shifts[j];
    CHK(phist_Dmvec_add_mvec(1.0, B, 0.0, R, &iflag));
    CHK(phist_DsparseMat_times_mvec_vadd_mvec(-1.0, A, negs.data(), X, 1.0, R, &iflag));
    CHK(phist_Dmvec_norm2(B, nb.data(), &iflag));
    CHK(phist_Dmvec_norm2(R, nr.data(), &iflag));
    for (int j = 0; j < nshifts; j++) relres[j] = nr[j] / nb[j];
    // the refinement loops stop on exactly this FP64 residual test
    if (mixed || batch)
      for (int j = 0; j < nshifts; j++) conv[j] = nr[j] <= tol * nb[j];
  }
  int nconv = 0;
  double maxres = 0.0;
  for (int j = 0; j < nshifts; j++) {
    nconv += conv[j];
    maxres = std::isfinite(relres[j]) ? std::max(maxres, relres[j]) : INFINITY;
  }
  printf("{\"problem\": \"%s\", \"mixed\": %d, \"innerTol\": %.3e, \"refinements\": [", problem, mixed,
         innerTol);
  for (size_t i = 0; i < refines.size(); i++) printf("%s%d", i ? ", " : "", refines[i]);
  printf("], \"fp64_refinements\": [");
  for (size_t i = 0; i < fp64_steps.size(); i++) printf("%s%d", i ? ", " : "", fp64_steps[i]);
  printf("], \"tuned_iter_us\": [");
  for (int k = 0; k < 6; k++) printf("%s%.2f", k ? ", " : "", iter_us[k]);
  printf("], \"n\": %d, \"nshifts\": %d, \"block\": %d, \"tol\": %.3e, \"maxIter\": %d, "
         "\"omega\": %g, \"nconv\": %d, \"launches\": %llu, \"max_relres\": ",
         nloc, nshifts, block, tol, maxIter, omega, nconv, (unsigned long long)launches);
  jnum("", maxres, "%.6e");
  printf(", \"batch\": %d, \"batch_iters\": [", batch);
  for (size_t i = 0; i < batch_iters.size(); i++) printf("%s%d", i ? ", " : "", batch_iters[i]);
  printf("], \"wall\": [");
  for (size_t i = 0; i < walls.size(); i++) printf("%s%.6f", i ? ", " : "", walls[i]);
  printf("], \"shifts\": [");
  for (int j = 0; j < nshifts; j++) printf("%s%.17g", j ? ", " : "", shifts[j]);
  printf("], \"relres\": [");
  for (int j = 0; j < nshifts; j++) jnum(j ? ", " : "", relres[j], "%.6e");
  printf("]}\n");
  fflush(stdout);
  if (!out.empty()) {
    std::vector<double> h((size_t)nloc * nshifts);
    CHK(phist_Dmvec_get_data(X, h.data(), nshifts, 1, &iflag));
    FILE* f = fopen(out.c_str(), "wb");
    if (!f || fwrite(h.data(), sizeof(double), h.size(), f) != h.size()) {
      fprintf(stderr, "cannot write %s\n", out.c_str());
      return 1;
    }
    fclose(f);
  }
  CHK(phist_Dmvec_delete(R, &iflag));
  CHK(phist_Dmvec_delete(X, &iflag));
  CHK(phist_Dmvec_delete(B, &iflag));
  CHK(phist_DsparseMat_delete(A, &iflag));
  CHK(phist_comm_delete(comm, &iflag));
  CHK(phist_kernels_finalize(&iflag));
  return 0;
}
