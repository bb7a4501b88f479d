// jada_run.cpp -- runs PHIST's unchanged block Jacobi-Davidson solver
// (phist_Dsubspacejada, src/jada/phist_subspacejada_def.hpp:78) on the b200
// kernel library and prints one JSON line with the eigenvalues, explicit
// residual norms, iteration count and wall time.
//
// This is the reference side of the drop-in boundary: the solver, the
// operator wrapper (phist_operator_def.hpp:84-105), orthogonalisation, GMRES
// and the Schur decompositions are PHIST's own code compiled from its
// sources; every kernel call they make lands in libphist_kernels_b200.so.
// The call sequence follows PHIST's driver drivers/subspacejada.cpp.in:155-300.
//
//   jada_run <problem> [key=value ...]
//   keys: numEigs which(SR|LR|SM|LM|TARGET) blockSize minBas maxBas convTol
//         maxIters innerSolvType(GMRES|MINRES) innerSolvMaxIters symmetry(GENERAL|HERMITIAN)
//         target arno initialShiftIters (fixed shift for the first iterations)
//         seed (start block uniform[-1,1) from this seed) sigma (SELL sigma)
//         reps (repeat the solve, report each wall time)
//         mixed=1 (FP32 correction equations through pb_mixed_jada.h; the
//         outer iteration, Rayleigh-Ritz, orthogonalisation and residuals
//         stay FP64)
//         devgmres=1 (correction equations on the library's device-resident
//         GMRES, FP64, or FP32 with mixed=1; its MINRES with
//         innerSolvType=MINRES)
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
#include "phist_jada.h"
#include "phist_enums.h"
#include "pb_mixed_jada.h"

extern "C" {
void phist_b200_Dcreate_problem(phist_DsparseMat_ptr* A, phist_const_comm_ptr comm,
                                const char* problem, int* iflag);
void phist_b200_set_sell_params(int C, int64_t sigma, int* iflag);
void phist_b200_synchronize(int* iflag);
void phist_b200_launch_count(uint64_t* count, int* iflag);
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

// uniform [-1,1) from a splitmix64 hash of (seed, index): the same numbers
// as the library's counter-based generator (pb_unif)
static uint64_t mix64(uint64_t z)
{
  z += 0x9E3779B97F4A7C15ull;
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return z ^ (z >> 31);
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
  phist_jadaOpts opts;
  phist_jadaOpts_setDefaults(&opts);
  opts.numEigs = 10;
  opts.which = phist_SR;
  opts.blockSize = 4;
  opts.minBas = 20;
  opts.maxBas = 40;
  opts.convTol = 1e-10;
  opts.maxIters = 300;
  opts.innerSolvType = phist_GMRES;
  opts.innerSolvMaxIters = 20;
  opts.symmetry = phist_HERMITIAN;
  uint64_t seed = 0;
  int64_t sigma = 1;
  int reps = 1;
  int mixed = 0, devgmres = 0;
  for (int a = 2; a < argc; a++) {
    const char* kv = argv[a];
    const char* eq = strchr(kv, '=');
    if (!eq) continue;
    std::string k(kv, eq - kv);
    const char* v = eq + 1;
    if (k == "numEigs") opts.numEigs = atoi(v);
    else if (k == "which") opts.which = str2eigSort(v);
    else if (k == "blockSize") opts.blockSize = atoi(v);
    else if (k == "minBas") opts.minBas = atoi(v);
    else if (k == "maxBas") opts.maxBas = atoi(v);
    else if (k == "convTol") opts.convTol = atof(v);
    else if (k == "maxIters") opts.maxIters = atoi(v);
    else if (k == "innerSolvType") opts.innerSolvType = str2linSolv(v);
    else if (k == "innerSolvMaxIters") opts.innerSolvMaxIters = atoi(v);
    else if (k == "symmetry") opts.symmetry = str2matSym(v);
    else if (k == "target") { opts.initialShift_r = atof(v); }
    else if (k == "arno") opts.arno = atoi(v);
    else if (k == "initialShiftIters") opts.initialShiftIters = atoi(v);
    else if (k == "seed") seed = strtoull(v, nullptr, 10);
    else if (k == "sigma") sigma = atoll(v);
    else if (k == "reps") reps = atoi(v);
    else if (k == "mixed") mixed = atoi(v);
    else if (k == "devgmres") devgmres = atoi(v);
  }

  CHK(phist_kernels_init(&argc, &argv, &iflag));
  phist_comm_ptr comm = NULL;
  CHK(phist_comm_create(&comm, &iflag));
  CHK(phist_b200_set_sell_params(32, sigma, &iflag));
  phist_DsparseMat_ptr A = NULL;
  auto t0 = std::chrono::steady_clock::now();
  iflag = sigma > 1 ? PHIST_SPARSEMAT_PERM_LOCAL : 0;
  phist_b200_Dcreate_problem(&A, comm, problem, &iflag);
  if (iflag < 0) { fprintf(stderr, "cannot create %s\n", problem); return 1; }
  const double t_create = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();

  phist_DlinearOp opA;
  CHK(phist_DlinearOp_wrap_sparseMat(&opA, A, &iflag));
  phist_const_map_ptr map = NULL;
  CHK(phist_DsparseMat_get_domain_map(A, &map, &iflag));
  phist_lidx nloc = 0;
  CHK(phist_map_get_local_length(map, &nloc, &iflag));

  pb_mixed_jada* mixedSolver = NULL;
  if (mixed || devgmres) {
    CHK(phist_b200_jada_inner_create(&mixedSolver, A, &opts, mixed ? 1 : 0, devgmres, &iflag));
    CHK(phist_b200_mixed_jada_install(mixedSolver, &opts, &iflag));
  }

  const int nEig = opts.numEigs, bs = opts.blockSize;
  const int nQ = nEig + bs - 1;
  std::vector<double> walls;
  std::vector<double> ev_out, res_out, resx_out;
  int nConv = 0, nIter = 0;
  uint64_t launches = 0;
  for (int rep = 0; rep < reps; rep++) {
    phist_Dmvec_ptr Q = NULL, v0 = NULL, res = NULL;
    phist_DsdMat_ptr R = NULL;
    CHK(phist_Dmvec_create(&Q, map, nQ, &iflag));
    CHK(phist_DsdMat_create(&R, nQ, nQ, comm, &iflag));
    CHK(phist_Dmvec_create(&v0, map, 1, &iflag));
    CHK(phist_Dmvec_create(&res, map, nQ, &iflag));
    {
      std::vector<double> h(nloc);
      for (phist_lidx i = 0; i < nloc; i++) h[i] = unif(seed, (uint64_t)i);
      CHK(phist_Dmvec_set_data(v0, h.data(), 1, 1, &iflag));
    }
    opts.v0 = v0;
    std::vector<phist_d_complex> ev(nQ);
    std::vector<double> resNorm(nQ, 0.0);
    nConv = nEig;
    nIter = opts.maxIters;
    uint64_t l0 = 0, l1 = 0;
    CHK(phist_b200_launch_count(&l0, &iflag));
    CHK(phist_b200_synchronize(&iflag));
    auto t1 = std::chrono::steady_clock::now();
    iflag = 0;
    phist_Dsubspacejada(&opA, NULL, opts, Q, R, ev.data(), resNorm.data(), &nConv, &nIter, &iflag);
    if (iflag < 0) {
      fprintf(stderr, "subspacejada returned %d\n", iflag);
      return 1;
    }
    CHK(phist_b200_synchronize(&iflag));
    walls.push_back(std::chrono::duration<double>(std::chrono::steady_clock::now() - t1).count());
    CHK(phist_b200_launch_count(&l1, &iflag));
    launches = l1 - l0;
    // explicit residuals ||A q_j - (Q R)_j|| (drivers/subspacejada.cpp.in:268-300)
    CHK(phist_DsparseMat_times_mvec(1.0, A, Q, 0.0, res, &iflag));
    CHK(phist_Dmvec_times_sdMat(-1.0, Q, R, 1.0, res, &iflag));
    std::vector<double> rn(nQ);
    CHK(phist_Dmvec_norm2(res, rn.data(), &iflag));
    ev_out.clear();
    res_out.clear();
    resx_out.clear();
    for (int j = 0; j < nConv; j++) {
      ev_out.push_back(std::real(ev[j]));
      res_out.push_back(resNorm[j]);
      resx_out.push_back(rn[j]);
    }
    CHK(phist_Dmvec_delete(res, &iflag));
    CHK(phist_Dmvec_delete(v0, &iflag));
    CHK(phist_Dmvec_delete(Q, &iflag));
    CHK(phist_DsdMat_delete(R, &iflag));
  }
  long mcalls = 0, msys = 0, munconv = 0;
  if (mixedSolver) CHK(phist_b200_mixed_jada_stats(mixedSolver, &mcalls, &msys, &munconv, &iflag));
  printf("{\"problem\": \"%s\", \"mixed\": %d, \"devgmres\": %d, \"inner_calls\": %ld, \"inner_systems\": %ld, "
         "\"inner_unconverged\": %ld, \"n\": %d, \"numEigs\": %d, \"blockSize\": %d, \"minBas\": %d, "
         "\"maxBas\": %d, \"convTol\": %.3e, \"nConv\": %d, \"nIter\": %d, \"t_create\": %.4f, "
         "\"launches\": %llu, \"wall\": [",
         problem, mixed, devgmres, mcalls, msys, munconv, nloc, nEig, bs, opts.minBas, opts.maxBas, opts.convTol, nConv, nIter, t_create,
         (unsigned long long)launches);
  for (size_t i = 0; i < walls.size(); i++) printf("%s%.6f", i ? ", " : "", walls[i]);
  printf("], \"ev\": [");
  for (size_t i = 0; i < ev_out.size(); i++) printf("%s%.17g", i ? ", " : "", ev_out[i]);
  printf("], \"resNorm\": [");
  for (size_t i = 0; i < res_out.size(); i++) printf("%s%.6e", i ? ", " : "", res_out[i]);
  printf("], \"resExplicit\": [");
  for (size_t i = 0; i < resx_out.size(); i++) printf("%s%.6e", i ? ", " : "", resx_out[i]);
  printf("]}\n");
  fflush(stdout);
  if (mixedSolver) CHK(phist_b200_mixed_jada_delete(mixedSolver, &iflag));
  CHK(phist_DsparseMat_delete(A, &iflag));
  CHK(phist_comm_delete(comm, &iflag));
  CHK(phist_kernels_finalize(&iflag));
  return 0;
}
