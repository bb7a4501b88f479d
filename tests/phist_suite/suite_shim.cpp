// Link-time pieces PHIST's kernel test suite takes from parts of PHIST that
// this library replaces or that cannot be built here.
//
// * phist_{D,S}create_matrix (src/kernels/phist_driver_utils_def.h) builds a
//   test matrix from a problem string.  The suite asks it for one problem,
//   "BENCH3D-8-A1": PHIST's 8^3 convection-diffusion benchmark from the
//   Fortran generator drivers/matfuncs/matpde3d.F90, which cannot be
//   compiled here (no Fortran compiler).  The suite only checks properties
//   on it (CARP determinism, sweeps of identity rows, operator
//   comparisons), so it gets this library's 8^3 problem of the same size
//   and pattern: the 7-point Laplacian with a random diagonal
//   (LAPDIAG3D-8-S1).  Other problem strings go to the library's generator
//   unchanged.
// * MATPDE3D_rowFunc (drivers/matfuncs/matfuncs.h), the Fortran row
//   function behind "BENCH3D", is called directly by two sparseMat tests on
//   that problem (SparseMatTest_def.hpp: compare_with_rowFunc,
//   fromRowFuncAndContext) and referenced by the complex-shift CARP tests,
//   which are compiled out without complex types.  The stand-in reports an
//   error, so those two tests fail; the Python runner lists them as
//   expected failures.
// * a crash handler that prints the call stack (below).
#include <cstdint>
#include <cstring>

extern "C" {
void phist_b200_Dcreate_problem(void** A, const void* comm, const char* problem, int* iflag);
void phist_b200_Screate_problem(void** A, const void* comm, const char* problem, int* iflag);

static const char* suite_problem(const char* problem)
{
  return std::strcmp(problem, "BENCH3D-8-A1") == 0 ? "LAPDIAG3D-8-S1" : problem;
}

void phist_Dcreate_matrix(void** A, const void* comm, const char* problem, int* iflag)
{
  phist_b200_Dcreate_problem(A, comm, suite_problem(problem), iflag);
}

void phist_Screate_matrix(void** A, const void* comm, const char* problem, int* iflag)
{
  phist_b200_Screate_problem(A, comm, suite_problem(problem), iflag);
}

int MATPDE3D_rowFunc(int64_t, int32_t*, int64_t*, void*, void*) { return -99; }
}

// A test that crashes the process shows where: on SIGSEGV/SIGBUS/SIGFPE the
// shim prints the call stack (module and offset per frame) to stderr before
// the process ends with the signal.
#include <csignal>
#include <execinfo.h>
#include <unistd.h>

namespace {
void suite_crash_trace(int sig)
{
  void* frames[64];
  const int n = backtrace(frames, 64);
  const char msg[] = "\n[suite] fatal signal, call stack:\n";
  (void)!write(2, msg, sizeof(msg) - 1);
  backtrace_symbols_fd(frames, n, 2);
  signal(sig, SIG_DFL);
  raise(sig);
}
struct SuiteCrashTrace {
  SuiteCrashTrace()
  {
    signal(SIGSEGV, suite_crash_trace);
    signal(SIGBUS, suite_crash_trace);
    signal(SIGFPE, suite_crash_trace);
  }
} suite_crash_trace_installed;
}  // namespace
