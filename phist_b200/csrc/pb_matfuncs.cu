// pb_matfuncs.cu -- seeded synthetic test problems as PHIST row functions.
//
// PHIST builds its benchmark matrices through row functions handed to
// sparseMat_create_fromRowFunc (drivers/matfuncs/, e.g. the BENCH3D family
// in matpde3d.F90, problem strings parsed in phist_driver_utils_def.h:232-470).
// Those generators seed from /dev/urandom and use octree ordering, so they are
// not reproducible; the functions here define the same physics with a
// counter-based generator (value of site i depends only on (seed, i)) and
// lexicographic ordering:
//   LAPLACE3D : 7-point Laplacian on L^3, Dirichlet, diag 6 (+ uniform[lo,hi]
//               random diagonal when hi > lo), off-diagonals -1
//   ANDERSON3D: 7-point hopping -1 on L^3 periodic, on-site uniform[-W/2,W/2]
//   HONEYCOMB : two sites per cell on Lx x Ly periodic cells, nearest-neighbour
//               hopping -1 (3 bonds per site), on-site uniform[lo,hi]
// Row entries are returned with ascending column indices.
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>

#include "pb_blas.cuh"

namespace {

struct Problem {
  int kind;        // 0 laplace3d, 1 anderson3d, 2 honeycomb
  int64_t L[3];
  double lo, hi;   // random on-site range (lo == hi: constant)
  double diag0;    // constant diagonal part
  uint64_t seed;
  int single;      // rows written as float
};

inline double site_rand(const Problem& p, int64_t i)
{
  if (p.hi == p.lo) return p.lo;
  const double u = (pb::pb_unif(p.seed, (uint64_t)i) + 1.0) * 0.5;  // [0,1)
  return p.lo + (p.hi - p.lo) * u;
}

inline void sort_row(int n, int64_t* c, double* v)
{
  for (int a = 1; a < n; a++) {
    int64_t ci = c[a];
    double vi = v[a];
    int b = a - 1;
    while (b >= 0 && c[b] > ci) {
      c[b + 1] = c[b];
      v[b + 1] = v[b];
      b--;
    }
    c[b + 1] = ci;
    v[b + 1] = vi;
  }
}

int row_of(const Problem& p, int64_t row, int32_t* len, int64_t* cols, double* v)
{
  int n = 0;
  if (p.kind == 0 || p.kind == 1) {
    const int64_t L0 = p.L[0], L1 = p.L[1], L2 = p.L[2];
    const int64_t x = row % L0, y = (row / L0) % L1, z = row / (L0 * L1);
    const bool per = (p.kind == 1);
    const int64_t d[3][2] = {{x, L0}, {y, L1}, {z, L2}};
    const int64_t stride[3] = {1, L0, L0 * L1};
    for (int a = 0; a < 3; a++) {
      const int64_t xa = d[a][0], La = d[a][1];
      for (int s = -1; s <= 1; s += 2) {
        int64_t xn = xa + s;
        if (xn < 0 || xn >= La) {
          if (!per) continue;
          xn = (xn + La) % La;
        }
        if (xn == xa) continue;  // L == 1
        cols[n] = row + (xn - xa) * stride[a];
        v[n] = -1.0;
        n++;
      }
    }
    cols[n] = row;
    v[n] = p.diag0 + site_rand(p, row);
    n++;
  } else {
    const int64_t Lx = p.L[0], Ly = p.L[1];
    const int64_t cell = row / 2, s = row % 2;
    const int64_t x = cell % Lx, y = cell / Lx;
    auto site = [&](int64_t xx, int64_t yy, int64_t ss) {
      xx = (xx % Lx + Lx) % Lx;
      yy = (yy % Ly + Ly) % Ly;
      return 2 * (xx + Lx * yy) + ss;
    };
    // A(x,y) -- B(x,y), B(x-1,y), B(x,y-1); B(x,y) -- A(x,y), A(x+1,y), A(x,y+1)
    if (s == 0) {
      cols[n++] = site(x, y, 1);
      cols[n++] = site(x - 1, y, 1);
      cols[n++] = site(x, y - 1, 1);
    } else {
      cols[n++] = site(x, y, 0);
      cols[n++] = site(x + 1, y, 0);
      cols[n++] = site(x, y + 1, 0);
    }
    for (int q = 0; q < 3; q++) v[q] = -1.0;
    cols[n] = row;
    v[n] = p.diag0 + site_rand(p, row);
    n++;
  }
  sort_row(n, cols, v);
  // merge duplicates (tiny periodic lattices)
  int m = 0;
  for (int q = 0; q < n; q++) {
    if (m > 0 && cols[m - 1] == cols[q]) {
      v[m - 1] += v[q];
    } else {
      cols[m] = cols[q];
      v[m] = v[q];
      m++;
    }
  }
  *len = m;
  return 0;
}

}  // namespace

extern "C" {

// problem description passed as the row function's last argument
struct phist_b200_problem {
  Problem p;
  int64_t nrows;
  int maxnne;
};

int phist_b200_problem_rowfunc(int64_t row, int32_t* len, int64_t* cols, void* vals, void* arg)
{
  const phist_b200_problem* pr = (const phist_b200_problem*)arg;
  if (!pr || row < 0 || row >= pr->nrows) return -1;
  double v[8];
  int e = row_of(pr->p, row, len, cols, v);
  if (pr->p.single)
    for (int q = 0; q < *len; q++) ((float*)vals)[q] = (float)v[q];
  else
    for (int q = 0; q < *len; q++) ((double*)vals)[q] = v[q];
  return e;
}

// Parse a problem string into a row-function argument:
//   "LAPLACE3D-<L>"              7-point Laplacian, Dirichlet
//   "LAPDIAG3D-<L>-S<seed>"      Laplacian + uniform[0,1] diagonal
//   "ANDERSON3D-<L>-S<seed>[-W<w>]"  periodic Anderson model, W default 16.5
//   "HONEYCOMB-<Lx>[x<Ly>]-S<seed>[-W<w>]" on-site uniform[-W/2,W/2], W default 1
// single != 0 makes the row function write float values.
// Returns a malloc'ed object (free with free()) or NULL, and fills nrows/maxnne.
void* phist_b200_problem_create(const char* str, int single, int64_t* nrows, int32_t* maxnne)
{
  if (!str) return nullptr;
  std::string s(str);
  phist_b200_problem* pr = (phist_b200_problem*)calloc(1, sizeof(phist_b200_problem));
  Problem& p = pr->p;
  p.single = single;
  auto num_after = [&](const std::string& key, double dflt) {
    size_t k = s.find(key);
    if (k == std::string::npos) return dflt;
    return atof(s.c_str() + k + key.size());
  };
  auto first_int = [&](size_t from) { return (int64_t)atoll(s.c_str() + from); };
  const size_t dash = s.find('-');
  if (dash == std::string::npos) { free(pr); return nullptr; }
  const std::string kind = s.substr(0, dash);
  p.seed = (uint64_t)num_after("-S", 0);
  if (kind == "LAPLACE3D" || kind == "LAPDIAG3D") {
    p.kind = 0;
    p.L[0] = p.L[1] = p.L[2] = first_int(dash + 1);
    p.diag0 = 6.0;
    p.lo = 0.0;
    p.hi = (kind == "LAPDIAG3D") ? 1.0 : 0.0;
    pr->nrows = p.L[0] * p.L[1] * p.L[2];
    pr->maxnne = 7;
  } else if (kind == "ANDERSON3D") {
    p.kind = 1;
    p.L[0] = p.L[1] = p.L[2] = first_int(dash + 1);
    const double W = num_after("-W", 16.5);
    p.diag0 = 0.0;
    p.lo = -W / 2;
    p.hi = W / 2;
    pr->nrows = p.L[0] * p.L[1] * p.L[2];
    pr->maxnne = 7;
  } else if (kind == "HONEYCOMB") {
    p.kind = 2;
    p.L[0] = first_int(dash + 1);
    size_t xk = s.find('x', dash + 1);
    p.L[1] = (xk != std::string::npos) ? first_int(xk + 1) : p.L[0];
    const double W = num_after("-W", 1.0);
    p.diag0 = 0.0;
    p.lo = -W / 2;
    p.hi = W / 2;
    pr->nrows = 2 * p.L[0] * p.L[1];
    pr->maxnne = 4;
  } else {
    free(pr);
    return nullptr;
  }
  if (pr->nrows <= 0) { free(pr); return nullptr; }
  if (nrows) *nrows = pr->nrows;
  if (maxnne) *maxnne = pr->maxnne;
  return pr;
}

void phist_DsparseMat_create_fromRowFunc(void** A, const void* comm, int64_t nrows, int64_t ncols,
                                         int32_t maxnne,
                                         int (*f)(int64_t, int32_t*, int64_t*, void*, void*),
                                         void* arg, int* iflag);
void phist_SsparseMat_create_fromRowFunc(void** A, const void* comm, int64_t nrows, int64_t ncols,
                                         int32_t maxnne,
                                         int (*f)(int64_t, int32_t*, int64_t*, void*, void*),
                                         void* arg, int* iflag);

// Counterpart of PHIST's driver utility create_matrix (problem string ->
// sparseMat, src/kernels/phist_driver_utils_def.h:232-470) for the problems
// above; *iflag carries the sparseMat input flags.
static void create_problem(void** A, const void* comm, const char* problem, int single, int* iflag)
{
  int64_t n = 0;
  int32_t maxnne = 0;
  void* pr = phist_b200_problem_create(problem, single, &n, &maxnne);
  if (!pr) {
    fprintf(stderr, "[phist_b200] unknown problem string '%s'\n", problem ? problem : "(null)");
    *iflag = -55;
    return;
  }
  if (single)
    phist_SsparseMat_create_fromRowFunc(A, comm, n, n, maxnne, phist_b200_problem_rowfunc, pr, iflag);
  else
    phist_DsparseMat_create_fromRowFunc(A, comm, n, n, maxnne, phist_b200_problem_rowfunc, pr, iflag);
  free(pr);
}
void phist_b200_Dcreate_problem(void** A, const void* comm, const char* problem, int* iflag)
{
  create_problem(A, comm, problem, 0, iflag);
}
void phist_b200_Screate_problem(void** A, const void* comm, const char* problem, int* iflag)
{
  create_problem(A, comm, problem, 1, iflag);
}

}  // extern "C"
