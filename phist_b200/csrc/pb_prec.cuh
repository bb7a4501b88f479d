// pb_prec.cuh -- compensated block products for PHIST_ROBUST_REDUCTIONS.
//
// PHIST's builtin library computes V'W in double-double when the caller sets
// PHIST_ROBUST_REDUCTIONS (mvec_module.F90:2421-2747 dispatching to
// gemm_kernels_sC_prec.c): orthogrrB passes the flag to every Gram product
// it needs (phist_orthogrr_def.hpp:89,152,167), and orthog then aims at
// ||Q'Q - I|| < eps*sqrt(eps) (phist_orthog_def.hpp:42-43).
//
// Here each output C(r,j) = sum_i V(i,r) W(i,j) is accumulated with Dot2
// (Ogita, Rump and Oishi, "Accurate sum and dot product", SIAM J. Sci.
// Comput. 26(6), 2005): every product is split exactly into p + e by an FMA
// (TwoProduct), p is added to the running sum with TwoSum, and the rounding
// errors of both are collected in a second accumulator.  Blocks stage row
// tiles of V and W in shared memory; each thread owns up to NQ outputs, or,
// for fewer outputs than threads, one output and a group of the tile's rows.
// Per-block (sum, error) pairs are combined by the last block to arrive, in
// block order with TwoSum, so the result does not depend on the schedule.
// Finally C = alpha*(s + c) + beta*C is evaluated in double-double and
// rounded once.
#pragma once
#include "pb_core.hpp"

namespace pb {

__device__ __forceinline__ void dd_two_sum(double a, double b, double& s, double& e)
{
  s = a + b;
  const double z = s - a;
  e = (a - (s - z)) + (b - z);
}

// s + c += x*y (one Dot2 step)
__device__ __forceinline__ void dd_dot_step(double x, double y, double& s, double& c)
{
  const double p = x * y;
  const double ep = fma(x, y, -p);
  double t, et;
  dd_two_sum(s, p, t, et);
  s = t;
  c += ep + et;
}

// (s, c) += (s2, c2)
__device__ __forceinline__ void dd_add(double& s, double& c, double s2, double c2)
{
  double t, et;
  dd_two_sum(s, s2, t, et);
  s = t;
  c += c2 + et;
}

struct MvTmvPrecArgs {
  int64_t n;
  int m, k;
  const double* V;
  int64_t ldv;
  const double* W;
  int64_t ldw;
  double alpha, beta;
  double* C;          // device, column-major, ldc
  int64_t ldc;
  double* part;       // [gridDim.x][m*k][2]
  unsigned int* counter;
};

constexpr int PREC_BS = 256;
constexpr int PREC_R = 32;  // rows per staged tile

// Thread t owns output o = t mod nout (NQ = 1, nout <= PREC_BS) and takes the
// rows g, g + G, ... of every tile, g = t / nout, G = PREC_BS / nout row
// groups; with more outputs than threads (NQ > 1) every thread owns NQ
// outputs and all rows.  The groups are combined in group order at the end.
template <int NQ>
__global__ void __launch_bounds__(PREC_BS) k_mvTmv_prec(MvTmvPrecArgs a)
{
  __shared__ double vs[PREC_R][64 + 1];
  __shared__ double ws[PREC_R][64 + 1];
  const int tid = threadIdx.x;
  const int m = a.m, k = a.k, nout = m * k;
  const int G = NQ == 1 ? PREC_BS / nout : 1;  // row groups
  const int g = NQ == 1 ? tid / nout : 0;
  const bool active = g < G;
  double s[NQ], c[NQ];
  int orow[NQ], ocol[NQ];
#pragma unroll
  for (int q = 0; q < NQ; q++) {
    s[q] = 0.0;
    c[q] = 0.0;
    const int o = NQ == 1 ? tid % nout : tid + q * PREC_BS;
    orow[q] = o < nout ? o % m : 0;
    ocol[q] = o < nout ? o / m : 0;
  }
  const int64_t ntiles = (a.n + PREC_R - 1) / PREC_R;
  for (int64_t t = blockIdx.x; t < ntiles; t += gridDim.x) {
    const int64_t i0 = t * PREC_R;
    const int rows = a.n - i0 < PREC_R ? (int)(a.n - i0) : PREC_R;
    __syncthreads();  // the previous tile has been consumed
    for (int e = tid; e < PREC_R * m; e += PREC_BS) {
      const int ii = e / m, r = e % m;
      vs[ii][r] = ii < rows ? a.V[(i0 + ii) * a.ldv + r] : 0.0;
    }
    for (int e = tid; e < PREC_R * k; e += PREC_BS) {
      const int ii = e / k, j = e % k;
      ws[ii][j] = ii < rows ? a.W[(i0 + ii) * a.ldw + j] : 0.0;
    }
    __syncthreads();
    if (active) {
      for (int ii = g; ii < rows; ii += G) {
#pragma unroll
        for (int q = 0; q < NQ; q++)
          if (NQ == 1 || tid + q * PREC_BS < nout) dd_dot_step(vs[ii][orow[q]], ws[ii][ocol[q]], s[q], c[q]);
      }
    }
  }
  if (NQ == 1 && G > 1) {
    // row groups of one output, combined in group order
    double* red = &vs[0][0];  // 2*PREC_BS <= PREC_R*65 entries
    __syncthreads();
    red[2 * tid] = s[0];
    red[2 * tid + 1] = c[0];
    __syncthreads();
    if (tid < nout) {
      double ss = 0.0, cc = 0.0;
      for (int q = 0; q < G; q++) dd_add(ss, cc, red[2 * (q * nout + tid)], red[2 * (q * nout + tid) + 1]);
      s[0] = ss;
      c[0] = cc;
    }
  }
  double* part = a.part + (int64_t)blockIdx.x * nout * 2;
#pragma unroll
  for (int q = 0; q < NQ; q++) {
    const int o = tid + q * PREC_BS;
    if (o < nout && (NQ > 1 || g == 0)) {
      part[2 * o] = s[q];
      part[2 * o + 1] = c[q];
    }
  }
  __shared__ bool am_last;
  __threadfence();
  __syncthreads();
  if (tid == 0) am_last = (atomicAdd(a.counter, 1u) == gridDim.x - 1);
  __syncthreads();
  if (!am_last) return;
  __threadfence();
  for (int o = tid; o < nout; o += PREC_BS) {
    double ss = 0.0, cc = 0.0;
    for (int b = 0; b < (int)gridDim.x; b++) {
      const double* pb = a.part + (int64_t)b * nout * 2;
      dd_add(ss, cc, __ldcg(pb + 2 * o), __ldcg(pb + 2 * o + 1));
    }
    // alpha*(ss + cc) + beta*C in double-double, rounded once
    const int r = o % m, j = o / m;
    double* cp = a.C + r + (int64_t)j * a.ldc;
    const double p = a.alpha * ss;
    double ep = fma(a.alpha, ss, -p) + a.alpha * cc;
    double qv = 0.0, eq = 0.0;
    if (a.beta != 0.0) {
      qv = a.beta * *cp;
      eq = fma(a.beta, *cp, -qv);
    }
    double t, et;
    dd_two_sum(p, qv, t, et);
    *cp = t + (et + ep + eq);
  }
  if (tid == 0) *a.counter = 0u;
}

}  // namespace pb
