// pb_gmres.cu -- device-resident GMRES for the Jacobi-Davidson correction
// equations.
//
// PHIST's subspacejada solves, per outer iteration, k correction equations
//     (I - Q Q')(A - sigma_j I) t_j = r_j
// with its blocked GMRES (src/jada/phist_jadaCorrectionSolver_def.hpp:372-
// 583; src/krylov/phist_blockedgmres_def.hpp).  There every Arnoldi step
// orthogonalises by iterated modified Gram-Schmidt, one mvec_dot_mvec per
// previous basis block, each a host round trip, and the Hessenberg matrix
// and Givens rotations live on the host.  Here the k systems run as k
// columns of one block: every basis block V_i is a contiguous n x k array,
// the Hessenberg matrices, rotations and residual estimates stay on the
// device, and the Gram-Schmidt step is classical with selective
// reorthogonalisation in row-parallel kernels (see k_gm_blk).  An iteration
// is ~10 asynchronous launches with no host synchronisation; after each step
// the host looks (without waiting) at a step counter and converged count the
// device writes into mapped host memory, and stops launching once every
// system has converged.
//
// The arithmetic of the GMRES iterate is PHIST's: x_0 = 0, Krylov space of
// the projected operator, Givens-rotated least squares; convergence when
// |g_{j+1}| < 1000 eps (absolute) or |g_{j+1}| / ||r_j|| < tol_j
// (phist_blockedgmres_def.hpp:604-606); restart after maxBas steps with the
// current iterate; at most maxIter steps in all; the solutions returned with
// unit norm (phist_jadaCorrectionSolver_def.hpp:576-578).  The small dense
// part (Hessenberg, rotations, triangular solve) is FP64 in both precisions.
//
// MINRES (phist_b200_{D,S}jadaCorrection_minres) is the same solver with
// PHIST's blocked MINRES step (src/krylov/phist_blockedminres_def.hpp:
// 185-277) in place of the Gram-Schmidt step: the Lanczos three-term
// recurrence alpha = V_j'W, W -= alpha V_j + beta V_{j-1} with beta the
// previous step's norm, beta' = ||W||, so H is tridiagonal and a step costs
// two passes over W whatever its index; the basis is kept (PHIST's ring
// buffer) for the update of the iterate, the rotations, least squares and
// restarts are GMRES's, and the absolute threshold is 100 eps
// (blockedminres_def.hpp:157).  For symmetric A and real shifts only, as in
// PHIST.
#include <algorithm>
#include <atomic>
#include <cmath>
#include <limits>
#include <vector>

#include "pb_api.cuh"

namespace pb {
namespace {

// per-system values passed by value to the small kernels (k <= 32)
struct GmIndex {
  int v[32];
};
struct GmTol {
  double v[32];
};

template <class T>
struct DBuf {
  T* p = nullptr;
  explicit DBuf(size_t count) { p = (T*)rt().dmalloc(sizeof(T) * (count ? count : 1)); }
  ~DBuf() { rt().dfree(p); }
  DBuf(const DBuf&) = delete;
  DBuf& operator=(const DBuf&) = delete;
};

template <class T>
void raw_view(Mvec<T>& m, T* d, int64_t n, int w, int64_t ld)
{
  m.map = nullptr;
  m.nrows = (int32_t)n;
  m.nvec = w;
  m.lda = ld;
  m.root = &m;
  m.col_off = 0;
  m.d_base = d;
  m.h_base = nullptr;
}

// dst(i, s) = src(i, s) * f[s]
template <class T>
__global__ void k_gm_scale_cols(const T* __restrict__ src, int64_t lds, T* dst, int64_t ldd, int64_t n, int k,
                                const T* __restrict__ f)
{
  PB_FOR_ELEMS(n, k, i, s) dst[i * ldd + s] = src[i * lds + s] * f[s];
}

// B(:, s) = R(:, idx[s]) (the right-hand sides in system order)
template <class T>
__global__ void k_gm_gather_cols(const T* __restrict__ R, int64_t ldr, T* B, int64_t n, int k, GmIndex idx)
{
  PB_FOR_ELEMS(n, k, i, s) B[i * k + s] = R[i * ldr + idx.v[s]];
}

// zero the columns of converged systems
template <class T>
__global__ void k_gm_mask_cols(T* W, int64_t n, int k, const int* __restrict__ conv)
{
  PB_FOR_ELEMS(n, k, i, s) if (conv[s]) W[i * k + s] = T(0);
}

// Start of a cycle: beta_s = ||r_s|| from the diagonal of R'R; g = beta e_1;
// f = 1/beta.  On the first cycle beta is the reference norm of the
// relative test.  A system whose start residual already passes the test is
// converged with no step.
template <class T>
__global__ void k_gm_start(const T* __restrict__ G, int k, int m, double* g, double* bnorm, T* f, int* conv,
                           int* jcount, int first, double eps_abs, GmTol tol)
{
  const int s = threadIdx.x;
  if (s >= k) return;
  const double beta = sqrt(fmax((double)G[s + s * k], 0.0));
  if (first) {
    bnorm[s] = beta;
    jcount[s] = 0;
    conv[s] = (beta < eps_abs) ? 1 : 0;
  }
  for (int i = 0; i <= m; i++) g[i * k + s] = 0.0;
  g[s] = conv[s] ? 0.0 : beta;
  if (!first) jcount[s] = 0;
  f[s] = (beta > 0.0 && !conv[s]) ? (T)(1.0 / beta) : T(0);
  (void)tol;
}

// After W is orthogonal to V_0..V_j: h(j+1, j, s) = ||w_s|| (diagonal of
// W'W), the earlier rotations applied to column j of H(:, :, s), a new
// rotation zeroing h(j+1, j), the residual estimate |g_{j+1}| and the
// convergence test; f_s = 1/h(j+1, j, s) for the next basis block.  Thread
// 0 then publishes (number converged, j) in mapped host memory, the count
// first.
template <class T>
__global__ void k_gm_step(const T* __restrict__ G, int gstride, int j, int k, int m, double* H, double* cs, double* sn,
                          double* g, const double* __restrict__ bnorm, T* f, int* conv, int* jcount, double eps_abs,
                          GmTol tol, volatile int* flags)
{
  const int s = threadIdx.x;
  __shared__ int nconv;
  if (s == 0) nconv = 0;
  __syncthreads();
  if (s < k) {
    const double hn = sqrt(fmax((double)G[s * gstride], 0.0));
    auto Hat = [&](int i) -> double& { return H[((int64_t)i * m + j) * k + s]; };
    // column j of H and the earlier rotations, all loads issued before the
    // dependent chain of rotations
    double hc[64], rc[64], rs[64];
    for (int i = 0; i <= j; i++) hc[i] = Hat(i);
    for (int i = 0; i < j; i++) {
      rc[i] = cs[i * k + s];
      rs[i] = sn[i * k + s];
    }
    for (int i = 0; i < j; i++) {
      const double a = hc[i], b = hc[i + 1];
      hc[i] = rc[i] * a + rs[i] * b;
      hc[i + 1] = -rs[i] * a + rc[i] * b;
    }
    for (int i = 0; i < j; i++) Hat(i) = hc[i];
    const double a = hc[j];
    double c = 1.0, sn_ = 0.0;
    const double r = hypot(a, hn);
    if (r > 0.0) {
      c = a / r;
      sn_ = hn / r;
    }
    cs[j * k + s] = c;
    sn[j * k + s] = sn_;
    Hat(j) = r;
    H[((int64_t)(j + 1) * m + j) * k + s] = 0.0;
    const double gj = g[j * k + s];
    g[j * k + s] = c * gj;
    g[(j + 1) * k + s] = -sn_ * gj;
    if (!conv[s]) {
      jcount[s] = j + 1;
      const double res = fabs(g[(j + 1) * k + s]);
      if (res < eps_abs || (bnorm[s] > 0.0 && res / bnorm[s] < tol.v[s])) conv[s] = 1;
    }
    f[s] = (hn > 0.0) ? (T)(1.0 / hn) : T(0);
    if (conv[s]) atomicAdd(&nconv, 1);
  }
  __syncthreads();
  if (s == 0) {
    flags[1] = nconv;
    __threadfence_system();
    flags[0] = j;
  }
}

// y_s = H(0:J_s, 0:J_s, s)^{-1} g(0:J_s, s), J_s = jcount[s], stored
// negated as update coefficients: Y[i*k + s] = -y_s(i) for i < J_s, 0 up to
// Jmax (x -= sum_i V_i Y_i is then x += V y).
template <class T>
__global__ void k_gm_solve(const double* __restrict__ H, const double* __restrict__ g, const int* __restrict__ jcount,
                           int k, int m, int Jmax, T* Y)
{
  const int s = threadIdx.x;
  if (s >= k) return;
  for (int i = 0; i < Jmax; i++) Y[i * k + s] = T(0);
  const int J = jcount[s];
  double y[64];
  for (int i = J - 1; i >= 0; i--) {
    double v = g[i * k + s];
    for (int l = i + 1; l < J; l++) v -= H[((int64_t)i * m + l) * k + s] * y[l];
    const double d = H[((int64_t)i * m + i) * k + s];
    y[i] = (d != 0.0) ? v / d : 0.0;
  }
  for (int i = 0; i < J; i++) Y[i * k + s] = (T)(-y[i]);
}

// 1/||x_s|| from the diagonal of X'X (0 for a zero column)
template <class T>
__global__ void k_gm_invnorm(const T* __restrict__ G, int k, T* f)
{
  const int s = threadIdx.x;
  if (s >= k) return;
  const double nr = sqrt(fmax((double)G[s + s * k], 0.0));
  f[s] = nr > 0.0 ? (T)(1.0 / nr) : T(0);
}

// Row-parallel Gram-Schmidt kernel over the basis blocks V_i, i in [i0, i1)
// (at most MJ <= GM_MAXJ of them, held in registers), V_i = V + i*n*k, each n x k contiguous.
// Thread (row r, system s), s = tid % KP (KP = k rounded up to a power of
// two): a warp covers 32/KP consecutive rows, so every load of V_i or W is
// one contiguous segment.
//   UPD:  w_s <- w_s - sum_i V_i(r, s) h[i*k + s]
//   DOTS: out[i*k + s] = sum_r V_i(r, s) w_s(r) (w after the update, from
//         the same loads of V), i in [i0, i1), at out + i0*k
//   always: ||w_s||^2 after the update, at out + i1*k (DOTS) or out (not)
// skip (may be NULL): the kernel does nothing when *skip == 0.
// Sums: butterfly over the lanes of one system, warps in order, then the
// fixed-order last-block pass: bitwise reproducible.
constexpr int GM_MAXJ = 16;
constexpr int GM_MAXOUT = 256;

template <class T, bool UPD, bool DOTS, int MJ>
__global__ void __launch_bounds__(256) k_gm_blk(int64_t n, int k, int kp, int i0, int i1, const T* __restrict__ V,
                                                T* W, const T* __restrict__ h, const int* __restrict__ skip, T* part,
                                                unsigned int* counter, T* out, int ext)
{
  if (skip && *skip == 0) return;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int s = tid % kp, nb = i1 - i0;
  const int nout = (DOTS ? nb + 1 : 1) * k;
  const int64_t nk = n * (int64_t)k;
  T hc[MJ], acc[MJ];
#pragma unroll
  for (int i = 0; i < MJ; i++) {
    hc[i] = (UPD && i < nb && s < k) ? h[(i0 + i) * k + s] : T(0);
    acc[i] = T(0);
  }
  T nacc = T(0);
  if (s < k) {
    const int64_t rstep = (int64_t)gridDim.x * (256 / kp);
    for (int64_t r = blockIdx.x * (int64_t)(256 / kp) + tid / kp; r < n; r += rstep) {
      const T* vr = V + (int64_t)i0 * nk + r * k + s;
      T v[MJ];
#pragma unroll
      for (int i = 0; i < MJ; i++) v[i] = (i < nb) ? vr[(int64_t)i * nk] : T(0);
      T w = W[r * k + s];
      if (UPD) {
#pragma unroll
        for (int i = 0; i < MJ; i++) w -= v[i] * hc[i];
        W[r * k + s] = w;
      }
      if (DOTS) {
#pragma unroll
        for (int i = 0; i < MJ; i++) acc[i] += v[i] * w;
      }
      nacc += w * w;
    }
  }
#pragma unroll
  for (int off = 16; off >= 1; off >>= 1) {
    if (off < kp) break;
#pragma unroll
    for (int i = 0; i < MJ; i++)
      if (DOTS && i < nb) acc[i] += __shfl_xor_sync(0xffffffffu, acc[i], off);
    nacc += __shfl_xor_sync(0xffffffffu, nacc, off);
  }
  __shared__ T red[8][GM_MAXOUT];
  if (lane < kp && s < k) {
    if (DOTS) {
#pragma unroll
      for (int i = 0; i < MJ; i++)
        if (i < nb) red[warp][i * k + s] = acc[i];
      red[warp][nb * k + s] = nacc;
    } else {
      red[warp][s] = nacc;
    }
  }
  __syncthreads();
  for (int o = tid; o < nout; o += 256) {
    T a = T(0);
    for (int w8 = 0; w8 < 8; w8++) a += red[w8][o];
    part[(int64_t)blockIdx.x * nout + o] = a;
  }
  if (ext) return;  // second pass: k_reduce_partials
  last_block_reduce<T>(part, nout, gridDim.x, counter, out + (DOTS ? (int64_t)i0 * k : 0), 1, nout, 0, T(1), T(0));
}

// After pass 1: O1 = (h1, ||w||^2 before), O2 = (h2, ||w||^2 after).  H(:, j)
// = h1 (+ h2 when a second pass follows).  The second pass runs (flag 1)
// when some system's norm fell below 1/sqrt(2) of its value before the
// pass (the "twice is enough" test); otherwise Nf takes the norms after
// pass 1 and the second-pass kernel is skipped.
template <class T>
__global__ void k_gm_decide(const T* __restrict__ O1, const T* __restrict__ O2, int J, int k, int m, int j, double* H,
                            T* Nf, int* reorth)
{
  __shared__ int any;
  const int s = threadIdx.x;
  if (s == 0) any = 0;
  __syncthreads();
  if (s < k) {
    const double before = (double)O1[J * k + s], after = (double)O2[J * k + s];
    if (after < 0.5 * before) atomicOr(&any, 1);
  }
  __syncthreads();
  if (s < k) {
    for (int i = 0; i < J; i++)
      H[((int64_t)i * m + j) * k + s] = (double)O1[i * k + s] + (any ? (double)O2[i * k + s] : 0.0);
    if (!any) Nf[s] = O2[J * k + s];
  }
  if (s == 0) *reorth = any;
}

// Lanczos step j (MINRES): alpha_s = V_j'w_s from the dots at O1 + j*k,
// beta_s = the previous step's unrotated norm h(j, j-1) = sqrt(Nf_s) (read
// before this step's update overwrites Nf); column j of H is 0 above j-1,
// beta at j-1, alpha at j, and the update coefficients of V_{j-1}, V_j are
// hL[(j-1)*k + s] = beta, hL[j*k + s] = alpha
template <class T>
__global__ void k_lz_coef(const T* __restrict__ O1, const T* __restrict__ Nf, int j, int k, int m, double* H, T* hL)
{
  const int s = threadIdx.x;
  if (s >= k) return;
  const double alpha = (double)O1[j * k + s];
  const double beta = j > 0 ? sqrt(fmax((double)Nf[s], 0.0)) : 0.0;
  for (int i = 0; i + 1 < j; i++) H[((int64_t)i * m + j) * k + s] = 0.0;
  if (j > 0) {
    H[((int64_t)(j - 1) * m + j) * k + s] = beta;
    hL[(j - 1) * k + s] = (T)beta;
  }
  H[((int64_t)j * m + j) * k + s] = alpha;
  hL[j * k + s] = (T)alpha;
}

// MINRES step with the projection P = I - Q Q' fused into its two passes
// (thread per (row, system) as k_gm_blk; Q n x nq, nq <= MQ, row-major with
// leading dimension ldq):
//   DOTS: out[i*k + s] = sum_r Q(r, i) w_s(r) (i < nq), out[nq*k + s] =
//         sum_r V_j(r, s) w_s(r): the projection's Q'W and alpha from one
//         read of W (alpha = V_j'W equals V_j'(P W) because V_j is
//         orthogonal to Q)
//   UPD:  w_s -= sum_i Q(r, i) c(i, s), then -= alpha_s V_j(r, s), then
//         -= beta_s V_{j-1}(r, s) (PHIST's order: the operator's projection,
//         then the Lanczos terms), out[s] = ||w_s||^2; coef = [c (nq*k) |
//         alpha (k) | beta (k)]
// Sums as in k_gm_blk (butterfly, warps in order, fixed-order last pass).
template <class T, bool UPD, int MQ>
__global__ void __launch_bounds__(256) k_lz_proj(int64_t n, int k, int kp, int nq, const T* __restrict__ Q,
                                                 int64_t ldq, const T* __restrict__ Vj, const T* __restrict__ Vjm1,
                                                 T* W, const T* __restrict__ coef, T* part, unsigned int* counter,
                                                 T* out, int ext)
{
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int s = tid % kp;
  const int nout = UPD ? k : (nq + 1) * k;
  T cq[MQ], acc[MQ];
  T ca = T(0), cb = T(0), aacc = T(0), nacc = T(0);
#pragma unroll
  for (int i = 0; i < MQ; i++) {
    cq[i] = (UPD && i < nq && s < k) ? coef[i * k + s] : T(0);
    acc[i] = T(0);
  }
  if (UPD && s < k) {
    ca = coef[nq * k + s];
    cb = Vjm1 ? coef[(nq + 1) * k + s] : T(0);
  }
  if (s < k) {
    const int64_t rstep = (int64_t)gridDim.x * (256 / kp);
    for (int64_t r = blockIdx.x * (int64_t)(256 / kp) + tid / kp; r < n; r += rstep) {
      T q[MQ];
#pragma unroll
      for (int i = 0; i < MQ; i++) q[i] = (i < nq) ? Q[r * ldq + i] : T(0);
      const T v = Vj[r * k + s];
      T w = W[r * k + s];
      if (UPD) {
#pragma unroll
        for (int i = 0; i < MQ; i++) w -= q[i] * cq[i];
        w -= v * ca;
        if (Vjm1) w -= Vjm1[r * k + s] * cb;
        W[r * k + s] = w;
        nacc += w * w;
      } else {
#pragma unroll
        for (int i = 0; i < MQ; i++) acc[i] += q[i] * w;
        aacc += v * w;
      }
    }
  }
#pragma unroll
  for (int off = 16; off >= 1; off >>= 1) {
    if (off < kp) break;
    if (UPD) {
      nacc += __shfl_xor_sync(0xffffffffu, nacc, off);
    } else {
#pragma unroll
      for (int i = 0; i < MQ; i++)
        if (i < nq) acc[i] += __shfl_xor_sync(0xffffffffu, acc[i], off);
      aacc += __shfl_xor_sync(0xffffffffu, aacc, off);
    }
  }
  __shared__ T red[8][GM_MAXOUT];
  if (lane < kp && s < k) {
    if (UPD) {
      red[warp][s] = nacc;
    } else {
#pragma unroll
      for (int i = 0; i < MQ; i++)
        if (i < nq) red[warp][i * k + s] = acc[i];
      red[warp][nq * k + s] = aacc;
    }
  }
  __syncthreads();
  for (int o = tid; o < nout; o += 256) {
    T a = T(0);
    for (int w8 = 0; w8 < 8; w8++) a += red[w8][o];
    part[(int64_t)blockIdx.x * nout + o] = a;
  }
  if (ext) return;  // second pass: k_reduce_partials
  last_block_reduce<T>(part, nout, gridDim.x, counter, out, 1, nout, 0, T(1), T(0));
}

// Lanczos coefficients of the fused step: alpha_s = O[nq*k + s], beta_s =
// sqrt(Nf_s) of the previous step (j > 0); column j of H as k_lz_coef;
// beta stored at O[(nq+1)*k + s] for the update pass
template <class T>
__global__ void k_lz_coef_proj(T* O, int nq, const T* __restrict__ Nf, int j, int k, int m, double* H)
{
  const int s = threadIdx.x;
  if (s >= k) return;
  const double alpha = (double)O[nq * k + s];
  const double beta = j > 0 ? sqrt(fmax((double)Nf[s], 0.0)) : 0.0;
  for (int i = 0; i + 1 < j; i++) H[((int64_t)i * m + j) * k + s] = 0.0;
  if (j > 0) H[((int64_t)(j - 1) * m + j) * k + s] = beta;
  H[((int64_t)j * m + j) * k + s] = alpha;
  O[(nq + 1) * k + s] = (T)beta;
}

// out[o] = sum over blocks of part[b*nout + o] (k_reduce_partials) unless
// *skip == 0
template <class T>
__global__ void __launch_bounds__(256) k_gm_reduce_if(const T* __restrict__ part, int nblocks, int nout, T* out,
                                                      const int* __restrict__ skip)
{
  if (skip && *skip == 0) return;
  k_reduce_partials_body<T>(part, nblocks, nout, out, nout, 0, T(1), T(0));
}

// resident 256-thread blocks per SM of one k_gm_blk instantiation (queried
// once)
template <class T, bool UPD, bool DOTS, int MJ>
int gm_occ()
{
  static std::atomic<int> occ{0};  // lanes on several threads may ask at once
  int o = occ.load(std::memory_order_relaxed);
  if (o == 0) {
    int b = 0;
    PB_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, k_gm_blk<T, UPD, DOTS, MJ>, 256, 0));
    o = std::max(1, b);
    occ.store(o, std::memory_order_relaxed);
  }
  return o;
}

// Blocks per launch of k_gm_blk for k systems
inline int gm_chunk(int k) { return std::max(1, std::min(GM_MAXJ, GM_MAXOUT / k - 1)); }

// one launch of k_gm_blk over the blocks [i0, i1)
template <class T, bool UPD, bool DOTS>
void gm_blk(int64_t n, int k, int i0, int i1, const T* V, T* W, const T* h, const int* skip, T* out)
{
  const int kp = k <= 1 ? 1 : k <= 2 ? 2 : k <= 4 ? 4 : k <= 8 ? 8 : k <= 16 ? 16 : 32;
  const int nout = (DOTS ? i1 - i0 + 1 : 1) * k;
  T* dst = out + (DOTS ? (int64_t)i0 * k : 0);
  // the fewest register-held blocks that cover this launch; one wave of
  // resident blocks, each thread walking several rows, so that few partial
  // sums are left; many partials go to the GPU-wide second pass
  const int nb = i1 - i0;
  auto launch = [&](auto kern, int occ) {
    const int grid = (int)std::max<int64_t>(1, std::min<int64_t>(ceil_div(n, 256 / kp), (int64_t)rt().num_sms() * occ));
    const int ext = (nout >= 32 && grid > 32) ? 1 : 0;
    T* part = (T*)rt().scratch(sizeof(T) * (size_t)grid * nout);
    kern<<<grid, 256, 0, stream()>>>(n, k, kp, i0, i1, V, W, h, skip, part, rt().counters(), out, ext);
    PB_LAUNCH_CHECK();
    if (ext) {
      // skipped passes leave their partials unread: k_gm_reduce_if checks the flag too
      k_gm_reduce_if<T><<<(nout + 31) / 32, 256, 0, stream()>>>(part, grid, nout, dst, skip);
      PB_LAUNCH_CHECK();
    }
  };
  if (nb <= 4) launch(k_gm_blk<T, UPD, DOTS, 4>, gm_occ<T, UPD, DOTS, 4>());
  else if (nb <= 8) launch(k_gm_blk<T, UPD, DOTS, 8>, gm_occ<T, UPD, DOTS, 8>());
  else launch(k_gm_blk<T, UPD, DOTS, 16>, gm_occ<T, UPD, DOTS, 16>());
}

// out[i*k + s] = V_i' w_s for i < J and out[J*k + s] = ||w_s||^2, over
// chunks of blocks in ascending order (a chunk's norm lands where the next
// chunk's dots go and is overwritten by them; the last one stays)
template <class T>
void gm_dots(int64_t n, int k, int J, const T* V, T* W, T* out)
{
  const int cj = gm_chunk(k);
  for (int i0 = 0; i0 < J; i0 += cj) gm_blk<T, false, true>(n, k, i0, std::min(J, i0 + cj), V, W, nullptr, nullptr, out);
}

// w -= sum_{i<J} V_i h_i; ||w||^2 into nrm
template <class T>
void gm_update(int64_t n, int k, int J, const T* V, T* W, const T* h, const int* skip, T* nrm)
{
  const int cj = gm_chunk(k);
  for (int i0 = 0; i0 < J; i0 += cj) gm_blk<T, true, false>(n, k, i0, std::min(J, i0 + cj), V, W, h, skip, nrm);
}

// one launch of k_lz_proj (MQ: nq rounded up to 4, 8, 16 or 32)
template <class T, bool UPD>
void lz_proj(int64_t n, int k, int nq, const T* Q, int64_t ldq, const T* Vj, const T* Vjm1, T* W, const T* coef,
             T* out)
{
  const int kp = k <= 1 ? 1 : k <= 2 ? 2 : k <= 4 ? 4 : k <= 8 ? 8 : k <= 16 ? 16 : 32;
  const int nout = UPD ? k : (nq + 1) * k;
  auto launch = [&](auto kern, std::atomic<int>& occ) {
    if (occ.load() == 0) {
      int b = 0;
      PB_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, kern, 256, 0));
      occ.store(std::max(1, b));
    }
    const int grid = (int)std::max<int64_t>(1, std::min<int64_t>(ceil_div(n, 256 / kp), (int64_t)rt().num_sms() * occ.load()));
    const int ext = (nout >= 32 && grid > 32) ? 1 : 0;
    T* part = (T*)rt().scratch(sizeof(T) * (size_t)grid * nout);
    kern<<<grid, 256, 0, stream()>>>(n, k, kp, nq, Q, ldq, Vj, Vjm1, W, coef, part, rt().counters(), out, ext);
    PB_LAUNCH_CHECK();
    if (ext) {
      k_gm_reduce_if<T><<<(nout + 31) / 32, 256, 0, stream()>>>(part, grid, nout, out, nullptr);
      PB_LAUNCH_CHECK();
    }
  };
  static std::atomic<int> occ[4];
  if (nq <= 4) launch(k_lz_proj<T, UPD, 4>, occ[0]);
  else if (nq <= 8) launch(k_lz_proj<T, UPD, 8>, occ[1]);
  else if (nq <= 16) launch(k_lz_proj<T, UPD, 16>, occ[2]);
  else launch(k_lz_proj<T, UPD, 32>, occ[3]);
}

}  // namespace

// W = alpha V C + beta W on device operands (C col-major m x k, ld ldc)
template <class T>
static void gm_mvsd(int64_t n, int m, int k, T alpha, const T* V, int64_t ldv, const T* C, int64_t ldc, T beta, T* W,
                    int64_t ldw)
{
  RowGemmArgs<T> a = rowgemm_args<T>();
  a.n = n;
  a.m = m;
  a.k = k;
  a.mv = 0;
  a.V = V;
  a.ldv = ldv;
  a.W = W;
  a.ldw = ldw;
  a.C = C;
  a.ldc = ldc;
  a.alpha = alpha;
  a.beta = beta;
  a.mode = RM_MVSD;
  a.gram = GM_NONE;
  launch_rowgemm<T>(a);
}

// lanczos: MINRES (three-term recurrence), else GMRES
template <class T>
int jada_krylov(const SparseMat<T>* A, const Mvec<T>* Q, const Mvec<T>* R, const int* resIndex, int k,
                const double* sigma, const double* tol, int maxIter, int maxBas, Mvec<T>* t, bool lanczos)
{
  PB_REQUIRE(A && R && t && sigma && tol, PB_INVALID_INPUT, "NULL argument");
  PB_REQUIRE(k >= 1 && k <= 32, PB_INVALID_INPUT, "1..32 systems per call (got %d)", k);
  PB_REQUIRE(t->nvec == k, PB_INVALID_INPUT, "t has %d columns, expected %d", t->nvec, k);
  PB_REQUIRE(maxIter >= 1, PB_INVALID_INPUT, "maxIter must be >= 1");
  const int64_t n = A->nrows;
  PB_REQUIRE(A->ncols == n && R->nrows == n && t->nrows == n && (!Q || Q->nrows == n), PB_INVALID_INPUT,
             "operand rows do not match the matrix");
  for (int s = 0; s < k; s++) {
    const int idx = resIndex ? resIndex[s] : s;
    PB_REQUIRE(idx >= 0 && idx < R->nvec, PB_INVALID_INPUT, "resIndex[%d] = %d out of range", s, idx);
  }
  const int nq = Q ? Q->nvec : 0;
  const int m = std::max(1, std::min(std::min(maxBas > 0 ? maxBas : maxIter, maxIter), 63));
  const int64_t nk = n * (int64_t)k;  // one basis block
  const double eps_abs = (lanczos ? 100.0 : 1000.0) * std::numeric_limits<T>::epsilon();

  DBuf<T> V((size_t)nk * (m + 1)), B((size_t)nk), X((size_t)nk), W((size_t)nk);
  DBuf<T> Y((size_t)(m + 1) * k), Cq((size_t)std::max(nq, 1) * k), dummy(k);
  DBuf<T> Gk((size_t)k * k), f(k);
  DBuf<double> H((size_t)(m + 1) * m * k), cs((size_t)m * k), sn((size_t)m * k), g((size_t)(m + 1) * k), bnorm(k);
  DBuf<int> conv(k), jcount(k), reorth(1);
  DBuf<T> O1((size_t)(m + 2) * k), O2((size_t)(m + 2) * k), Nf(k), hL((size_t)(m + 1) * k);
  // MINRES with a projection block of at most 32 columns: the projection is
  // fused into the two Lanczos passes (k_lz_proj); P1 = [Q'W | alpha | beta]
  const bool fuse = lanczos && nq > 0 && nq <= 32 && (nq + 1) * k <= GM_MAXOUT;
  DBuf<T> P1((size_t)(nq + 2) * k);
  GmIndex gi;
  GmTol gt;
  for (int s = 0; s < k; s++) {
    gi.v[s] = resIndex ? resIndex[s] : s;
    gt.v[s] = tol[s];
  }
  std::vector<T> negsig(k);
  for (int s = 0; s < k; s++) negsig[s] = (T)(-sigma[s]);
  volatile int* hflags = (volatile int*)rt().mailbox_host();
  int* dflags = (int*)rt().mailbox_dev();
  const int gw = grid_for(n * (int64_t)k);

  Mvec<T> mX, mW, mVj;
  raw_view(mX, X.p, n, k, k);
  raw_view(mW, W.p, n, k, k);

  // W = P W with P = I - Q Q'
  auto project = [&]() {
    if (nq == 0) return;
    launch_mvTmv<T>(n, nq, k, T(1), Q->d(), Q->lda, W.p, k, T(0), Cq.p, nq);
    gm_mvsd<T>(n, nq, k, T(-1), Q->d(), Q->lda, Cq.p, nq, T(1), W.p, k);
  };
  // G = M'M for an n x k block (only the diagonal is used)
  auto gram = [&](const T* M) { launch_mvTmv<T>(n, k, k, T(1), M, k, M, k, T(0), Gk.p, k); };

  k_gm_gather_cols<T><<<gw, 256, 0, stream()>>>(R->d(), R->lda, B.p, n, k, gi);
  PB_LAUNCH_CHECK();
  k_put_value<T><<<gw, 256, 0, stream()>>>(X.p, k, n, k, T(0));
  PB_LAUNCH_CHECK();
  PB_CUDA(cudaMemcpyAsync(W.p, B.p, sizeof(T) * (size_t)n * k, cudaMemcpyDeviceToDevice, stream()));

  int total = 0, nconv = 0;
  for (int cycle = 0; total < maxIter && nconv < k; cycle++) {
    if (cycle > 0) {
      // restart from the current iterate: W = B - P (A - sigma I) X, converged systems masked
      spmv_general<T>(T(1), A, negsig.data(), &mX, T(0), &mW, nullptr, nullptr, T(0), T(0), nullptr);
      project();
      k_axpby<T><<<gw, 256, 0, stream()>>>(B.p, k, W.p, k, n, k, T(1), nullptr, T(-1));
      PB_LAUNCH_CHECK();
      k_gm_mask_cols<T><<<gw, 256, 0, stream()>>>(W.p, n, k, conv.p);
      PB_LAUNCH_CHECK();
    }
    gram(W.p);
    k_gm_start<T><<<1, 32, 0, stream()>>>(Gk.p, k, m, g.p, bnorm.p, f.p, conv.p, jcount.p, cycle == 0 ? 1 : 0,
                                          eps_abs, gt);
    PB_LAUNCH_CHECK();
    k_gm_scale_cols<T><<<gw, 256, 0, stream()>>>(W.p, k, V.p, k, n, k, f.p);
    PB_LAUNCH_CHECK();
    hflags[1] = 0;
    hflags[0] = -1;
    int j = 0, steps = 0;
    const int jmax = std::min(m, maxIter - total);
    bool stop = false;
    for (j = 0; j < jmax && !stop; j++) {
      // W = P (A - sigma I) V_j
      raw_view(mVj, V.p + (int64_t)j * nk, n, k, k);
      spmv_general<T>(T(1), A, negsig.data(), &mVj, T(0), &mW, nullptr, nullptr, T(0), T(0), nullptr);
      if (!fuse) project();
      // Gram-Schmidt against V_0..V_j: h1 = V'W and ||W||^2; W -= V h1,
      // then h2 = V'W and ||W||^2 of the result (in one pass while the
      // blocks fit one launch); a second subtraction only where a norm fell
      // below 1/sqrt(2) of its value before (a device flag the second-pass
      // kernels read)
      const int J = j + 1;
      if (fuse) {
        // [Q V_j]'W in one pass; W -= Q (Q'W) + V_j alpha + V_{j-1} beta and
        // ||W||^2 into Nf in the next
        const T* vj = V.p + (int64_t)j * nk;
        lz_proj<T, false>(n, k, nq, Q->d(), Q->lda, vj, nullptr, W.p, nullptr, P1.p);
        k_lz_coef_proj<T><<<1, 32, 0, stream()>>>(P1.p, nq, Nf.p, j, k, m, H.p);
        PB_LAUNCH_CHECK();
        lz_proj<T, true>(n, k, nq, Q->d(), Q->lda, vj, j > 0 ? vj - nk : nullptr, W.p, P1.p, Nf.p);
      } else if (lanczos) {
        // alpha = V_j'W; W -= V_{j-1} beta + V_j alpha and ||W||^2 into Nf
        gm_blk<T, false, true>(n, k, j, J, V.p, W.p, nullptr, nullptr, O1.p);
        k_lz_coef<T><<<1, 32, 0, stream()>>>(O1.p, Nf.p, j, k, m, H.p, hL.p);
        PB_LAUNCH_CHECK();
        gm_blk<T, true, false>(n, k, std::max(0, j - 1), J, V.p, W.p, hL.p, nullptr, Nf.p);
      } else {
        if (J <= gm_chunk(k)) {
          gm_blk<T, false, true>(n, k, 0, J, V.p, W.p, nullptr, nullptr, O1.p);
          gm_blk<T, true, true>(n, k, 0, J, V.p, W.p, O1.p, nullptr, O2.p);
        } else {
          gm_dots<T>(n, k, J, V.p, W.p, O1.p);
          gm_update<T>(n, k, J, V.p, W.p, O1.p, nullptr, dummy.p);
          gm_dots<T>(n, k, J, V.p, W.p, O2.p);
        }
        k_gm_decide<T><<<1, 32, 0, stream()>>>(O1.p, O2.p, J, k, m, j, H.p, Nf.p, reorth.p);
        PB_LAUNCH_CHECK();
        gm_update<T>(n, k, J, V.p, W.p, O2.p, reorth.p, Nf.p);
      }
      const T* nrm_p = Nf.p;
      const int nrm_stride = 1;
      k_gm_step<T><<<1, 32, 0, stream()>>>(nrm_p, nrm_stride, j, k, m, H.p, cs.p, sn.p, g.p, bnorm.p, f.p, conv.p,
                                           jcount.p, eps_abs, gt, dflags);
      PB_LAUNCH_CHECK();
      k_gm_scale_cols<T><<<gw, 256, 0, stream()>>>(W.p, k, V.p + (int64_t)(j + 1) * nk, k, n, k, f.p);
      PB_LAUNCH_CHECK();
      steps = j + 1;
      // stop launching once the device reports every system converged (a
      // look at the flags, no wait: the host never blocks inside a cycle,
      // so concurrent solves on other threads keep their cores)
      if (hflags[0] >= 0 && hflags[1] >= k) stop = true;
    }
    total += steps;
    // x += [V_0..V_{J-1}] y with J the largest step count of a system
    rt().sync();
    nconv = hflags[1];
    const int J = steps;
    k_gm_solve<T><<<1, 32, 0, stream()>>>(H.p, g.p, jcount.p, k, m, J, Y.p);
    PB_LAUNCH_CHECK();
    gm_update<T>(n, k, J, V.p, X.p, Y.p, nullptr, dummy.p);
  }
  // t = x / ||x||, column by column
  gram(X.p);
  k_gm_invnorm<T><<<1, 32, 0, stream()>>>(Gk.p, k, f.p);
  PB_LAUNCH_CHECK();
  k_gm_scale_cols<T><<<gw, 256, 0, stream()>>>(X.p, k, t->d(), t->lda, n, k, f.p);
  PB_LAUNCH_CHECK();
  std::vector<int> hc(k);
  PB_CUDA(cudaMemcpyAsync(hc.data(), conv.p, sizeof(int) * k, cudaMemcpyDeviceToHost, stream()));
  rt().sync();
  int unconverged = 0;
  for (int s = 0; s < k; s++) unconverged += hc[s] ? 0 : 1;
  return unconverged;
}

template <class T>
int jada_gmres(const SparseMat<T>* A, const Mvec<T>* Q, const Mvec<T>* R, const int* resIndex, int k,
               const double* sigma, const double* tol, int maxIter, int maxBas, Mvec<T>* t)
{
  return jada_krylov<T>(A, Q, R, resIndex, k, sigma, tol, maxIter, maxBas, t, false);
}
template <class T>
int jada_minres(const SparseMat<T>* A, const Mvec<T>* Q, const Mvec<T>* R, const int* resIndex, int k,
                const double* sigma, const double* tol, int maxIter, int maxBas, Mvec<T>* t)
{
  return jada_krylov<T>(A, Q, R, resIndex, k, sigma, tol, maxIter, maxBas, t, true);
}

template int jada_gmres<double>(const SparseMat<double>*, const Mvec<double>*, const Mvec<double>*, const int*, int,
                                const double*, const double*, int, int, Mvec<double>*);
template int jada_gmres<float>(const SparseMat<float>*, const Mvec<float>*, const Mvec<float>*, const int*, int,
                               const double*, const double*, int, int, Mvec<float>*);
template int jada_minres<double>(const SparseMat<double>*, const Mvec<double>*, const Mvec<double>*, const int*, int,
                                 const double*, const double*, int, int, Mvec<double>*);
template int jada_minres<float>(const SparseMat<float>*, const Mvec<float>*, const Mvec<float>*, const int*, int,
                                const double*, const double*, int, int, Mvec<float>*);

}  // namespace pb

extern "C" {

void phist_b200_DjadaCorrection_gmres(const void* A, const void* Q, const void* res, const int* resIndex, int k,
                                      const double* sigma, const double* tol, int maxIter, int maxBas, void* t,
                                      int* iflag)
{
  PB_API_BEGIN(iflag);
  const int u = pb::jada_gmres<double>(pb::SP<double>(A), Q ? pb::MV<double>(Q) : nullptr, pb::MV<double>(res),
                                       resIndex, k, sigma, tol, maxIter, maxBas, pb::MV<double>(t));
  *iflag = u;
  PB_API_END(iflag);
}

void phist_b200_SjadaCorrection_gmres(const void* A, const void* Q, const void* res, const int* resIndex, int k,
                                      const double* sigma, const double* tol, int maxIter, int maxBas, void* t,
                                      int* iflag)
{
  PB_API_BEGIN(iflag);
  const int u = pb::jada_gmres<float>(pb::SP<float>(A), Q ? pb::MV<float>(Q) : nullptr, pb::MV<float>(res),
                                      resIndex, k, sigma, tol, maxIter, maxBas, pb::MV<float>(t));
  *iflag = u;
  PB_API_END(iflag);
}

void phist_b200_DjadaCorrection_minres(const void* A, const void* Q, const void* res, const int* resIndex, int k,
                                       const double* sigma, const double* tol, int maxIter, int maxBas, void* t,
                                       int* iflag)
{
  PB_API_BEGIN(iflag);
  const int u = pb::jada_minres<double>(pb::SP<double>(A), Q ? pb::MV<double>(Q) : nullptr, pb::MV<double>(res),
                                        resIndex, k, sigma, tol, maxIter, maxBas, pb::MV<double>(t));
  *iflag = u;
  PB_API_END(iflag);
}

void phist_b200_SjadaCorrection_minres(const void* A, const void* Q, const void* res, const int* resIndex, int k,
                                       const double* sigma, const double* tol, int maxIter, int maxBas, void* t,
                                       int* iflag)
{
  PB_API_BEGIN(iflag);
  const int u = pb::jada_minres<float>(pb::SP<float>(A), Q ? pb::MV<float>(Q) : nullptr, pb::MV<float>(res),
                                       resIndex, k, sigma, tol, maxIter, maxBas, pb::MV<float>(t));
  *iflag = u;
  PB_API_END(iflag);
}

}  // extern "C"
