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
// columns of one block: every basis block V_i is n x k, the Hessenberg
// matrices, rotations and residual estimates stay on the device, and the
// Gram-Schmidt step is classical Gram-Schmidt done twice (CGS2) as two
// block products per pass: C = [V_0..V_j]' W on the tensor-core mvTmv
// kernels, then W -= [V_0..V_j] D with D the block-diagonal part of C
// (system s only uses the coefficients of its own column).  An iteration is
// ~15 asynchronous launches with no host synchronisation; after each step
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
#include <algorithm>
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

// One CGS pass: from C = [V_0..V_j]' W (rows (j+1)k, column-major, ld ldc)
// take h(i, s) = C(i*k + s, s) into H(i, j, s) (pass 0 sets, pass 1 adds)
// and build D ((j+1)k x k, ld (j+1)k) with D(i*k + s, s) = h(i, s), zero
// elsewhere.
template <class T>
__global__ void k_gm_extract(const T* __restrict__ C, int ldc, int j, int k, int m, double* H, T* D, int pass)
{
  const int rows = (j + 1) * k;
  for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < rows * k; e += gridDim.x * blockDim.x) {
    const int r = e % rows, c = e / rows;
    const int i = r / k, s = r - i * k;
    T v = T(0);
    if (s == c) {
      v = C[r + (int64_t)c * ldc];
      double* h = H + ((int64_t)i * m + j) * k + s;
      *h = pass ? *h + (double)v : (double)v;
    }
    D[r + (int64_t)c * rows] = v;
  }
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
    for (int i = 0; i < j; i++) {
      const double a = Hat(i), b = Hat(i + 1);
      const double c = cs[i * k + s], sn_ = sn[i * k + s];
      Hat(i) = c * a + sn_ * b;
      Hat(i + 1) = -sn_ * a + c * b;
    }
    const double a = Hat(j);
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

// y_s = H(0:J_s, 0:J_s, s)^{-1} g(0:J_s, s), J_s = jcount[s], into the
// coefficient block Y (Jmax*k x k, ld Jmax*k): Y(i*k + s, s) = y_s(i).
template <class T>
__global__ void k_gm_solve(const double* __restrict__ H, const double* __restrict__ g, const int* __restrict__ jcount,
                           int k, int m, int Jmax, T* Y)
{
  const int s = threadIdx.x;
  if (s >= k) return;
  const int rows = Jmax * k;
  for (int r = 0; r < rows; r++) Y[r + (int64_t)s * rows] = T(0);
  const int J = jcount[s];
  double y[64];
  for (int i = J - 1; i >= 0; i--) {
    double v = g[i * k + s];
    for (int l = i + 1; l < J; l++) v -= H[((int64_t)i * m + l) * k + s] * y[l];
    const double d = H[((int64_t)i * m + i) * k + s];
    y[i] = (d != 0.0) ? v / d : 0.0;
  }
  for (int i = 0; i < J; i++) Y[(i * k + s) + (int64_t)s * rows] = (T)y[i];
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

// Row-parallel Gram-Schmidt kernels.  One warp per row of V (four rows of a
// warp in flight together): the J*k coefficients of the row are read as
// 32-wide coalesced chunks, lane l owning columns c = l + 32q (q < NQ).  k
// divides 32, so every column a lane owns belongs to system s = l mod k.
//   UPD:  w_s <- w_s - sum_i V(r, i*k+s) h[i*k+s]: each lane sums its
//         columns, the lanes of one system are combined by a butterfly,
//         and the new w_s is broadcast back to them
//   DOTS: out[c] = sum_r V(r, c) w_{c mod k}(r) for c < J*k (of w after the
//         update, from the same loads of V), and out[J*k+s] = ||w_s||^2;
//         without DOTS only out[s] = ||w_s||^2.
// skip (may be NULL): the kernel does nothing when *skip == 0.
// Sums: per lane over rows, warps in order, then the fixed-order last-block
// pass: bitwise reproducible.
constexpr int GM_MAXOUT = 256;  // (J+1)*k outputs at most

template <class T, bool UPD, bool DOTS, int NQ>
__global__ void __launch_bounds__(256) k_gm_rows(int64_t n, int k, int J, const T* __restrict__ V, int64_t ldV, T* W,
                                                 const T* __restrict__ h, const int* __restrict__ skip, T* part,
                                                 unsigned int* counter, T* out)
{
  if (skip && *skip == 0) return;
  constexpr int RU = 4;  // rows of one warp in flight together
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int ncol = J * k;
  const int s = lane % k;
  const int nout = DOTS ? ncol + k : k;
  T hq[NQ], acc[NQ];
#pragma unroll
  for (int q = 0; q < NQ; q++) {
    const int c = lane + 32 * q;
    hq[q] = (UPD && c < ncol) ? h[c] : T(0);
    acc[q] = T(0);
  }
  T nacc = T(0);
  const int64_t wstep = (int64_t)gridDim.x * 8;
  for (int64_t r0 = blockIdx.x * (int64_t)8 + warp; r0 < n; r0 += RU * wstep) {
    T v[RU][NQ], w[RU];
#pragma unroll
    for (int u = 0; u < RU; u++) {
      const int64_t r = r0 + u * wstep;
      const bool in = r < n;
      const T* vr = V + (in ? r : 0) * ldV;
#pragma unroll
      for (int q = 0; q < NQ; q++) {
        const int c = lane + 32 * q;
        v[u][q] = (in && c < ncol) ? vr[c] : T(0);
      }
      w[u] = in ? W[r * k + s] : T(0);
    }
#pragma unroll
    for (int u = 0; u < RU; u++) {
      const int64_t r = r0 + u * wstep;
      if (UPD) {
        T p = T(0);
#pragma unroll
        for (int q = 0; q < NQ; q++) p += v[u][q] * hq[q];
        for (int off = 16; off >= k; off >>= 1) p += __shfl_xor_sync(0xffffffffu, p, off);
        w[u] -= p;  // every lane of system s now holds the same new w_s
        if (lane < k && r < n) W[r * k + s] = w[u];
      }
      if (DOTS) {
#pragma unroll
        for (int q = 0; q < NQ; q++) acc[q] += v[u][q] * w[u];
      }
      if (lane < k) nacc += w[u] * w[u];
    }
  }
  __shared__ T red[8][GM_MAXOUT];
  if (DOTS) {
#pragma unroll
    for (int q = 0; q < NQ; q++) {
      const int c = lane + 32 * q;
      if (c < ncol) red[warp][c] = acc[q];
    }
    if (lane < k) red[warp][ncol + lane] = nacc;
  } else if (lane < k) {
    red[warp][lane] = nacc;
  }
  __syncthreads();
  for (int o = tid; o < nout; o += 256) {
    T v = T(0);
    for (int w8 = 0; w8 < 8; w8++) v += red[w8][o];
    part[(int64_t)blockIdx.x * nout + o] = v;
  }
  last_block_reduce<T>(part, nout, gridDim.x, counter, out, 1, nout, 0, T(1), T(0));
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

template <class T, bool UPD, bool DOTS>
void gm_rows(int64_t n, int k, int J, const T* V, int64_t ldV, T* W, const T* h, const int* skip, T* out)
{
  const int grid = (int)std::max<int64_t>(1, std::min<int64_t>(ceil_div(n, 32), rt().num_sms() * 8));
  const int nout = DOTS ? (J + 1) * k : k;
  const int nq = (J * k + 31) / 32;
  T* part = (T*)rt().scratch(sizeof(T) * (size_t)grid * nout);
#define PB_GMR(NQv) \
  k_gm_rows<T, UPD, DOTS, NQv><<<grid, 256, 0, stream()>>>(n, k, J, V, ldV, W, h, skip, part, rt().counters(), out)
  if (nq <= 1) PB_GMR(1);
  else if (nq <= 2) PB_GMR(2);
  else if (nq <= 4) PB_GMR(4);
  else PB_GMR(8);
#undef PB_GMR
  PB_LAUNCH_CHECK();
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

template <class T>
int jada_gmres(const SparseMat<T>* A, const Mvec<T>* Q, const Mvec<T>* R, const int* resIndex, int k,
               const double* sigma, const double* tol, int maxIter, int maxBas, Mvec<T>* t)
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
  const int64_t ldV = (int64_t)(m + 1) * k;
  const double eps_abs = 1000.0 * std::numeric_limits<T>::epsilon();

  DBuf<T> V((size_t)n * ldV), B((size_t)n * k), X((size_t)n * k), W((size_t)n * k);
  DBuf<T> C((size_t)(m + 1) * k * k), D((size_t)(m + 1) * k * k), Cq((size_t)std::max(nq, 1) * k);
  DBuf<T> Gk((size_t)k * k), f(k);
  DBuf<double> H((size_t)(m + 1) * m * k), cs((size_t)m * k), sn((size_t)m * k), g((size_t)(m + 1) * k), bnorm(k);
  DBuf<int> conv(k), jcount(k), reorth(1);
  DBuf<T> O1(GM_MAXOUT), O2(GM_MAXOUT), Nf(k);
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
    k_gm_scale_cols<T><<<gw, 256, 0, stream()>>>(W.p, k, V.p, ldV, n, k, f.p);
    PB_LAUNCH_CHECK();
    hflags[1] = 0;
    hflags[0] = -1;
    int j = 0, steps = 0;
    const int jmax = std::min(m, maxIter - total);
    bool stop = false;
    for (j = 0; j < jmax && !stop; j++) {
      // W = P (A - sigma I) V_j
      raw_view(mVj, V.p + (int64_t)j * k, n, k, ldV);
      spmv_general<T>(T(1), A, negsig.data(), &mVj, T(0), &mW, nullptr, nullptr, T(0), T(0), nullptr);
      project();
      // Gram-Schmidt against V_0..V_j
      const int rows = (j + 1) * k;
      const T* nrm_p = Gk.p;
      int nrm_stride = k + 1;
      if ((j + 2) * k <= GM_MAXOUT && (32 % k) == 0) {
        // row-parallel kernels: h1 = V'W and ||W||^2; W -= V h1 with
        // h2 = V'W and ||W||^2 of the result in the same pass; a second
        // pass only where a norm fell below 1/sqrt(2) of its value before
        // (the decision is a device flag the second-pass kernel reads)
        const int J = j + 1;
        gm_rows<T, false, true>(n, k, J, V.p, ldV, W.p, nullptr, nullptr, O1.p);
        gm_rows<T, true, true>(n, k, J, V.p, ldV, W.p, O1.p, nullptr, O2.p);
        k_gm_decide<T><<<1, 32, 0, stream()>>>(O1.p, O2.p, J, k, m, j, H.p, Nf.p, reorth.p);
        PB_LAUNCH_CHECK();
        gm_rows<T, true, false>(n, k, J, V.p, ldV, W.p, O2.p, reorth.p, Nf.p);
        nrm_p = Nf.p;
        nrm_stride = 1;
      } else {
        // CGS2 as block products
        for (int pass = 0; pass < 2; pass++) {
          launch_mvTmv<T>(n, rows, k, T(1), V.p, ldV, W.p, k, T(0), C.p, rows);
          k_gm_extract<T><<<std::max(1, (rows * k + 255) / 256), 256, 0, stream()>>>(C.p, rows, j, k, m, H.p, D.p,
                                                                                     pass);
          PB_LAUNCH_CHECK();
          gm_mvsd<T>(n, rows, k, T(-1), V.p, ldV, D.p, rows, T(1), W.p, k);
        }
        gram(W.p);
      }
      k_gm_step<T><<<1, 32, 0, stream()>>>(nrm_p, nrm_stride, j, k, m, H.p, cs.p, sn.p, g.p, bnorm.p, f.p, conv.p,
                                           jcount.p, eps_abs, gt, dflags);
      PB_LAUNCH_CHECK();
      k_gm_scale_cols<T><<<gw, 256, 0, stream()>>>(W.p, k, V.p + (int64_t)(j + 1) * k, ldV, n, k, f.p);
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
    k_gm_solve<T><<<1, 32, 0, stream()>>>(H.p, g.p, jcount.p, k, m, J, D.p);
    PB_LAUNCH_CHECK();
    gm_mvsd<T>(n, J * k, k, T(1), V.p, ldV, D.p, J * k, T(1), X.p, k);
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

template int jada_gmres<double>(const SparseMat<double>*, const Mvec<double>*, const Mvec<double>*, const int*, int,
                                const double*, const double*, int, int, Mvec<double>*);
template int jada_gmres<float>(const SparseMat<float>*, const Mvec<float>*, const Mvec<float>*, const int*, int,
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

}  // extern "C"
