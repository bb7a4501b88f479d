// pb_carpcg.cu -- batched multi-shift CARP-CG (CGMN) on the GPU.
//
// Solves (A - sigma_j I) x_j = b_j for a queue of systems j < nsys on a block
// of `w` slots.  Every slot runs the CGMN iteration of PHIST's carp_cg
// (src/krylov/phist_carp_cg_def.hpp:440-690: r = dkswp(x, b) - x, p = r,
// q = p - dkswp(p, 0), alpha = r'r / p'q, x += alpha p, r -= alpha q,
// beta = r'r_new / r'r, p = r + beta p), all slots at once: one double
// Kaczmarz sweep per iteration over the w columns, with every scalar of the
// recurrence (r'r, p'q, alpha, beta) kept on the device, so an iteration
// issues no host synchronisation.  Every `check_every` iterations the
// explicit residuals are measured; a converged system leaves its slot, its
// solution is written to X, and the next queued system takes the slot
// (x = 0, new shift, new right-hand side, CG restarted for that column
// only).  A slot is never iterated after convergence, so PHIST's
// alpha = (1-conv) r'r / p'q on a converged column (which turns into NaN
// once p'q underflows to zero) does not arise.
//
// mixed = 1: the CGMN iteration and its sweeps run in FP32 on an FP32 copy
// of A (FP32 accumulation), inside FP64 iterative refinement per slot:
//   x64 += s_j d_j;  r64 = b - (A - sigma_j I) x64 (FP64);
//   converged if ||r64|| <= tol ||b||, else restart the FP32 CGMN on
//   c_j = r64 / s_j with s_j = ||r64|| (unit-norm right-hand side).
// The inner solve of a slot ends when its FP32 explicit residual
// ||c - (A - sigma I) d|| drops below innerTol or stops decreasing.
#include "pb_api.cuh"

namespace pb {

// ------------------------------------------------------------------ kernels
// per-column scalar updates (w <= 32 columns; one thread per column)
template <class T>
__global__ void k_cg_alpha(const T* rr, const T* pq, const int* active, T* alpha, int w)
{
  const int j = threadIdx.x;
  if (j >= w) return;
  const T d = pq[j];
  alpha[j] = (active[j] && d > T(0)) ? rr[j] / d : T(0);
}

template <class T>
__global__ void k_cg_beta(const T* rr_new, T* rr, const int* active, T* beta, int w)
{
  const int j = threadIdx.x;
  if (j >= w) return;
  const T o = rr[j];
  beta[j] = (active[j] && o > T(0)) ? rr_new[j] / o : T(0);
  rr[j] = rr_new[j];
}

// d += alpha p, r -= alpha q (alpha per column, on the device)
template <class T>
__global__ void k_cg_xr(T* d, T* r, const T* __restrict__ p, const T* __restrict__ q, const T* __restrict__ alpha,
                        int64_t n, int w)
{
  PB_FOR_ELEMS(n, w, i, j)
  {
    const T a = alpha[j];
    if (a != T(0)) {
      d[i * w + j] += a * p[i * w + j];
      r[i * w + j] -= a * q[i * w + j];
    }
  }
}

// p = r + beta p
template <class T>
__global__ void k_cg_p(T* p, const T* __restrict__ r, const T* __restrict__ beta, int64_t n, int w)
{
  PB_FOR_ELEMS(n, w, i, j) p[i * w + j] = r[i * w + j] + beta[j] * p[i * w + j];
}

// q = p - q
template <class T>
__global__ void k_cg_pmq(T* q, const T* __restrict__ p, int64_t n, int w)
{
  PB_FOR_ELEMS(n, w, i, j) q[i * w + j] = p[i * w + j] - q[i * w + j];
}

// columns with mask[j] != 0: dst = src (src may have another leading dim)
template <class TD, class TS>
__global__ void k_cols_masked_copy(TD* dst, int64_t ldd, const TS* __restrict__ src, int64_t lds,
                                   const float* __restrict__ scale, const int* __restrict__ mask, int64_t n, int w)
{
  PB_FOR_ELEMS(n, w, i, j)
  if (mask[j]) dst[i * ldd + j] = TD(scale ? (double)src[i * lds + j] * (double)scale[j] : (double)src[i * lds + j]);
}

// columns with mask[j] != 0: dst = value
template <class T>
__global__ void k_cols_masked_set(T* dst, T value, const int* __restrict__ mask, int64_t n, int w)
{
  PB_FOR_ELEMS(n, w, i, j) if (mask[j]) dst[i * w + j] = value;
}

// x64 += scale_j * d (columns with mask[j] != 0)
template <class TI>
__global__ void k_refine_add(double* x, const TI* __restrict__ d, const double* __restrict__ scale,
                             const int* __restrict__ mask, int64_t n, int w)
{
  PB_FOR_ELEMS(n, w, i, j) if (mask[j]) x[i * w + j] += scale[j] * (double)d[i * w + j];
}

// Fused CG updates on contiguous n x w blocks viewed as flat arrays of
// N = n*w entries, w a power of two dividing 256: thread t of every block
// always touches column t mod w (the grid stride is a multiple of w), and
// the column sums of the fused dot are formed in a fixed tree, then across
// blocks in block order (last_block_reduce): bitwise reproducible.
template <class T>
__device__ __forceinline__ void col_block_sum(T acc, int w, T* part, unsigned int* counter, T* out)
{
  __shared__ T red[256];
  const T s = block_sum_mod<T>(acc, w, red);
  if ((int)threadIdx.x < w) part[(int64_t)blockIdx.x * w + threadIdx.x] = s;
  last_block_reduce<T>(part, w, gridDim.x, counter, out, 1, w, 0, T(1), T(0));
}

// q = p - q and pq_j = p_j' q_j
template <class T>
__global__ void __launch_bounds__(256) k_cg_pmq_dot(T* q, const T* __restrict__ p, int64_t N, int w, T* part,
                                                    unsigned int* counter, T* out)
{
  T acc = T(0);
  const int64_t st = (int64_t)gridDim.x * 256;
  int64_t e = blockIdx.x * 256 + threadIdx.x;
  for (; e + 3 * st < N; e += 4 * st) {  // four entries in flight per thread
    T pv[4], qv[4];
#pragma unroll
    for (int u = 0; u < 4; u++) {
      pv[u] = p[e + u * st];
      qv[u] = q[e + u * st];
    }
#pragma unroll
    for (int u = 0; u < 4; u++) {
      qv[u] = pv[u] - qv[u];
      q[e + u * st] = qv[u];
      acc += pv[u] * qv[u];
    }
  }
  for (; e < N; e += st) {
    const T pv = p[e];
    const T qv = pv - q[e];
    q[e] = qv;
    acc += pv * qv;
  }
  col_block_sum<T>(acc, w, part, counter, out);
}

// d += alpha p, r -= alpha q, rr_j = r_j' r_j
template <class T>
__global__ void __launch_bounds__(256) k_cg_xr_dot(T* d, T* r, const T* __restrict__ p, const T* __restrict__ q,
                                                   const T* __restrict__ alpha, int64_t N, int w, T* part,
                                                   unsigned int* counter, T* out)
{
  const T a = alpha[threadIdx.x % w];
  T acc = T(0);
  const int64_t st = (int64_t)gridDim.x * 256;
  int64_t e = blockIdx.x * 256 + threadIdx.x;
  if (a != T(0)) {
    for (; e + 3 * st < N; e += 4 * st) {  // four entries in flight per thread
      T dv[4], rv[4], pv[4], qv[4];
#pragma unroll
      for (int u = 0; u < 4; u++) {
        dv[u] = d[e + u * st];
        rv[u] = r[e + u * st];
        pv[u] = p[e + u * st];
        qv[u] = q[e + u * st];
      }
#pragma unroll
      for (int u = 0; u < 4; u++) {
        d[e + u * st] = dv[u] + a * pv[u];
        rv[u] -= a * qv[u];
        r[e + u * st] = rv[u];
        acc += rv[u] * rv[u];
      }
    }
  }
  for (; e < N; e += st) {
    T rv = r[e];
    if (a != T(0)) {
      d[e] += a * p[e];
      rv -= a * q[e];
      r[e] = rv;
    }
    acc += rv * rv;
  }
  col_block_sum<T>(acc, w, part, counter, out);
}

// p = r + beta p
template <class T>
__global__ void __launch_bounds__(256) k_cg_p_flat(T* p, const T* __restrict__ r, const T* __restrict__ beta,
                                                   int64_t N, int w)
{
  const T b = beta[threadIdx.x % w];
  const int64_t st = (int64_t)gridDim.x * 256;
  int64_t e = blockIdx.x * 256 + threadIdx.x;
  for (; e + 3 * st < N; e += 4 * st) {
    T rv[4], pv[4];
#pragma unroll
    for (int u = 0; u < 4; u++) {
      rv[u] = r[e + u * st];
      pv[u] = p[e + u * st];
    }
#pragma unroll
    for (int u = 0; u < 4; u++) p[e + u * st] = rv[u] + b * pv[u];
  }
  for (; e < N; e += st) p[e] = r[e] + b * p[e];
}

// one column of a w-wide block into column s of an nsys-wide block and back
template <class T>
__global__ void k_col_copy(T* dst, int64_t ldd, const T* __restrict__ src, int64_t lds, int64_t n)
{
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    dst[i * ldd] = src[i * lds];
}

}  // namespace pb

// --------------------------------------------------------------------- host
namespace pb {
namespace {

template <class T>
struct DevBuf {
  T* p = nullptr;
  explicit DevBuf(size_t count) { p = (T*)rt().dmalloc(sizeof(T) * (count ? count : 1)); }
  ~DevBuf() { rt().dfree(p); }
  DevBuf(const DevBuf&) = delete;
  DevBuf& operator=(const DevBuf&) = delete;
};

// an n x w row-major block on raw device memory, as the internal kernels
// launchers expect it
template <class T>
void as_mvec(Mvec<T>& m, T* d, int64_t n, int w)
{
  m.map = nullptr;
  m.nrows = (int32_t)n;
  m.nvec = w;
  m.lda = w;
  m.root = &m;
  m.col_off = 0;
  m.d_base = d;
  m.h_base = nullptr;
}

// blocks of the column-dot kernel for n rows (the partial sums need
// dots_grid(n) * 32 entries)
inline int dots_grid(int64_t n) { return std::max(1, std::min(grid_for(n), rt().num_sms() * 4)); }

// column dots a'b of two n x w blocks into a device array out[w]; part and
// counter default to the lane's scratch and arrival counter
template <class T>
void dots_dev(const T* a, const T* b, int64_t n, int w, T* out, T* part = nullptr, unsigned int* counter = nullptr)
{
  const int grid = dots_grid(n);
  if (!part) part = (T*)rt().scratch(sizeof(T) * (size_t)grid * 32);
  if (!counter) counter = rt().counters();
#define PB_DD(NVv)                                                                                     \
  {                                                                                                    \
    const int ext = (NVv >= 16 && grid > 1) ? 1 : 0;                                                   \
    k_coldot<T, NVv><<<grid, 256, 0, stream()>>>(a, w, b, w, n, w, part, counter, out, ext);           \
    if (ext) k_reduce_partials<T><<<1, 256, 0, stream()>>>(part, grid, NVv, out, NVv, 0, T(1), T(0));  \
  }
  if (w <= 1) PB_DD(1)
  else if (w <= 2) PB_DD(2)
  else if (w <= 4) PB_DD(4)
  else if (w <= 8) PB_DD(8)
  else if (w <= 16) PB_DD(16)
  else PB_DD(32)
#undef PB_DD
  PB_LAUNCH_CHECK();
}

template <class T>
void dots_host(const T* a, const T* b, int64_t n, int w, double* out)
{
  T* dd = (T*)rt().mailbox_dev();
  dots_dev<T>(a, b, n, w, dd);
  rt().sync();
  const T* h = (const T*)rt().mailbox_host();
  for (int j = 0; j < w; j++) out[j] = (double)h[j];
}

template <class T>
void upload(T* d, const T* h, int w)
{
  PB_CUDA(cudaMemcpyAsync(d, h, sizeof(T) * w, cudaMemcpyHostToDevice, stream()));
}

}  // namespace

// The solver.  TI: type of the CGMN iteration (double: plain FP64 CARP-CG;
// float: FP32 inner solves inside FP64 refinement).  Returns the number of
// systems that did not converge within maxIter iterations of their slot.
template <class TI>
int carpcg_batch(const SparseMat<double>* A64, const SparseMat<TI>* Ain, CarpWork<TI>* work, int nsys,
                 const double* sigma, const Mvec<double>* B, Mvec<double>* X, int w, double tol, int maxIter, int K,
                 double innerTol, int* iters, double* relres)
{
  constexpr bool MIXED = std::is_same<TI, float>::value;
  const int64_t n = A64->nrows;
  const size_t nw = (size_t)n * w;
  DevBuf<double> x64(nw), b64(nw), r64(nw);
  DevBuf<TI> d(nw), r(nw), p(nw), q(nw), c(nw), t(nw);
  DevBuf<TI> rr(w), pq(w), alpha(w), beta(w), rrn(w);
  DevBuf<int> active(w), mask(w);
  DevBuf<double> scale64(w);
  DevBuf<float> scale32(w);
  Mvec<double> mx64, mb64, mr64;
  as_mvec(mx64, x64.p, n, w);
  as_mvec(mb64, b64.p, n, w);
  as_mvec(mr64, r64.p, n, w);
  Mvec<TI> md, mc, mt, mq;
  as_mvec(md, d.p, n, w);
  as_mvec(mc, c.p, n, w);
  as_mvec(mt, t.p, n, w);
  as_mvec(mq, q.p, n, w);

  std::vector<int> sys(w, -1), hmask(w, 0), hact(w, 0), inner_it(w, 0), best_it(w, 0);
  std::vector<double> sig(w, 0.0), negsig(w, 0.0), bnorm(w, 1.0), s(w, 1.0), last_rho(w, 1e300), nrm(w);
  std::vector<TI> sigI(w, TI(0)), omegaI(w, TI(1)), negsigI(w, TI(0));
  std::vector<float> hscale32(w, 1.0f);
  for (int j = 0; j < nsys; j++) {
    iters[j] = 0;
    relres[j] = -1.0;
  }
  int next = 0, unconverged = 0;
  const int gridw = grid_for((int64_t)nw);
  // fused flat CG kernels when w divides 256
  const bool flat = (256 % w) == 0;
  const int gridf = (int)std::max<int64_t>(1, std::min<int64_t>(ceil_div((int64_t)nw, 256 * 8), rt().num_sms() * 8));

  // partial sums and arrival counter of the iteration's dots: buffers of
  // their own, so that the pointers recorded in the CUDA graph stay valid
  // whatever the lane's scratch does in between
  DevBuf<TI> ipart((size_t)std::max<int64_t>((int64_t)gridf * w, (int64_t)dots_grid(n) * 32));
  DevBuf<unsigned int> icnt(1);
  PB_CUDA(cudaMemsetAsync(icnt.p, 0, sizeof(unsigned int), stream()));

  auto sweep = [&](const Mvec<TI>* rhs, Mvec<TI>* v) {
    carp_run<TI, false>(work, w, sigI.data(), nullptr, rhs, v, nullptr, omegaI.data());
  };
  bool graph_stale = true;  // the shifts recorded in the graph changed
  auto set_shift = [&](int j, double sg) {
    graph_stale = true;
    sig[j] = sg;
    negsig[j] = -sg;
    sigI[j] = (TI)sg;
    negsigI[j] = (TI)(-sg);
  };
  // restart the CGMN of the slots in hmask from d = 0 on their current c
  auto restart_inner = [&]() {
    upload(mask.p, hmask.data(), w);
    k_cols_masked_set<TI><<<gridw, 256, 0, stream()>>>(d.p, TI(0), mask.p, n, w);
    PB_LAUNCH_CHECK();
    k_put_value<TI><<<gridw, 256, 0, stream()>>>(t.p, w, n, w, TI(0));
    PB_LAUNCH_CHECK();
    sweep(&mc, &mt);  // t = dkswp(0, c)
    k_cols_masked_copy<TI, TI><<<gridw, 256, 0, stream()>>>(r.p, w, t.p, w, nullptr, mask.p, n, w);
    PB_LAUNCH_CHECK();
    k_cols_masked_copy<TI, TI><<<gridw, 256, 0, stream()>>>(p.p, w, t.p, w, nullptr, mask.p, n, w);
    PB_LAUNCH_CHECK();
    dots_dev<TI>(r.p, r.p, n, w, rr.p);
    for (int j = 0; j < w; j++)
      if (hmask[j]) {
        inner_it[j] = 0;
        best_it[j] = 0;
        last_rho[j] = 1e300;
      }
  };
  // c = r64 * scale32 for the slots in hmask (unit-norm right-hand sides)
  auto narrow_rhs = [&]() {
    upload(mask.p, hmask.data(), w);
    upload(scale32.p, hscale32.data(), w);
    k_cols_masked_copy<TI, double><<<gridw, 256, 0, stream()>>>(c.p, w, r64.p, w, scale32.p, mask.p, n, w);
    PB_LAUNCH_CHECK();
  };
  // put the next queued systems into the slots in `slots`
  auto refill = [&](const std::vector<int>& slots) {
    std::fill(hmask.begin(), hmask.end(), 0);
    for (int j : slots) {
      hmask[j] = 1;
      sys[j] = next < nsys ? next++ : -1;
      if (sys[j] >= 0) set_shift(j, sigma[sys[j]]);
    }
    upload(mask.p, hmask.data(), w);
    k_cols_masked_set<double><<<gridw, 256, 0, stream()>>>(x64.p, 0.0, mask.p, n, w);
    PB_LAUNCH_CHECK();
    k_cols_masked_set<double><<<gridw, 256, 0, stream()>>>(b64.p, 0.0, mask.p, n, w);  // empty slots
    PB_LAUNCH_CHECK();
    for (int j : slots)
      if (sys[j] >= 0) {
        k_col_copy<double><<<grid_for(n), 256, 0, stream()>>>(b64.p + j, w, B->d() + sys[j], B->lda, n);
        PB_LAUNCH_CHECK();
      }
    dots_host<double>(b64.p, b64.p, n, w, nrm.data());
    for (int j : slots) {
      bnorm[j] = std::sqrt(nrm[j]);
      // mixed: unit-norm inner right-hand sides; FP64: the CGMN iterate is x
      s[j] = (MIXED && bnorm[j] > 0.0) ? bnorm[j] : 1.0;
      hscale32[j] = (float)(1.0 / s[j]);
      hact[j] = sys[j] >= 0;
    }
    // first inner right-hand side: c = b / ||b|| (r64 = b)
    PB_CUDA(cudaMemcpyAsync(r64.p, b64.p, sizeof(double) * nw, cudaMemcpyDeviceToDevice, stream()));
    narrow_rhs();
    upload(active.p, hact.data(), w);
    restart_inner();
  };
  // r64 = b - (A - sigma I) x64 for all slots; relative norms into nrm
  auto outer_residual = [&]() {
    PB_CUDA(cudaMemcpyAsync(r64.p, b64.p, sizeof(double) * nw, cudaMemcpyDeviceToDevice, stream()));
    spmv_general<double>(-1.0, A64, negsig.data(), &mx64, 1.0, &mr64, nullptr, nullptr, 0.0, 0.0, nullptr);
    dots_host<double>(r64.p, r64.p, n, w, nrm.data());
    for (int j = 0; j < w; j++) nrm[j] = std::sqrt(nrm[j]) / (bnorm[j] > 0.0 ? bnorm[j] : 1.0);
  };
  auto finish = [&](int j, double rel) {
    k_col_copy<double><<<grid_for(n), 256, 0, stream()>>>(X->d() + sys[j], X->lda, x64.p + j, w, n);
    PB_LAUNCH_CHECK();
    relres[sys[j]] = rel;
  };

  {
    std::vector<int> all(w);
    std::iota(all.begin(), all.end(), 0);
    refill(all);
  }
  // one CGMN iteration on every slot: only kernel launches and a device
  // copy, all scalars device-resident, so it can be recorded as a graph
  auto iteration = [&]() {
    PB_CUDA(cudaMemcpyAsync(q.p, p.p, sizeof(TI) * nw, cudaMemcpyDeviceToDevice, stream()));
    sweep(nullptr, &mq);  // q = dkswp(p, 0)
    if (flat) {
      k_cg_pmq_dot<TI><<<gridf, 256, 0, stream()>>>(q.p, p.p, (int64_t)nw, w, ipart.p, icnt.p, pq.p);
      PB_LAUNCH_CHECK();
      k_cg_alpha<TI><<<1, 32, 0, stream()>>>(rr.p, pq.p, active.p, alpha.p, w);
      PB_LAUNCH_CHECK();
      k_cg_xr_dot<TI><<<gridf, 256, 0, stream()>>>(d.p, r.p, p.p, q.p, alpha.p, (int64_t)nw, w, ipart.p, icnt.p,
                                                   rrn.p);
      PB_LAUNCH_CHECK();
      k_cg_beta<TI><<<1, 32, 0, stream()>>>(rrn.p, rr.p, active.p, beta.p, w);
      PB_LAUNCH_CHECK();
      k_cg_p_flat<TI><<<gridf, 256, 0, stream()>>>(p.p, r.p, beta.p, (int64_t)nw, w);
      PB_LAUNCH_CHECK();
    } else {
      k_cg_pmq<TI><<<gridw, 256, 0, stream()>>>(q.p, p.p, n, w);
      PB_LAUNCH_CHECK();
      dots_dev<TI>(p.p, q.p, n, w, pq.p, ipart.p, icnt.p);
      k_cg_alpha<TI><<<1, 32, 0, stream()>>>(rr.p, pq.p, active.p, alpha.p, w);
      PB_LAUNCH_CHECK();
      k_cg_xr<TI><<<gridw, 256, 0, stream()>>>(d.p, r.p, p.p, q.p, alpha.p, n, w);
      PB_LAUNCH_CHECK();
      dots_dev<TI>(r.p, r.p, n, w, rrn.p, ipart.p, icnt.p);
      k_cg_beta<TI><<<1, 32, 0, stream()>>>(rrn.p, rr.p, active.p, beta.p, w);
      PB_LAUNCH_CHECK();
      k_cg_p<TI><<<gridw, 256, 0, stream()>>>(p.p, r.p, beta.p, n, w);
      PB_LAUNCH_CHECK();
    }
  };
  // The iteration as a CUDA graph, replayed K times between two checks: one
  // graph launch instead of ~2 ncolors + 5 kernel launches per iteration.
  // The shifts are kernel arguments, so a refill that changes them records
  // the graph again.
  struct GraphGuard {
    cudaGraphExec_t g = nullptr;
    ~GraphGuard()
    {
      if (g) cudaGraphExecDestroy(g);
    }
  } graph;
  uint64_t graph_launches = 0;
  auto record = [&]() {
    if (graph.g) {
      PB_CUDA(cudaGraphExecDestroy(graph.g));
      graph.g = nullptr;
    }
    const uint64_t l0 = rt().launches.load();
    PB_CUDA(cudaStreamBeginCapture(stream(), cudaStreamCaptureModeThreadLocal));
    cudaGraph_t g = nullptr;
    try {
      iteration();
    } catch (...) {
      cudaStreamEndCapture(stream(), &g);
      if (g) cudaGraphDestroy(g);
      throw;
    }
    PB_CUDA(cudaStreamEndCapture(stream(), &g));
    graph_launches = rt().launches.load() - l0;
    rt().launches -= graph_launches;  // counted when the graph runs
    const cudaError_t e = cudaGraphInstantiate(&graph.g, g, 0);
    cudaGraphDestroy(g);
    PB_CUDA(e);
    graph_stale = false;
  };

  for (;;) {
    bool any = false;
    for (int j = 0; j < w; j++) any = any || sys[j] >= 0;
    if (!any) break;
    // K CGMN iterations on every slot
    if (rt().use_graphs) {
      if (graph_stale || !graph.g) record();
      for (int k = 0; k < K; k++) {
        PB_CUDA(cudaGraphLaunch(graph.g, stream()));
        rt().launches += graph_launches;
      }
    } else {
      for (int k = 0; k < K; k++) iteration();
    }
    for (int j = 0; j < w; j++)
      if (sys[j] >= 0) {
        iters[sys[j]] += K;
        inner_it[j] += K;
      }

    // ---- check
    std::vector<int> done;  // slots whose system converged or ran out of iterations
    if (!MIXED) {
      // the CGMN iterate is the solution itself
      PB_CUDA(cudaMemcpyAsync(x64.p, d.p, sizeof(double) * nw, cudaMemcpyDeviceToDevice, stream()));
      outer_residual();
      for (int j = 0; j < w; j++)
        if (sys[j] >= 0 && (nrm[j] <= tol || iters[sys[j]] >= maxIter)) {
          finish(j, nrm[j]);
          if (!(nrm[j] <= tol)) unconverged++;
          done.push_back(j);
        }
    } else {
      // inner residuals rho = ||c - (A - sigma I) d||, c of unit norm
      PB_CUDA(cudaMemcpyAsync(t.p, c.p, sizeof(TI) * nw, cudaMemcpyDeviceToDevice, stream()));
      spmv_general<TI>(TI(-1), Ain, negsigI.data(), &md, TI(1), &mt, nullptr, nullptr, TI(0), TI(0), nullptr);
      std::vector<double> rho(w);
      dots_host<TI>(t.p, t.p, n, w, rho.data());
      std::fill(hmask.begin(), hmask.end(), 0);
      bool refine = false;
      for (int j = 0; j < w; j++) {
        if (sys[j] < 0) continue;
        rho[j] = std::sqrt(rho[j]);
        // progress: a 1 % drop of the best inner residual so far
        if (rho[j] < 0.99 * last_rho[j]) {
          last_rho[j] = rho[j];
          best_it[j] = inner_it[j];
        }
        // inner solve done: tolerance reached, or no progress in the last
        // 100 checks (the FP32 rounding floor of this system)
        if (rho[j] <= innerTol || inner_it[j] - best_it[j] >= 100 * K || iters[sys[j]] >= maxIter) {
          hmask[j] = 1;
          refine = true;
        }
      }
      if (refine) {
        upload(mask.p, hmask.data(), w);
        upload(scale64.p, s.data(), w);
        k_refine_add<TI><<<gridw, 256, 0, stream()>>>(x64.p, d.p, scale64.p, mask.p, n, w);
        PB_LAUNCH_CHECK();
        outer_residual();
        std::vector<int> restart(w, 0);
        for (int j = 0; j < w; j++) {
          if (!hmask[j]) continue;
          if (nrm[j] <= tol || iters[sys[j]] >= maxIter) {
            finish(j, nrm[j]);
            if (!(nrm[j] <= tol)) unconverged++;
            done.push_back(j);
          } else {
            restart[j] = 1;
            s[j] = nrm[j] * bnorm[j];
            hscale32[j] = (float)(1.0 / s[j]);
          }
        }
        if (std::count(restart.begin(), restart.end(), 1) > 0) {
          hmask = restart;
          narrow_rhs();
          restart_inner();
        }
      }
    }
    if (!done.empty()) refill(done);
  }
  rt().sync();
  return unconverged;
}

// Device time of one CGMN iteration of the batched solver for w slots (the
// colour sweep q = dkswp(p, 0) and the fused CG updates with their column
// dots, as in carpcg_batch) on scratch blocks: median of reps replays after
// a warm-up, in microseconds.  The values in the blocks do not matter for
// the time; they are set to a fixed pattern.
template <class TI>
double carpcg_iteration_us(const SparseMat<TI>* Ain, CarpWork<TI>* work, int w, int reps)
{
  const int64_t n = Ain->nrows;
  const size_t nw = (size_t)n * w;
  DevBuf<TI> d(nw), r(nw), p(nw), q(nw);
  DevBuf<TI> rr(w), pq(w), alpha(w), beta(w), rrn(w);
  DevBuf<int> active(w);
  DevBuf<unsigned int> icnt(1);
  const int gridf = (int)std::max<int64_t>(1, std::min<int64_t>(ceil_div((int64_t)nw, 256 * 8), rt().num_sms() * 8));
  DevBuf<TI> ipart((size_t)gridf * w);
  PB_CUDA(cudaMemsetAsync(icnt.p, 0, sizeof(unsigned int), stream()));
  TI* const fill[3] = {d.p, r.p, p.p};
  for (int k = 0; k < 3; k++)
    k_random<TI><<<grid_for((int64_t)nw), 256, 0, stream()>>>(fill[k], w, n, w, w, 0, 77 + k);
  PB_LAUNCH_CHECK();
  k_put_value<TI><<<1, 32, 0, stream()>>>(rr.p, w, 1, w, TI(1));
  k_put_value<int><<<1, 32, 0, stream()>>>(active.p, w, 1, w, 1);
  PB_LAUNCH_CHECK();
  std::vector<TI> sig(w, TI(0.5)), om(w, TI(1));
  Mvec<TI> mq;
  as_mvec(mq, q.p, n, w);
  auto iteration = [&]() {
    PB_CUDA(cudaMemcpyAsync(q.p, p.p, sizeof(TI) * nw, cudaMemcpyDeviceToDevice, stream()));
    carp_run<TI, false>(work, w, sig.data(), nullptr, nullptr, &mq, nullptr, om.data());
    k_cg_pmq_dot<TI><<<gridf, 256, 0, stream()>>>(q.p, p.p, (int64_t)nw, w, ipart.p, icnt.p, pq.p);
    k_cg_alpha<TI><<<1, 32, 0, stream()>>>(rr.p, pq.p, active.p, alpha.p, w);
    k_cg_xr_dot<TI><<<gridf, 256, 0, stream()>>>(d.p, r.p, p.p, q.p, alpha.p, (int64_t)nw, w, ipart.p, icnt.p,
                                                 rrn.p);
    k_cg_beta<TI><<<1, 32, 0, stream()>>>(rrn.p, rr.p, active.p, beta.p, w);
    k_cg_p_flat<TI><<<gridf, 256, 0, stream()>>>(p.p, r.p, beta.p, (int64_t)nw, w);
    PB_LAUNCH_CHECK();
  };
  cudaEvent_t e0, e1;
  PB_CUDA(cudaEventCreate(&e0));
  PB_CUDA(cudaEventCreate(&e1));
  std::vector<float> ts;
  try {
    iteration();  // warm-up
    for (int k = 0; k < std::max(1, reps); k++) {
      PB_CUDA(cudaEventRecord(e0, stream()));
      iteration();
      PB_CUDA(cudaEventRecord(e1, stream()));
      PB_CUDA(cudaEventSynchronize(e1));
      float ms = 0.0f;
      PB_CUDA(cudaEventElapsedTime(&ms, e0, e1));
      ts.push_back(ms);
    }
  } catch (...) {
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    throw;
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  std::sort(ts.begin(), ts.end());
  return 1e3 * (double)ts[ts.size() / 2];
}

// Slot count of the batched solver with the most system-iterations per
// second, w / t_iteration(w), over w in {1, 2, 4, 8, 16, 32} up to nsys.
// us[6] (may be NULL) receives each candidate's iteration time (0: not
// tried).
template <class TI>
int carpcg_tune_block(const SparseMat<TI>* Ain, CarpWork<TI>* work, int nsys, int reps, double* us)
{
  int best = 1;
  double best_rate = -1.0;
  for (int k = 0; k < 6; k++) {
    const int w = 1 << k;
    if (us) us[k] = 0.0;
    if (w > std::max(1, nsys)) continue;
    const double t = carpcg_iteration_us<TI>(Ain, work, w, reps);
    if (us) us[k] = t;
    const double rate = w / t;
    if (rate > best_rate) {
      best_rate = rate;
      best = w;
    }
  }
  return best;
}

template int carpcg_batch<double>(const SparseMat<double>*, const SparseMat<double>*, CarpWork<double>*, int,
                                  const double*, const Mvec<double>*, Mvec<double>*, int, double, int, int, double,
                                  int*, double*);
template int carpcg_batch<float>(const SparseMat<double>*, const SparseMat<float>*, CarpWork<float>*, int,
                                 const double*, const Mvec<double>*, Mvec<double>*, int, double, int, int, double,
                                 int*, double*);

}  // namespace pb

extern "C" {
void phist_b200_sparseMat_DtoS(const void* vA, void** vAs, int* iflag);
void phist_SsparseMat_delete(void* A, int* iflag);
}

namespace {
// the FP32 copy of A for the mixed solver, deleted with the guard
struct SCopy {
  void* a = nullptr;
  ~SCopy()
  {
    int e = 0;
    if (a) phist_SsparseMat_delete(a, &e);
  }
};

template <class TI>
struct WorkGuard {
  pb::CarpWork<TI>* w = nullptr;
  ~WorkGuard() { pb::carp_free<TI>(w); }
};
}  // namespace

extern "C" {

void phist_b200_DcarpCG_tune_block(const void* vA, int nsys, int mixed, int reps, int* block, double* iter_us,
                                   int* iflag)
{
  PB_API_BEGIN(iflag);
  using namespace pb;
  const SparseMat<double>* A = SP<double>(vA);
  PB_REQUIRE(block, PB_INVALID_INPUT, "block is NULL");
  PB_REQUIRE(A->nrows == A->ncols, PB_INVALID_INPUT, "CARP-CG needs a square matrix");
  const float zs = 0.0f;
  const double zd = 0.0;
  if (mixed) {
    SCopy s;
    int e = 0;
    phist_b200_sparseMat_DtoS(vA, &s.a, &e);
    PB_REQUIRE(e == 0 && s.a, e ? e : PB_FUNCTIONAL_ERROR, "FP32 copy of the matrix failed");
    WorkGuard<float> g{carp_build<float>(SP<float>(s.a), 1, &zs, nullptr, std::min(nsys, 16))};
    *block = carpcg_tune_block<float>(SP<float>(s.a), g.w, nsys, reps, iter_us);
  } else {
    WorkGuard<double> g{carp_build<double>(A, 1, &zd, nullptr, std::min(nsys, 16))};
    *block = carpcg_tune_block<double>(A, g.w, nsys, reps, iter_us);
  }
  PB_API_END(iflag);
}

void phist_b200_DcarpCG_batch(const void* vA, int nsys, const double* sigma, const void* vB, void* vX, int block,
                              double tol, int maxIter, int checkEvery, int mixed, double innerTol, int* iters,
                              double* relres, int* iflag)
{
  PB_API_BEGIN(iflag);
  using namespace pb;
  const SparseMat<double>* A = SP<double>(vA);
  const Mvec<double>* B = MV<double>(vB);
  Mvec<double>* X = MV<double>(vX);
  PB_REQUIRE(nsys >= 0 && block <= 32, PB_INVALID_INPUT,
             "need nsys >= 0 and block <= 32 (got %d, %d; block <= 0: tuned)", nsys, block);
  if (nsys == 0) {
    *iflag = 0;
    return;
  }
  PB_REQUIRE(A->nrows == A->ncols, PB_INVALID_INPUT, "CARP-CG needs a square matrix");
  PB_REQUIRE(B->nvec == nsys && X->nvec == nsys && B->nrows == A->nrows && X->nrows == A->nrows, PB_INVALID_INPUT,
             "B and X must be n x nsys");
  PB_REQUIRE(nsys == 0 || (sigma && iters && relres), PB_INVALID_INPUT, "sigma, iters and relres are required");
  PB_REQUIRE(tol > 0.0 && maxIter > 0 && checkEvery > 0, PB_INVALID_INPUT, "tol, maxIter, checkEvery must be > 0");
  int unconverged = 0;
  if (nsys > 0) {
    // the colouring does not depend on the shifts: built once, for the
    // given slot count or, when the tuner picks it, for 16 slots (what it
    // picks on the benchmark matrices), and used by the tuner and the solver
    const float zs = 0.0f;
    const double zd = 0.0;
    if (mixed) {
      SCopy s;
      int e = 0;
      phist_b200_sparseMat_DtoS(vA, &s.a, &e);
      PB_REQUIRE(e == 0 && s.a, e ? e : PB_FUNCTIONAL_ERROR, "FP32 copy of the matrix failed");
      const SparseMat<float>* As = SP<float>(s.a);
      WorkGuard<float> g{carp_build<float>(As, 1, &zs, nullptr, block >= 1 ? block : std::min(nsys, 16))};
      const int w = block >= 1 ? std::min(block, nsys) : carpcg_tune_block<float>(As, g.w, nsys, 3, nullptr);
      unconverged = carpcg_batch<float>(A, As, g.w, nsys, sigma, B, X, w, tol, maxIter, checkEvery,
                                        innerTol > 0.0 ? innerTol : 1e-5, iters, relres);
    } else {
      WorkGuard<double> g{carp_build<double>(A, 1, &zd, nullptr, block >= 1 ? block : std::min(nsys, 16))};
      const int w = block >= 1 ? std::min(block, nsys) : carpcg_tune_block<double>(A, g.w, nsys, 3, nullptr);
      unconverged = carpcg_batch<double>(A, A, g.w, nsys, sigma, B, X, w, tol, maxIter, checkEvery, tol, iters,
                                         relres);
    }
  }
  *iflag = unconverged;
  PB_API_END(iflag);
}
}
