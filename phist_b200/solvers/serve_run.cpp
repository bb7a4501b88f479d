// serve_run.cpp -- a served stream of eigen-solves on one GPU: PHIST's
// unchanged block Jacobi-Davidson (phist_Dsubspacejada) per request, many
// requests in flight at once.
//
// Requests arrive as a Poisson stream (exponential gaps of mean 1/rate from a
// seeded generator).  Request i asks for the `numEigs` smallest eigenpairs of
// the 7-point Laplacian plus a random diagonal uniform[0,1) on an L^3 grid
// (L log-uniform in [lmin, lmax], own seed).  A pool of `workers` host
// threads serves them: a free worker takes the next request once it has
// arrived, waits until the request's estimated device-memory footprint fits
// in the budget (admission by footprint; the budget is budget_frac of the
// free device memory at start), builds the matrix and solves.  Every worker
// drives the library on its own lane (CUDA stream, scratch, memory cache),
// so the kernels of concurrent solves overlap on the GPU and a worker that
// finishes refills its slot with the next waiting request: continuous
// batching, not a queue served one at a time.
//
//   serve_run [key=value ...]
//   keys: nreq (32) rate (200) workers (8) lmin (24) lmax (128) seed (5)
//         numEigs (8) blockSize (4) minBas (16) maxBas (32) tol (1e-10)
//         maxIters (400) mixed (0: FP64; 1: FP32 correction equations,
//         pb_mixed_jada.h) devgmres (1: correction equations on the
//         library's device-resident GMRES) minres (1: MINRES for the
//         correction equations, on the device with devgmres=1; the served
//         matrices are symmetric) budget_frac (0.8)
//         only=<i> : serve request i alone (arrival at once), for checking
//                    that a result is the same alone and in the mix
// Output: one JSON line with per-request latency (completion - arrival),
// p50/p99, solves/s, outer iterations, explicit residuals and eigenvalues.
#include <algorithm>
#include <atomic>
#include <chrono>
#include <cmath>
#include <condition_variable>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <mutex>
#include <string>
#include <thread>
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
void phist_b200_device_memory(uint64_t* free_bytes, uint64_t* total_bytes, int* iflag);
void phist_b200_synchronize(int* iflag);
void phist_b200_lane_count(int* nlanes, int* iflag);
}

namespace {

uint64_t mix64(uint64_t z)
{
  z += 0x9E3779B97F4A7C15ull;
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return z ^ (z >> 31);
}
// uniform [0,1) and [-1,1) from a splitmix64 hash of (seed, index)
double u01(uint64_t seed, uint64_t idx)
{
  return (double)(mix64(seed * 0x632BE59BD9B4E019ull + mix64(idx)) >> 11) * (1.0 / 9007199254740992.0);
}
double unif(uint64_t seed, uint64_t idx) { return 2.0 * u01(seed, idx) - 1.0; }

struct Request {
  int id = 0;
  double arrival = 0.0;  // seconds after the stream start
  int L = 0;
  uint64_t seed = 0;
  double footprint = 0.0;  // bytes
};

struct Result {
  double start = 0.0, end = 0.0;
  int nConv = 0, nIter = 0, err = 0;
  std::vector<double> ev, res;
};

struct Opts {
  int numEigs = 8, blockSize = 4, minBas = 16, maxBas = 32, maxIters = 400, mixed = 0, devgmres = 0, minres = 0;
  double tol = 1e-10;
};

// device bytes a solve of an n-row problem holds: matrix (SELL, 7 entries a
// row, and its host-side FP32 copy for the mixed form) plus the block
// vectors of subspacejada and its GMRES states
double footprint(int64_t n, const Opts& o)
{
  const double mat = 7.0 * 12.0 * n * (o.mixed ? 1.5 : 1.0);
  const double vecs = 8.0 * n * (3.0 * o.maxBas + 25.0 * o.blockSize + o.numEigs + 8.0);
  return mat + vecs;
}

#define WCHK(call)              \
  do {                          \
    iflag = 0;                  \
    call;                       \
    if (iflag < 0) {            \
      r.err = iflag;            \
      return;                   \
    }                           \
  } while (0)

void solve(const Request& q, const Opts& o, phist_const_comm_ptr comm, Result& r)
{
  int iflag = 0;
  char prob[64];
  snprintf(prob, sizeof(prob), "LAPDIAG3D-%d-S%llu", q.L, (unsigned long long)q.seed);
  phist_DsparseMat_ptr A = NULL;
  iflag = 0;
  phist_b200_Dcreate_problem(&A, comm, prob, &iflag);
  if (iflag < 0) {
    r.err = iflag;
    return;
  }
  phist_jadaOpts opts;
  phist_jadaOpts_setDefaults(&opts);
  opts.numEigs = o.numEigs;
  opts.which = phist_SR;
  opts.blockSize = o.blockSize;
  opts.minBas = o.minBas;
  opts.maxBas = o.maxBas;
  opts.convTol = o.tol;
  opts.maxIters = o.maxIters;
  opts.innerSolvType = o.minres ? phist_MINRES : phist_GMRES;
  opts.innerSolvMaxIters = 20;
  opts.symmetry = phist_HERMITIAN;
  pb_mixed_jada* mj = NULL;
  if (o.mixed || o.devgmres) {
    WCHK(phist_b200_jada_inner_create(&mj, A, &opts, o.mixed ? 1 : 0, o.devgmres, &iflag));
    WCHK(phist_b200_mixed_jada_install(mj, &opts, &iflag));
  }
  phist_DlinearOp opA;
  WCHK(phist_DlinearOp_wrap_sparseMat(&opA, A, &iflag));
  phist_const_map_ptr map = NULL;
  WCHK(phist_DsparseMat_get_domain_map(A, &map, &iflag));
  phist_lidx nloc = 0;
  WCHK(phist_map_get_local_length(map, &nloc, &iflag));
  const int nQ = o.numEigs + o.blockSize - 1;
  phist_Dmvec_ptr Q = NULL, v0 = NULL, res = NULL;
  phist_DsdMat_ptr R = NULL;
  WCHK(phist_Dmvec_create(&Q, map, nQ, &iflag));
  WCHK(phist_DsdMat_create(&R, nQ, nQ, comm, &iflag));
  WCHK(phist_Dmvec_create(&v0, map, 1, &iflag));
  WCHK(phist_Dmvec_create(&res, map, nQ, &iflag));
  {
    std::vector<double> h(nloc);
    for (phist_lidx i = 0; i < nloc; i++) h[i] = unif(q.seed, (uint64_t)i);
    WCHK(phist_Dmvec_set_data(v0, h.data(), 1, 1, &iflag));
  }
  opts.v0 = v0;
  std::vector<phist_d_complex> ev(nQ);
  std::vector<double> resNorm(nQ, 0.0);
  int nConv = o.numEigs, nIter = o.maxIters;
  iflag = 0;
  phist_Dsubspacejada(&opA, NULL, opts, Q, R, ev.data(), resNorm.data(), &nConv, &nIter, &iflag);
  if (iflag < 0) {
    r.err = iflag;
    return;
  }
  // explicit residuals ||A q_j - (Q R)_j||
  WCHK(phist_DsparseMat_times_mvec(1.0, A, Q, 0.0, res, &iflag));
  WCHK(phist_Dmvec_times_sdMat(-1.0, Q, R, 1.0, res, &iflag));
  std::vector<double> rn(nQ);
  WCHK(phist_Dmvec_norm2(res, rn.data(), &iflag));
  r.nConv = nConv;
  r.nIter = nIter;
  for (int j = 0; j < std::min(nConv, o.numEigs); j++) {
    r.ev.push_back(std::real(ev[j]));
    r.res.push_back(rn[j]);
  }
  std::sort(r.ev.begin(), r.ev.end());
  WCHK(phist_Dmvec_delete(res, &iflag));
  WCHK(phist_Dmvec_delete(v0, &iflag));
  WCHK(phist_Dmvec_delete(Q, &iflag));
  WCHK(phist_DsdMat_delete(R, &iflag));
  if (mj) WCHK(phist_b200_mixed_jada_delete(mj, &iflag));
  WCHK(phist_DsparseMat_delete(A, &iflag));
  WCHK(phist_b200_synchronize(&iflag));
}

double percentile(std::vector<double> v, double p)
{
  if (v.empty()) return 0.0;
  std::sort(v.begin(), v.end());
  const double pos = p * (v.size() - 1);
  const size_t i = (size_t)pos;
  const double f = pos - i;
  return i + 1 < v.size() ? v[i] * (1 - f) + v[i + 1] * f : v[i];
}

}  // namespace

int main(int argc, char** argv)
{
  int nreq = 32, workers = 8, lmin = 24, lmax = 128, only = -1;
  double rate = 200.0, budget_frac = 0.8;
  uint64_t seed = 5;
  Opts o;
  for (int a = 1; a < argc; a++) {
    const char* kv = argv[a];
    const char* eq = strchr(kv, '=');
    if (!eq) continue;
    std::string k(kv, eq - kv);
    const char* v = eq + 1;
    if (k == "nreq") nreq = atoi(v);
    else if (k == "rate") rate = atof(v);
    else if (k == "workers") workers = atoi(v);
    else if (k == "lmin") lmin = atoi(v);
    else if (k == "lmax") lmax = atoi(v);
    else if (k == "seed") seed = strtoull(v, nullptr, 10);
    else if (k == "numEigs") o.numEigs = atoi(v);
    else if (k == "blockSize") o.blockSize = atoi(v);
    else if (k == "minBas") o.minBas = atoi(v);
    else if (k == "maxBas") o.maxBas = atoi(v);
    else if (k == "tol") o.tol = atof(v);
    else if (k == "maxIters") o.maxIters = atoi(v);
    else if (k == "mixed") o.mixed = atoi(v);
    else if (k == "devgmres") o.devgmres = atoi(v);
    else if (k == "minres") o.minres = atoi(v);
    else if (k == "budget_frac") budget_frac = atof(v);
    else if (k == "only") only = atoi(v);
  }
  if (nreq < 1 || workers < 1 || lmin < 4 || lmax < lmin || rate <= 0.0) return 2;

  // the request stream (the same for every run with this seed)
  std::vector<Request> reqs(nreq);
  double t = 0.0;
  for (int i = 0; i < nreq; i++) {
    t += -std::log(1.0 - u01(seed, 2 * (uint64_t)i)) / rate;
    const double lu = std::log((double)lmin) + u01(seed, 2 * (uint64_t)i + 1) * (std::log((double)lmax) - std::log((double)lmin));
    reqs[i].id = i;
    reqs[i].arrival = t;
    reqs[i].L = std::min(lmax, std::max(lmin, (int)std::lround(std::exp(lu))));
    reqs[i].seed = seed * 1000003ull + (uint64_t)i;
    reqs[i].footprint = footprint((int64_t)reqs[i].L * reqs[i].L * reqs[i].L, o);
  }
  std::vector<int> order;
  if (only >= 0 && only < nreq) {
    order.push_back(only);
    reqs[only].arrival = 0.0;
  } else {
    for (int i = 0; i < nreq; i++) order.push_back(i);
  }

  int iflag = 0;
  phist_kernels_init(&argc, &argv, &iflag);
  if (iflag < 0) return 1;
  phist_comm_ptr comm = NULL;
  phist_comm_create(&comm, &iflag);
  uint64_t freeb = 0, totalb = 0;
  phist_b200_device_memory(&freeb, &totalb, &iflag);
  const double budget = budget_frac * (double)freeb;

  std::vector<Result> results(nreq);
  std::atomic<int> next{0};
  std::mutex mu;
  std::condition_variable cv;
  double inflight = 0.0, peak_inflight = 0.0;
  int max_concurrent = 0, concurrent = 0;
  const auto t0 = std::chrono::steady_clock::now();
  auto now = [&]() { return std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count(); };

  auto worker = [&]() {
    for (;;) {
      const int k = next.fetch_add(1);
      if (k >= (int)order.size()) break;
      const Request& q = reqs[order[k]];
      const double wait = q.arrival - now();
      if (wait > 0) std::this_thread::sleep_for(std::chrono::duration<double>(wait));
      {
        // admission by footprint (a request larger than the whole budget
        // runs alone)
        std::unique_lock<std::mutex> lk(mu);
        cv.wait(lk, [&] { return inflight == 0.0 || inflight + q.footprint <= budget; });
        inflight += q.footprint;
        peak_inflight = std::max(peak_inflight, inflight);
        max_concurrent = std::max(max_concurrent, ++concurrent);
      }
      Result& r = results[q.id];
      r.start = now();
      solve(q, o, comm, r);
      r.end = now();
      {
        std::lock_guard<std::mutex> lk(mu);
        inflight -= q.footprint;
        concurrent--;
      }
      cv.notify_all();
    }
  };
  std::vector<std::thread> pool;
  for (int w = 0; w < workers; w++) pool.emplace_back(worker);
  for (auto& th : pool) th.join();
  const double wall = now();

  std::vector<double> lat;
  double first_arr = 1e300, last_end = 0.0, maxres = 0.0;
  int failed = 0, unconverged = 0;
  for (int i : order) {
    const Result& r = results[i];
    lat.push_back(r.end - reqs[i].arrival);
    first_arr = std::min(first_arr, reqs[i].arrival);
    last_end = std::max(last_end, r.end);
    failed += r.err != 0;
    unconverged += r.nConv < o.numEigs;
    for (double x : r.res) maxres = std::max(maxres, x);
  }
  int nlanes = 0;
  phist_b200_lane_count(&nlanes, &iflag);
  printf("{\"served\": %d, \"workers\": %d, \"mixed\": %d, \"devgmres\": %d, \"minres\": %d, \"rate\": %g, \"seed\": %llu, \"numEigs\": %d, "
         "\"tol\": %.1e, \"failed\": %d, \"unconverged\": %d, \"max_resExplicit\": %.3e, \"wall\": %.4f, "
         "\"solves_per_s\": %.4f, \"latency_p50\": %.4f, \"latency_p99\": %.4f, \"latency_mean\": %.4f, "
         "\"max_concurrent\": %d, \"lanes\": %d, \"budget_GB\": %.2f, \"peak_admitted_GB\": %.3f, \"requests\": [",
         (int)order.size(), workers, o.mixed, o.devgmres, o.minres, rate, (unsigned long long)seed, o.numEigs, o.tol, failed, unconverged,
         maxres, wall, order.size() / std::max(1e-9, last_end - first_arr), percentile(lat, 0.5),
         percentile(lat, 0.99), [&] { double s = 0; for (double x : lat) s += x; return s / lat.size(); }(),
         max_concurrent, nlanes, budget / 1e9, peak_inflight / 1e9);
  for (size_t k = 0; k < order.size(); k++) {
    const int i = order[k];
    const Result& r = results[i];
    printf("%s{\"id\": %d, \"L\": %d, \"arrival\": %.5f, \"start\": %.5f, \"end\": %.5f, \"nIter\": %d, "
           "\"nConv\": %d, \"err\": %d, \"ev\": [",
           k ? ", " : "", i, reqs[i].L, reqs[i].arrival, r.start, r.end, r.nIter, r.nConv, r.err);
    for (size_t j = 0; j < r.ev.size(); j++) printf("%s%.17g", j ? ", " : "", r.ev[j]);
    printf("]}");
  }
  printf("]}\n");
  fflush(stdout);
  phist_comm_delete(comm, &iflag);
  phist_kernels_finalize(&iflag);
  return failed ? 1 : 0;
}
