// pb_runtime.cu -- runtime (device, stream, memory cache) and the
// type-independent part of the phist_kernels C API
// (src/kernels/phist_kernels.h:79-185 in the PHIST sources).
#include <chrono>
#include <string>

#include "pb_core.hpp"
#include "pb_tma.cuh"


namespace pb {

void report(const char* fcn, const char* msg)
{
  if (getenv("PHIST_B200_QUIET")) return;
  fprintf(stderr, "[phist_b200] %s: %s\n", fcn, msg);
}

Runtime& Runtime::get()
{
  static Runtime r;
  return r;
}

void Runtime::init()
{
  std::lock_guard<std::mutex> g(mu_);
  if (inited_) return;
  int ndev = 0;
  cudaError_t e = cudaGetDeviceCount(&ndev);
  PB_REQUIRE(e == cudaSuccess && ndev > 0, PB_FUNCTIONAL_ERROR,
             "no CUDA device available (%s): this library has no CPU path",
             cudaGetErrorString(e));
  // one process per GPU: honour LOCAL_RANK when launched by torchrun
  const char* lr = getenv("LOCAL_RANK");
  device_ = lr ? atoi(lr) % ndev : 0;
  PB_CUDA(cudaSetDevice(device_));
  cudaDeviceProp prop;
  PB_CUDA(cudaGetDeviceProperties(&prop, device_));
  num_sms_ = prop.multiProcessorCount;
  if (prop.l2CacheSize > 0) l2_bytes_ = prop.l2CacheSize;
  if (const char* v = getenv("PHIST_B200_VERBOSE")) verbose = atoi(v);
  if (const char* v = getenv("PHIST_B200_TMA")) use_tma = atoi(v) != 0;
  if (const char* v = getenv("PHIST_B200_DMMA")) use_dmma = atoi(v) != 0;
  if (const char* v = getenv("PHIST_B200_GRAPHS")) use_graphs = atoi(v) != 0;
  if (const char* c = getenv("PHIST_B200_SELL_C")) sell_C = atoi(c);
  if (const char* s = getenv("PHIST_B200_SELL_SIGMA")) sell_sigma_default = atoll(s);
  if (const char* v = getenv("PHIST_B200_SPMV_PREFETCH")) spmv_pf = atoi(v) != 0;
  if (const char* v = getenv("PHIST_B200_SPMV_V256")) spmv_v256 = atoi(v) != 0;
  if (const char* v = getenv("PHIST_B200_CARP_BLOCKS")) carp_blocks = atoi(v) != 0;
  if (const char* v = getenv("PHIST_B200_CARP_BLOCK_ROWS")) carp_block_rows = std::max(0, std::min(256, atoi(v)));
  if (const char* v = getenv("PHIST_B200_CARP_PDL")) carp_pdl = atoi(v) != 0;
  noalloc_setup_current_device();
  inited_ = true;
}

Lane* Runtime::create_lane_locked()
{
  PB_CUDA(cudaSetDevice(device_));
  Lane* l = new Lane();
  PB_CUDA(cudaStreamCreateWithFlags(&l->stream, cudaStreamNonBlocking));
  PB_CUDA(cudaMalloc(&l->counters, 64 * sizeof(unsigned int)));
  PB_CUDA(cudaMemset(l->counters, 0, 64 * sizeof(unsigned int)));
  PB_CUDA(cudaHostAlloc(&l->mbox_h, kMailboxBytes, cudaHostAllocMapped));
  PB_CUDA(cudaHostGetDevicePointer(&l->mbox_d, l->mbox_h, 0));
  memset(l->mbox_h, 0, kMailboxBytes);
  l->generation = generation_;
  return l;
}

void Runtime::free_lane_locked(Lane* l)
{
  if (l->stream) cudaStreamSynchronize(l->stream);
  for (auto& kv : l->free_blocks) cudaFree(kv.second);
  l->free_blocks.clear();
  if (l->scratch) cudaFree(l->scratch);
  if (l->counters) cudaFree(l->counters);
  if (l->mbox_h) cudaFreeHost(l->mbox_h);
  if (l->stream) cudaStreamDestroy(l->stream);
  l->scratch = nullptr;
  l->scratch_bytes = 0;
  l->counters = nullptr;
  l->mbox_h = l->mbox_d = nullptr;
  l->stream = nullptr;
}

namespace {
// the calling thread's lane; returned to the pool when the thread exits
struct LaneHolder {
  Lane* lane = nullptr;
  unsigned generation = 0;
  ~LaneHolder()
  {
    if (lane) Runtime::get().release_lane(lane, generation);
  }
};
thread_local LaneHolder tl_lane;
}  // namespace

Lane& Runtime::lane()
{
  if (tl_lane.lane && tl_lane.generation == generation_ && inited_) return *tl_lane.lane;
  if (!inited_) init();
  std::lock_guard<std::mutex> g(mu_);
  Lane* l = nullptr;
  for (Lane* c : lanes_)
    if (!c->in_use && c->generation == generation_) {
      l = c;
      break;
    }
  if (!l) {
    l = create_lane_locked();
    lanes_.push_back(l);
  }
  l->in_use = true;
  tl_lane.lane = l;
  tl_lane.generation = generation_;
  return *l;
}

void Runtime::release_lane(Lane* l, unsigned generation)
{
  if (!inited_ || generation != generation_) return;
  if (l->stream) cudaStreamSynchronize(l->stream);
  std::lock_guard<std::mutex> g(mu_);
  l->in_use = false;
}

void Runtime::finalize()
{
  std::lock_guard<std::mutex> g(mu_);
  if (!inited_) return;
  for (Lane* l : lanes_) {
    free_lane_locked(l);
    delete l;
  }
  lanes_.clear();
  for (auto& kv : live_blocks_) cudaFree(kv.first);
  live_blocks_.clear();
  generation_++;  // lanes still referenced by threads are stale from now on
  inited_ = false;
}

static size_t round_block(size_t bytes)
{
  // 512-byte granularity below 1 MiB, 2 MiB granularity above
  if (bytes < (1u << 20)) return (bytes + 511) & ~size_t(511);
  return (bytes + (2u << 20) - 1) & ~size_t((2u << 20) - 1);
}

void* Runtime::dmalloc(size_t bytes)
{
  Lane& L = lane();
  size_t rb = round_block(bytes ? bytes : 1);
  std::lock_guard<std::mutex> g(mu_);
  auto it = L.free_blocks.find(rb);
  void* p = nullptr;
  if (it != L.free_blocks.end()) {
    p = it->second;
    L.free_blocks.erase(it);
  } else {
    cudaError_t e = cudaMalloc(&p, rb);
    if (e != cudaSuccess) {
      // release every lane's cache (cudaFree waits for the device) and retry once
      cudaGetLastError();
      for (Lane* l : lanes_) {
        if (l->stream) cudaStreamSynchronize(l->stream);
        for (auto& kv : l->free_blocks) cudaFree(kv.second);
        l->free_blocks.clear();
      }
      e = cudaMalloc(&p, rb);
      if (e != cudaSuccess) {
        cudaGetLastError();
        PB_THROW(PB_MEM_ALLOC_FAILED, "device allocation of %zu bytes failed", rb);
      }
    }
  }
  live_blocks_[p] = rb;
  return p;
}

void Runtime::dfree(void* p)
{
  if (!p || !inited_) return;
  Lane& L = lane();
  std::lock_guard<std::mutex> g(mu_);
  auto it = live_blocks_.find(p);
  if (it == live_blocks_.end()) return;
  L.free_blocks.emplace(it->second, p);
  live_blocks_.erase(it);
}

void* Runtime::hmalloc_pinned(size_t bytes)
{
  if (!inited_) init();
  void* p = nullptr;
  PB_CUDA(cudaMallocHost(&p, bytes ? bytes : 1));
  return p;
}

void Runtime::hfree_pinned(void* p)
{
  if (p) cudaFreeHost(p);
}

void Runtime::sync()
{
  Lane& L = lane();
  PB_CUDA(cudaStreamSynchronize(L.stream));
  volatile int* err = (volatile int*)((char*)L.mbox_h + kMailboxResultBytes);
  if (*err != 0) {
    const int e = *err;
    *err = 0;
    PB_THROW(PB_FUNCTIONAL_ERROR, "a device-side wait timed out (code %d); results of the last calls are invalid", e);
  }
}

void* Runtime::scratch(size_t bytes)
{
  Lane& L = lane();
  if (bytes > L.scratch_bytes) {
    // grow: the old buffer may still be read by enqueued kernels
    PB_CUDA(cudaStreamSynchronize(L.stream));
    if (L.scratch) PB_CUDA(cudaFree(L.scratch));
    L.scratch = nullptr;
    L.scratch_bytes = 0;
    size_t nb = bytes < (4u << 20) ? (4u << 20) : bytes * 2;
    PB_CUDA(cudaMalloc(&L.scratch, nb));
    L.scratch_bytes = nb;
  }
  return L.scratch;
}

unsigned int* Runtime::counters() { return lane().counters; }

// ----------------------------------------------------- STREAM benchmarks
__global__ void k_stream_load(const double* __restrict__ a, int64_t n, double* out)
{
  double s = 0.0;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x)
    s += a[i];
  if (s == 12345.678) out[0] = s;  // keep the loads alive
}
__global__ void k_stream_store(double* __restrict__ a, int64_t n, double v)
{
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x)
    a[i] = v;
}
__global__ void k_stream_copy(const double* __restrict__ a, double* __restrict__ b, int64_t n)
{
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x)
    b[i] = a[i];
}
__global__ void k_stream_triad(const double* __restrict__ a, const double* __restrict__ b,
                               double* __restrict__ c, int64_t n, double s)
{
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x)
    c[i] = a[i] + s * b[i];
}

// kind: 0 load, 1 store, 2 copy, 3 triad; Gbyte/s over 10 runs
static void stream_bench(int kind, double* mean_bw, double* max_bw)
{
  Runtime& r = rt();
  if (!r.initialized()) r.init();
  const int64_t n = int64_t(1) << 27;  // 1 GiB per array
  double *a = (double*)r.dmalloc(n * 8), *b = (double*)r.dmalloc(n * 8),
         *c = (double*)r.dmalloc(n * 8);
  cudaStream_t s = r.stream();
  PB_CUDA(cudaMemsetAsync(a, 0, n * 8, s));
  PB_CUDA(cudaMemsetAsync(b, 0, n * 8, s));
  cudaEvent_t e0, e1;
  PB_CUDA(cudaEventCreate(&e0));
  PB_CUDA(cudaEventCreate(&e1));
  const int grid = r.num_sms() * 8, block = 256;
  const double bytes[4] = {8.0 * n, 8.0 * n, 16.0 * n, 24.0 * n};
  double sum = 0, best = 0;
  const int reps = 10;
  for (int it = 0; it <= reps; it++) {
    PB_CUDA(cudaEventRecord(e0, s));
    switch (kind) {
      case 0: k_stream_load<<<grid, block, 0, s>>>(a, n, c); break;
      case 1: k_stream_store<<<grid, block, 0, s>>>(a, n, 1.0); break;
      case 2: k_stream_copy<<<grid, block, 0, s>>>(a, b, n); break;
      default: k_stream_triad<<<grid, block, 0, s>>>(a, b, c, n, 3.0); break;
    }
    PB_LAUNCH_CHECK();
    PB_CUDA(cudaEventRecord(e1, s));
    PB_CUDA(cudaEventSynchronize(e1));
    float ms = 0;
    PB_CUDA(cudaEventElapsedTime(&ms, e0, e1));
    if (it == 0) continue;  // warm-up
    double bw = bytes[kind] / (ms * 1e-3) / 1e9;
    sum += bw;
    if (bw > best) best = bw;
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  r.dfree(a);
  r.dfree(b);
  r.dfree(c);
  *mean_bw = sum / reps;
  *max_bw = best;
}

}  // namespace pb

using namespace pb;

extern "C" {

void phist_kernels_init(int* argc, char*** argv, int* iflag)
{
  (void)argc;
  (void)argv;
  PB_API_BEGIN(iflag);
  rt().init();
  PB_API_END(iflag);
}

void phist_kernels_finalize(int* iflag)
{
  PB_API_BEGIN(iflag);
  rt().finalize();
  PB_API_END(iflag);
}

void phist_kernels_common_init(int* argc, char*** argv, int* iflag)
{
  phist_kernels_init(argc, argv, iflag);
}

void phist_kernels_common_finalize(int* iflag) { *iflag = 0; }

const char* phist_kernel_lib(void) { return "b200"; }
int phist_sizeof_lidx(void) { return (int)sizeof(int32_t); }
int phist_sizeof_gidx(void) { return (int)sizeof(int64_t); }

void phist_comm_create(void** comm, int* iflag)
{
  PB_API_BEGIN(iflag);
  PB_REQUIRE(comm, PB_BAD_CAST, "comm is NULL");
  if (!rt().initialized()) rt().init();
  *comm = new Comm();
  PB_API_END(iflag);
}

void phist_comm_delete(void* comm, int* iflag)
{
  PB_API_BEGIN(iflag);
  delete (Comm*)comm;
  PB_API_END(iflag);
}

// A NULL comm is the single process, as in PHIST's builds without MPI
// (their kernel tests never create a comm then, KernelTest.h:69-84).
void phist_comm_get_rank(const void* comm, int* rank, int* iflag)
{
  PB_API_BEGIN(iflag);
  PB_REQUIRE(rank, PB_BAD_CAST, "rank is NULL");
  *rank = comm ? ((const Comm*)comm)->rank : 0;
  PB_API_END(iflag);
}

void phist_comm_get_size(const void* comm, int* size, int* iflag)
{
  PB_API_BEGIN(iflag);
  PB_REQUIRE(size, PB_BAD_CAST, "size is NULL");
  *size = comm ? ((const Comm*)comm)->size : 1;
  PB_API_END(iflag);
}

void phist_comm_get_mpi_comm(const void* comm, int* mpiComm, int* iflag)
{
  PB_API_BEGIN(iflag);
  (void)comm;
  if (mpiComm) *mpiComm = 0;
  PB_API_END(iflag);
}

void phist_map_create(void** map, const void* comm, int64_t nglob, int* iflag)
{
  PB_API_BEGIN(iflag);
  PB_REQUIRE(map, PB_BAD_CAST, "map is NULL");  // comm NULL: the single process
  PB_REQUIRE(nglob >= 0 && nglob < (int64_t(1) << 31), PB_INTEGER_OVERFLOW,
             "global length %lld does not fit the 32-bit local index", (long long)nglob);
  Map* m = new Map();
  m->comm = (const Comm*)comm;
  m->nglob = nglob;
  m->nloc = (int32_t)nglob;
  m->ilower = 0;
  *map = m;
  PB_API_END(iflag);
}

void phist_map_delete(void* map, int* iflag)
{
  PB_API_BEGIN(iflag);
  delete (Map*)map;
  PB_API_END(iflag);
}

void phist_map_get_comm(const void* map, const void** comm, int* iflag)
{
  PB_API_BEGIN(iflag);
  PB_REQUIRE(map, PB_BAD_CAST, "map is NULL");
  *comm = ((const Map*)map)->comm;
  PB_API_END(iflag);
}

void phist_map_get_local_length(const void* map, int32_t* nloc, int* iflag)
{
  PB_API_BEGIN(iflag);
  PB_REQUIRE(map, PB_BAD_CAST, "map is NULL");
  *nloc = ((const Map*)map)->nloc;
  PB_API_END(iflag);
}

void phist_map_get_global_length(const void* map, int64_t* nglob, int* iflag)
{
  PB_API_BEGIN(iflag);
  PB_REQUIRE(map, PB_BAD_CAST, "map is NULL");
  *nglob = ((const Map*)map)->nglob;
  PB_API_END(iflag);
}

void phist_map_get_ilower(const void* map, int64_t* ilower, int* iflag)
{
  PB_API_BEGIN(iflag);
  PB_REQUIRE(map, PB_BAD_CAST, "map is NULL");
  *ilower = ((const Map*)map)->ilower;
  PB_API_END(iflag);
}

void phist_map_get_iupper(const void* map, int64_t* iupper, int* iflag)
{
  PB_API_BEGIN(iflag);
  PB_REQUIRE(map, PB_BAD_CAST, "map is NULL");
  const Map* m = (const Map*)map;
  *iupper = m->ilower + m->nloc - 1;
  PB_API_END(iflag);
}

void phist_maps_compatible(const void* map1, const void* map2, int* iflag)
{
  PB_API_BEGIN(iflag);
  PB_REQUIRE(map1 && map2, PB_BAD_CAST, "map is NULL");
  const Map* a = (const Map*)map1;
  const Map* b = (const Map*)map2;
  // block vectors are always stored in the original row order, so maps of
  // equal length describe the same distribution and ordering
  *iflag = (a->nglob == b->nglob && a->nloc == b->nloc && a->ilower == b->ilower) ? 0 : -1;
  PB_API_END(iflag);
}

void phist_context_create(void** ctx, const void* row_map, const void* col_map,
                          const void* range_map, const void* domain_map, int* iflag)
{
  PB_API_BEGIN(iflag);
  PB_REQUIRE(ctx && row_map, PB_BAD_CAST, "context or row map is NULL");
  Context* c = new Context();
  c->row_map = (const Map*)row_map;
  c->col_map = (const Map*)col_map;
  c->range_map = range_map ? (const Map*)range_map : c->row_map;
  c->domain_map = domain_map ? (const Map*)domain_map : c->row_map;
  *ctx = c;
  PB_API_END(iflag);
}

void phist_context_delete(void* ctx, int* iflag)
{
  PB_API_BEGIN(iflag);
  delete (Context*)ctx;
  PB_API_END(iflag);
}

void phist_bench_stream_load(double* mean_bw, double* max_bw, int* iflag)
{
  PB_API_BEGIN(iflag);
  stream_bench(0, mean_bw, max_bw);
  PB_API_END(iflag);
}
void phist_bench_stream_store(double* mean_bw, double* max_bw, int* iflag)
{
  PB_API_BEGIN(iflag);
  stream_bench(1, mean_bw, max_bw);
  PB_API_END(iflag);
}
void phist_bench_stream_copy(double* mean_bw, double* max_bw, int* iflag)
{
  PB_API_BEGIN(iflag);
  stream_bench(2, mean_bw, max_bw);
  PB_API_END(iflag);
}
void phist_bench_stream_triad(double* mean_bw, double* max_bw, int* iflag)
{
  PB_API_BEGIN(iflag);
  stream_bench(3, mean_bw, max_bw);
  PB_API_END(iflag);
}

void phist_b200_set_sell_params(int C, int64_t sigma, int* iflag)
{
  PB_API_BEGIN(iflag);
  PB_REQUIRE(C >= 1 && C <= 32 && (C & (C - 1)) == 0, PB_INVALID_INPUT,
             "SELL chunk height must be a power of two in [1,32], got %d", C);
  rt().sell_C = C;
  rt().sell_sigma_default = sigma;
  PB_API_END(iflag);
}

void phist_b200_set_spmv_config(int nvec, int tpr, int unroll, int* iflag)
{
  PB_API_BEGIN(iflag);
  static const int allowed[6][3] = {{1, 1, 1}, {1, 1, 1}, {1, 2, 2}, {1, 2, 4}, {2, 4, 8}, {4, 8, 16}};
  int lg = -1;
  for (int q = 0; q < 6; q++)
    if (nvec == (1 << q)) lg = q;
  PB_REQUIRE(lg >= 0, PB_INVALID_INPUT, "nvec must be 1,2,4,8,16 or 32, got %d", nvec);
  PB_REQUIRE(tpr == allowed[lg][0] || tpr == allowed[lg][1] || tpr == allowed[lg][2], PB_INVALID_INPUT,
             "threads per row %d not available for nvec %d (use %d, %d or %d)", tpr, nvec,
             allowed[lg][0], allowed[lg][1], allowed[lg][2]);
  rt().spmv_tpr[lg] = tpr;
  if (unroll >= 0) rt().spmv_unroll = unroll != 0;
  PB_API_END(iflag);
}

void phist_b200_set_spmv_staged(int min_nvec, int* iflag)
{
  PB_API_BEGIN(iflag);
  rt().spmv_staged_min_nvec = min_nvec;
  PB_API_END(iflag);
}

void phist_b200_set_spmv_prefetch(int on, int* iflag)
{
  PB_API_BEGIN(iflag);
  rt().spmv_pf = on != 0;
  PB_API_END(iflag);
}

void phist_b200_set_graphs(int on, int* iflag)
{
  PB_API_BEGIN(iflag);
  rt().use_graphs = on != 0;
  PB_API_END(iflag);
}

void phist_b200_set_option(const char* name, int value, int* iflag)
{
  PB_API_BEGIN(iflag);
  PB_REQUIRE(name, PB_INVALID_INPUT, "option name is NULL");
  const std::string o(name);
  if (o == "tma") rt().use_tma = value != 0;
  else if (o == "dmma") rt().use_dmma = value != 0;
  else if (o == "graphs") rt().use_graphs = value != 0;
  else if (o == "carp_blocks") rt().carp_blocks = value != 0;
  else if (o == "spmv_v256") rt().spmv_v256 = value != 0;
  else PB_REQUIRE(false, PB_INVALID_INPUT, "unknown option '%s'", name);
  PB_API_END(iflag);
}

void phist_b200_synchronize(int* iflag)
{
  PB_API_BEGIN(iflag);
  if (rt().initialized()) rt().sync();
  PB_API_END(iflag);
}

}  // extern "C"

namespace pb {
// One thread waits, bounded, on an mbarrier that nothing completes: the wait
// runs out after about a second and stores its code in the device error
// word, exactly as a production kernel's timed-out copy wait does.
__global__ void k_bounded_wait_probe(int* err)
{
  __shared__ uint64_t bar;
  if (threadIdx.x == 0) {
    mbar_init(&bar, 1);
    mbar_fence_init();
  }
  __syncthreads();
  if (threadIdx.x == 0) mbar_wait(&bar, 0u, err);
  __syncthreads();
}
}  // namespace pb

extern "C" {

void phist_b200_selftest_bounded_wait(int* iflag)
{
  PB_API_BEGIN(iflag);
  pb::rt().init();
  pb::k_bounded_wait_probe<<<1, 32, 0, pb::stream()>>>(pb::rt().device_error_word());
  PB_LAUNCH_CHECK();
  pb::rt().sync();  // reports the timed-out wait and clears the word
  PB_API_END(iflag);
}

void phist_b200_launch_count(uint64_t* count, int* iflag)
{
  PB_API_BEGIN(iflag);
  *count = rt().launches;
  PB_API_END(iflag);
}

void phist_b200_lane_count(int* nlanes, int* iflag)
{
  PB_API_BEGIN(iflag);
  *nlanes = rt().lanes_created();
  PB_API_END(iflag);
}

void phist_b200_device_memory(uint64_t* free_bytes, uint64_t* total_bytes, int* iflag)
{
  PB_API_BEGIN(iflag);
  if (!rt().initialized()) rt().init();
  size_t f = 0, t = 0;
  PB_CUDA(cudaMemGetInfo(&f, &t));
  if (free_bytes) *free_bytes = f;
  if (total_bytes) *total_bytes = t;
  PB_API_END(iflag);
}

void phist_b200_get_stream(void** s, int* iflag)
{
  PB_API_BEGIN(iflag);
  if (!rt().initialized()) rt().init();
  *s = (void*)rt().stream();
  PB_API_END(iflag);
}

}  // extern "C"
