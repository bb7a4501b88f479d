// pb_noalloc.cu -- C = alpha*V'W + beta*C on raw device pointers, without
// any device allocation.
//
// The regular entry point phist_DmvecT_times_mvec keeps its per-block
// partial sums in a scratch buffer that the library allocates (and grows) on
// demand.  Some callers cannot allow that: an application that hands the
// library a fixed device-memory budget at start-up and owns every later
// allocation through its own pool, or a host that forbids cudaMalloc once it
// has initialised.  For them, phist_b200_DmvecT_times_mvec_noalloc computes
// the same product with its scratch in a fixed, file-scope device array, so a
// call never allocates.
//
// Limits and rules of use:
//  * V is n x m, W is n x k, both row-major with leading dimensions ldv >= m
//    and ldw >= k; C is m x k column-major with ldc >= m; all three are device
//    pointers the caller provides.  m and k must be in [1, 64]: the partial
//    sums of up to 128 thread blocks of a 64 x 64 result fill the 4 MiB
//    scratch array exactly.  Larger m or k are rejected with -55.
//  * The scratch array (4 MiB + 256 bytes) lives in every GPU that loads the
//    library, for the life of the process.
//  * The array's device address is looked up with cudaGetSymbolAddress once
//    per device, with that device current.  phist_kernels_init does this for
//    the device it selects; on any other device the first call does it, so
//    make that first call before any stream capture begins.  The looked-up
//    address is kept for the life of the process and is not looked up again
//    after a cudaDeviceReset: a host application that resets a device must
//    not call this entry point on that device afterwards.
//  * All calls share the one array, which keeps the last call's contents.
//    Calls that overlap on the GPU (for example on two streams at once) race
//    on it and give wrong results; serialise them.
#include <mutex>

#include "pb_block.cuh"

namespace {

constexpr size_t kScratchDoubles = size_t(1) << 19;  // 4 MiB of partial sums
constexpr int kMaxWidth = 64;
constexpr int kMaxDevices = 64;

__device__ __align__(256) double g_noalloc_scratch[kScratchDoubles];
__device__ __align__(256) unsigned int g_noalloc_counter[64];

struct DeviceSlot {
  bool ready = false;
  double* scratch = nullptr;         // device address of g_noalloc_scratch
  unsigned int* counter = nullptr;   // device address of g_noalloc_counter
  int num_sms = 0;
};

std::mutex g_mu;
DeviceSlot g_slot[kMaxDevices];

// one-time per-device set-up, with the device current
cudaError_t device_slot(DeviceSlot** out)
{
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  if (dev < 0 || dev >= kMaxDevices) return cudaErrorInvalidDevice;
  std::lock_guard<std::mutex> g(g_mu);
  DeviceSlot& s = g_slot[dev];
  if (!s.ready) {
    void* p = nullptr;
    e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess) return e;
    s.scratch = (double*)p;
    e = cudaGetSymbolAddress(&p, g_noalloc_counter);
    if (e != cudaSuccess) return e;
    s.counter = (unsigned int*)p;
    e = cudaDeviceGetAttribute(&s.num_sms, cudaDevAttrMultiProcessorCount, dev);
    if (e != cudaSuccess) return e;
    s.ready = true;
  }
  *out = &s;
  return cudaSuccess;
}

void fail(int* iflag, int code, const char* msg)
{
  if (!getenv("PHIST_B200_QUIET")) fprintf(stderr, "[phist_b200] mvecT_times_mvec_noalloc: %s\n", msg);
  *iflag = code;
}

}  // namespace

namespace pb {
// eager per-device set-up for the device current at library initialisation
void noalloc_setup_current_device()
{
  DeviceSlot* slot = nullptr;
  if (device_slot(&slot) != cudaSuccess) cudaGetLastError();
}
}  // namespace pb

extern "C" void phist_b200_DmvecT_times_mvec_noalloc(int64_t n, int m, int k, double alpha,
                                                     const double* V, int64_t ldv, const double* W,
                                                     int64_t ldw, double beta, double* C,
                                                     int64_t ldc, void* stream, int* iflag)
{
  if (!iflag) return;
  *iflag = 0;
  if (n < 0 || m < 1 || k < 1) return fail(iflag, -55, "need n >= 0, m >= 1, k >= 1");
  if (m > kMaxWidth || k > kMaxWidth)
    return fail(iflag, -55, "m and k must not exceed 64 (the fixed scratch holds 128 blocks of 64x64 partial sums)");
  if (ldv < m || ldw < k || ldc < m) return fail(iflag, -55, "leading dimension too small");
  if (!C || (n > 0 && (!V || !W))) return fail(iflag, -88, "NULL device pointer");

  DeviceSlot* slot = nullptr;
  cudaError_t e = device_slot(&slot);
  if (e != cudaSuccess) return fail(iflag, -1, cudaGetErrorString(e));
  cudaStream_t s = (cudaStream_t)stream;

  // launch shape of the library's k_mvTmv (same micro-tiles as launch_mvTmv)
  const bool big = m * k >= 256;
  const int TM = big ? 8 : 4, TK = big ? 8 : 4;
  const int mp = (m + TM - 1) / TM * TM, kp = (k + TK - 1) / TK * TK;
  const int nt = (mp / TM) * (kp / TK);
  const int RG = pb::BLK_BS / nt;
  int R = ((RG * 4 + 31) / 32) * 32;
  R = R < 32 ? 32 : (R > 128 ? 128 : R);
  size_t smem = sizeof(double) * (size_t)R * (mp + kp);
  const size_t red = sizeof(double) * (size_t)RG * mp * kp;
  if (red > smem) smem = red;
  const int64_t rows = n > 0 ? n : 1;
  int64_t grid = (rows + R - 1) / R;
  if (grid > 2 * (int64_t)slot->num_sms) grid = 2 * (int64_t)slot->num_sms;
  const int64_t cap = (int64_t)(kScratchDoubles / ((size_t)m * k));
  if (grid > cap) grid = cap;

  pb::MvTmvArgs<double> a;
  a.n = n; a.m = m; a.k = k;
  a.V = V; a.ldv = ldv; a.W = W; a.ldw = ldw;
  a.alpha = alpha; a.beta = beta;
  a.Cd = C; a.ldc = ldc;
  a.part = slot->scratch;
  a.counter = slot->counter;
  a.R = R;

  // the arrival counter must start at zero (an interrupted earlier launch
  // could have left it elsewhere)
  e = cudaMemsetAsync(slot->counter, 0, sizeof(unsigned int), s);
  if (e != cudaSuccess) return fail(iflag, -1, cudaGetErrorString(e));
  if (big) {
    auto kern = pb::k_mvTmv<double, 8, 8>;
    e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e == cudaSuccess) kern<<<(int)grid, pb::BLK_BS, smem, s>>>(a);
  } else {
    auto kern = pb::k_mvTmv<double, 4, 4>;
    e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e == cudaSuccess) kern<<<(int)grid, pb::BLK_BS, smem, s>>>(a);
  }
  if (e == cudaSuccess) e = cudaGetLastError();
  if (e != cudaSuccess) return fail(iflag, -1, cudaGetErrorString(e));
}
