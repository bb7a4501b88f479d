// pb_core.hpp -- object model, runtime and error conventions of the B200
// kernel library behind PHIST's phist_kernels C API.
//
// Layout decisions (all objects live on one GPU, one process per GPU):
//  * mvec  : row-major block vector, element (i,j) at d[i*lda + j] on the
//            device; a host mirror of the same shape is allocated lazily and
//            synchronised only by mvec_to_device / mvec_from_device /
//            mvec_get_data / mvec_set_data (phist_kernels_decl.h:201-246,
//            :286-299 define this contract for accelerator libraries).
//  * sdMat : column-major small dense matrix, element (i,j) at [i + j*lda],
//            kept coherent on host AND device after every call (GHOST's
//            default protocol: host compute + upload, src/kernels/ghost/
//            kernels_def.hpp:31-56).
//  * sparseMat : SELL-C-sigma (chunk height C, sorting window sigma) on the
//            device; block vectors stay in the original row order, the
//            sigma permutation is applied inside the kernels.
//
// Error convention: *iflag on exit, 0 ok, <0 error, codes of
// src/tools/phist_defs.h:53-71.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <atomic>
#include <map>
#include <mutex>
#include <stdexcept>
#include <string>
#include <vector>

namespace pb {

// ----------------------------------------------------------- error codes
enum : int {
  PB_SUCCESS = 0,
  PB_FUNCTIONAL_ERROR = -1,
  PB_MEM_ALLOC_FAILED = -44,
  PB_INVALID_INPUT = -55,
  PB_INTEGER_OVERFLOW = -66,
  PB_CAUGHT_EXCEPTION = -77,
  PB_BAD_CAST = -88,
  PB_NOT_IMPLEMENTED = -99,
};

// input flags (values of src/kernels/phist_kernel_flags.h)
enum : int {
  PB_ROBUST_REDUCTIONS = 1,
  PB_NO_GLOBAL_REDUCTION = 2,
  PB_SPARSEMAT_PERM_LOCAL = 1,
  PB_SPARSEMAT_PERM_GLOBAL = 2,
  PB_SPARSEMAT_DIST2_COLOR = 4,
  PB_SPARSEMAT_OPT_CARP = 32,
  PB_SPMVM_ONLY_LOCAL = 1024,
  PB_SDMAT_RUN_ON_HOST = 1024,
  PB_SDMAT_RUN_ON_DEVICE = 2048,
};

struct Error : std::runtime_error {
  int code;
  Error(int c, const std::string& m) : std::runtime_error(m), code(c) {}
};

void report(const char* fcn, const char* msg);
// looks up the allocation-free entry point's scratch address on the current
// device (pb_noalloc.cu); called once at library initialisation
void noalloc_setup_current_device();

#define PB_THROW(code, ...)                                     \
  do {                                                          \
    char pb_msg_[512];                                          \
    snprintf(pb_msg_, sizeof(pb_msg_), __VA_ARGS__);            \
    throw ::pb::Error((code), pb_msg_);                         \
  } while (0)

#define PB_REQUIRE(cond, code, ...) \
  do {                              \
    if (!(cond)) PB_THROW(code, __VA_ARGS__); \
  } while (0)

#define PB_CUDA(call)                                                        \
  do {                                                                       \
    cudaError_t e_ = (call);                                                 \
    if (e_ != cudaSuccess)                                                   \
      PB_THROW(e_ == cudaErrorMemoryAllocation ? ::pb::PB_MEM_ALLOC_FAILED   \
                                               : ::pb::PB_FUNCTIONAL_ERROR,  \
               "CUDA error %s at %s:%d", cudaGetErrorString(e_), __FILE__,   \
               __LINE__);                                                    \
  } while (0)

// Every extern "C" entry point wraps its body in PB_API_BEGIN/END: C++
// exceptions never cross the C ABI, they become iflag codes (the reference's
// PHIST_CHK_IERR converts exceptions to -77, src/tools/phist_macros.h:111-133).
//
// The input flag word is read once.  PHIST's flags all lie in [0, 2^14)
// (src/kernels/phist_kernel_flags.h: the largest is PHIST_SPMVM_TASK = 8192);
// callers that only want iflag as an output sometimes pass it uninitialised
// (test/kernels/TestWithType_def.h:155-162, SdMatEqual, passes a fresh `int iflag`
// to sdMat_extract_view), so a word outside that range reads as no flags.
inline int input_flags(int w) { return (w >= 0 && w < (1 << 14)) ? w : 0; }
#define PB_API_BEGIN(iflag)                          \
  int pb_iflag_in_ = ::pb::input_flags(*(iflag));    \
  (void)pb_iflag_in_;                                \
  *(iflag) = 0;                                      \
  try {
#define PB_API_END(iflag)                                   \
  }                                                         \
  catch (const ::pb::Error& e) {                            \
    ::pb::report(__func__, e.what());                       \
    *(iflag) = e.code;                                      \
  }                                                         \
  catch (const std::exception& e) {                         \
    ::pb::report(__func__, e.what());                       \
    *(iflag) = ::pb::PB_CAUGHT_EXCEPTION;                   \
  }

// ---------------------------------------------------------------- runtime
// Lanes: every host thread that calls the library gets its own lane -- a
// CUDA stream with its own reduction scratch, arrival counters, result
// mailbox and device-memory cache -- so independent solves driven from
// several host threads overlap on the GPU without sharing any mutable
// device state.  A thread's lane is created on its first call and returned
// to a pool (after its stream drained) when the thread exits.  Objects
// (mvecs, sdMats, matrices) are meant to be used by one thread; matrices
// that are only read may be shared.
//
// Device memory cache: blocks freed by objects are kept per rounded size in
// the freeing thread's lane and handed out again to that lane only.  Its
// kernels run in stream order on one stream, so a block freed after a kernel
// was enqueued may be reused by the next kernel without a sync.
struct Lane {
  cudaStream_t stream = nullptr;
  void* scratch = nullptr;
  size_t scratch_bytes = 0;
  unsigned int* counters = nullptr;  // 64 zero-initialised counters
  void* mbox_h = nullptr;            // pinned, device-mapped result mailbox
  void* mbox_d = nullptr;
  std::multimap<size_t, void*> free_blocks;  // guarded by the runtime mutex
  bool in_use = false;
  unsigned generation = 0;
};

class Runtime {
 public:
  static Runtime& get();
  void init();
  void finalize();
  bool initialized() const { return inited_; }
  cudaStream_t stream() { return lane().stream; }
  int device() const { return device_; }
  int num_sms() const { return num_sms_; }
  int64_t l2_bytes() const { return l2_bytes_; }

  // the calling thread's lane (created or taken from the pool on first use)
  Lane& lane();
  void release_lane(Lane* l, unsigned generation);
  int lanes_created() const { return (int)lanes_.size(); }

  void* dmalloc(size_t bytes);
  void dfree(void* p);
  void* hmalloc_pinned(size_t bytes);
  void hfree_pinned(void* p);
  void sync();  // drains the calling thread's lane

  // reusable device scratch for multi-block reductions: partial results per
  // block plus one arrival counter per launch (kept zero between launches)
  void* scratch(size_t bytes);
  unsigned int* counters();

  // Result mailbox (per lane): kMailboxBytes of pinned host memory mapped
  // into the device address space.  Calls that return values to the host
  // (dots, norms, Gram matrices) have their final kernel or copy write here
  // and read it after one stream synchronisation, with no pageable staging
  // copy.  One call at a time per lane.
  static constexpr size_t kMailboxBytes = 1u << 20;
  // results use the first kMailboxResultBytes; the last 64 bytes hold the
  // device error word (kernels with bounded waits store a code there, and
  // sync() reports and clears it)
  static constexpr size_t kMailboxResultBytes = kMailboxBytes - 64;
  void* mailbox_host() { return lane().mbox_h; }
  void* mailbox_dev() { return lane().mbox_d; }
  int* device_error_word() { return (int*)((char*)lane().mbox_d + kMailboxResultBytes); }

  // SELL parameters used for new matrices (C chunk height, sigma window)
  int sell_C = 32;
  int64_t sell_sigma_default = 256;  // when PERM_LOCAL is requested
  int verbose = 0;

  // SpMMV launch shape: threads per matrix row for block widths 1,2,4,8,16,32
  // and whether the fully unrolled short-row kernel may be used
  // (with 256-bit gathers, 4 threads per row at width 32: two 32-byte loads
  // per entry and thread, 8 rows of 128-byte segments per warp load, measured
  // 273 us against 299 us for 8 threads on the L=128 Anderson matrix)
  int spmv_tpr[6] = {1, 1, 1, 2, 4, 4};
  bool spmv_unroll = true;
  // block widths >= this use the shared-memory staged kernel (> 32: never).
  // Off by default: with one chunk per pipeline stage it measured slower
  // than the register kernel on the 3D Anderson matrix (nvec 8/16/32:
  // 219/436/1077 us against 152/285/545 us).
  int spmv_staged_min_nvec = 99;
  // SpMMV on matrices with rows of at most 8 entries: resident grid with the
  // next tile's entries prefetched into shared memory (pb_spmmv_pf.cuh);
  // false: one tile per block (pb_spmmv.cuh)
  bool spmv_pf = true;
  // the prefetching SpMMV kernel gathers X row segments of 32 bytes or more
  // with 256-bit loads (ld.global.v4.f64 / v8.f32) when X and Y rows start
  // on 32-byte boundaries: half the load instructions per gathered row, and
  // 12 / 17 / 21 % more bandwidth at widths 4 / 8 / 16 on the L=128 Anderson
  // matrix (bitwise the same results)
  bool spmv_v256 = true;
  // stage block-vector tiles of the Gram kernels with TMA (else cp.async)
  bool use_tma = true;
  // FP64 block products on the tensor cores (DMMA) for widths multiple of 8
  bool use_dmma = true;
  // batched CARP-CG replays its iteration as a CUDA graph (PHIST_B200_GRAPHS=0: plain launches)
  bool use_graphs = true;
  // CARP sweeps over a block colouring with the footprint of X staged in
  // shared memory (pb_carp_blocks.hpp); false: one launch per class of a
  // distance-2 row colouring.  Read when the CARP work is set up.
  bool carp_blocks = true;
  // row limit of a block (footprint limit twice that, pattern limit 16x);
  // 0: chosen from the sweep width the work is set up for (128 rows up to 8
  // columns, 64 beyond: the X footprint in shared memory grows with the
  // width)
  int carp_block_rows = 0;
  // block sweep launches with a programmatic dependency on the previous
  // launch (overlap of its segment copies with that launch's tail)
  bool carp_pdl = true;

  // statistics: kernel launches issued by this library (all lanes)
  std::atomic<uint64_t> launches{0};

 private:
  Runtime() = default;
  Lane* create_lane_locked();
  void free_lane_locked(Lane* l);
  bool inited_ = false;
  unsigned generation_ = 1;
  int device_ = 0;
  int num_sms_ = 148;
  int64_t l2_bytes_ = 126ll << 20;
  std::mutex mu_;
  std::vector<Lane*> lanes_;
  std::map<void*, size_t> live_blocks_;
};

inline Runtime& rt() { return Runtime::get(); }
inline cudaStream_t stream() { return rt().stream(); }

// check the last kernel launch
#define PB_LAUNCH_CHECK()                        \
  do {                                           \
    ::pb::rt().launches++;                       \
    PB_CUDA(cudaGetLastError());                 \
  } while (0)

// ---------------------------------------------------------------- objects
struct Comm {
  int rank = 0;
  int size = 1;
};

struct Map {
  const Comm* comm = nullptr;
  int64_t nglob = 0;
  int32_t nloc = 0;
  int64_t ilower = 0;
};

struct Context {
  const Map* row_map = nullptr;
  const Map* col_map = nullptr;
  const Map* range_map = nullptr;
  const Map* domain_map = nullptr;
  bool owns_maps = false;
};

template <class T>
struct Mvec {
  const Map* map = nullptr;
  int32_t nrows = 0;
  int nvec = 0;
  int64_t lda = 0;          // row stride of the underlying storage
  Mvec* root = nullptr;     // owning object (this if not a view)
  int col_off = 0;          // first column of this view inside root
  // owning object only:
  T* d_base = nullptr;
  T* h_base = nullptr;      // lazily allocated host mirror
  bool is_view() const { return root != this; }
  T* d() const { return root->d_base + col_off; }
  T* h();                   // allocates the root's host mirror on demand
};

template <class T>
struct SdMat {
  const Comm* comm = nullptr;
  int nrows = 0, ncols = 0;
  int64_t lda = 0;          // column stride
  SdMat* root = nullptr;
  int row_off = 0, col_off = 0;
  T* d_base = nullptr;
  T* h_base = nullptr;      // pinned host copy, always allocated
  bool is_view() const { return root != this; }
  T* d() const { return root->d_base + row_off + col_off * lda; }
  T* h() const { return root->h_base + row_off + col_off * lda; }
};

// SELL-C-sigma matrix resident in HBM.
//   chunk c covers SELL rows [c*C, c*C+C); entry k of SELL row r (r = c*C+l)
//   sits at val[chunk_ptr[c] + k*C + l]; padding has val=0, col=own row.
//   perm[r] = original row of SELL row r (nullptr when the identity).
template <class T>
struct SparseMat {
  const Comm* comm = nullptr;
  Map* row_map = nullptr;    // owned
  Map* dom_map = nullptr;    // owned (same as row_map when square)
  Context* ctx = nullptr;    // owned
  int64_t nrows = 0, ncols = 0, nnz = 0, nnz_padded = 0;
  int C = 32;
  int64_t sigma = 1;
  int64_t nchunks = 0;
  int max_row_len = 0;
  int64_t* d_chunk_ptr = nullptr;
  int32_t* d_chunk_len = nullptr;
  int32_t* d_col = nullptr;
  T* d_val = nullptr;
  int32_t* d_perm = nullptr;       // SELL row -> original row
  int32_t* d_iperm = nullptr;      // original row -> SELL row (nullptr: identity)
  int32_t* d_row_len = nullptr;    // per SELL row
  T* d_diag = nullptr;             // diagonal per original row (CARP)
  // host copy of the CRS structure (original order, for colouring/CARP)
  std::vector<int64_t> h_row_ptr;
  std::vector<int32_t> h_col;
  std::vector<T> h_val;
  std::vector<int32_t> h_perm;
  // SpMMV kernel variant per block-width class 1, 2, 4, 8, 16, 32, set by
  // the autotuner (pb_tune.cu); -1: the runtime default
  int tune_tpr[6] = {-1, -1, -1, -1, -1, -1};
  int tune_unroll[6] = {-1, -1, -1, -1, -1, -1};
  int tune_staged[6] = {-1, -1, -1, -1, -1, -1};
};

// ----------------------------------------------------------------- helpers
template <class T>
inline T* Mvec<T>::h()
{
  Mvec* r = root;
  if (!r->h_base) {
    size_t bytes = sizeof(T) * (size_t)r->lda * (size_t)(r->nrows > 0 ? r->nrows : 1);
    r->h_base = (T*)malloc(bytes);
    PB_REQUIRE(r->h_base, PB_MEM_ALLOC_FAILED, "host mirror allocation of %zu bytes failed", bytes);
    memset(r->h_base, 0, bytes);
  }
  return r->h_base + col_off;
}

inline int64_t ceil_div(int64_t a, int64_t b) { return (a + b - 1) / b; }

}  // namespace pb
