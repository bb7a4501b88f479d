// pb_api.cuh -- typed implementation of the phist_kernels C API
// (phist_kernels_decl.h, phist_kernels_common_decl.h,
// phist_kernels_fused_decl.h, phist_kernels_carp_decl.h).  Instantiated for
// double (phist_D*) in pb_api_D.cu and float (phist_S*) in pb_api_S.cu.
#pragma once
#include <cudaTypedefs.h>
#include <algorithm>
#include <atomic>
#include <type_traits>
#include <cmath>
#include <numeric>

#include "pb_blas.cuh"
#include "pb_block.cuh"
#include "pb_carp.cuh"
#include "pb_core.hpp"
#include "pb_spmmv.cuh"
#include "pb_spmmv_staged.cuh"
#include "pb_spmmv_pf.cuh"
#include "pb_prec.cuh"
#include "pb_tile.cuh"
#include "pb_dmma.cuh"

namespace pb {

// widths and leading dimensions in whole 16-byte vectors, 16-byte aligned start
template <class T>
inline bool vec_ok(const T* p, int64_t ld, int ncols)
{
  const int vw = 16 / (int)sizeof(T);
  return (((uintptr_t)p) & 15u) == 0 && ld % vw == 0 && ncols % vw == 0;
}

// raise a kernel's dynamic shared-memory limit once (the attribute call is a
// host round trip that would otherwise precede every launch)
template <class K>
inline void set_smem(K kern, size_t smem)
{
  static std::mutex mu;
  static std::map<const void*, size_t> done;
  std::lock_guard<std::mutex> g(mu);
  size_t& have = done[(const void*)kern];
  if (smem > have) {
    PB_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    have = smem;
  }
}

inline int grid_for(int64_t work, int bs = 256)
{
  int64_t g = ceil_div(work > 0 ? work : 1, bs);
  int64_t cap = (int64_t)rt().num_sms() * 16;
  return (int)(g < cap ? g : cap);
}

template <class T>
inline Mvec<T>* MV(const void* p)
{
  PB_REQUIRE(p, PB_BAD_CAST, "mvec handle is NULL");
  return (Mvec<T>*)p;
}
template <class T>
inline SdMat<T>* SD(const void* p)
{
  PB_REQUIRE(p, PB_BAD_CAST, "sdMat handle is NULL");
  return (SdMat<T>*)p;
}
template <class T>
inline SparseMat<T>* SP(const void* p)
{
  PB_REQUIRE(p, PB_BAD_CAST, "sparseMat handle is NULL");
  return (SparseMat<T>*)p;
}

inline void ensure_init()
{
  if (!rt().initialized()) rt().init();
}

// ======================================================================
// mvec object model
// ======================================================================
template <class T>
void mvec_create(void** V, const void* vmap, int nvec, int flags)
{
  (void)flags;
  ensure_init();
  PB_REQUIRE(V && vmap, PB_BAD_CAST, "NULL argument");
  PB_REQUIRE(nvec >= 1, PB_INVALID_INPUT, "nvec must be >= 1, got %d", nvec);
  const Map* map = (const Map*)vmap;
  Mvec<T>* v = new Mvec<T>();
  v->map = map;
  v->nrows = map->nloc;
  v->nvec = nvec;
  v->lda = nvec;
  v->root = v;
  v->col_off = 0;
  size_t bytes = sizeof(T) * (size_t)nvec * (size_t)(map->nloc > 0 ? map->nloc : 1);
  try {
    v->d_base = (T*)rt().dmalloc(bytes);
  } catch (...) {
    delete v;
    throw;
  }
  // new objects are zero, as the builtin allocation touches them with zeros
  PB_CUDA(cudaMemsetAsync(v->d_base, 0, bytes, stream()));
  *V = v;
}

template <class T>
void mvec_delete(void* vV)
{
  if (!vV) return;
  Mvec<T>* v = (Mvec<T>*)vV;
  if (!v->is_view()) {
    rt().dfree(v->d_base);
    free(v->h_base);
  }
  delete v;
}

template <class T>
void mvec_view_block(void* vV, void** vblock, int jmin, int jmax)
{
  Mvec<T>* V = MV<T>(vV);
  PB_REQUIRE(vblock, PB_BAD_CAST, "Vblock is NULL");
  PB_REQUIRE(jmin >= 0 && jmax < V->nvec && jmin <= jmax, PB_INVALID_INPUT,
             "view columns %d:%d out of range for %d columns", jmin, jmax, V->nvec);
  Mvec<T>* b = (Mvec<T>*)*vblock;
  if (b && !b->is_view()) {
    mvec_delete<T>(b);
    b = nullptr;
  }
  if (!b) b = new Mvec<T>();
  b->map = V->map;
  b->nrows = V->nrows;
  b->nvec = jmax - jmin + 1;
  b->lda = V->lda;
  b->root = V->root;
  b->col_off = V->col_off + jmin;
  b->d_base = nullptr;
  b->h_base = nullptr;
  *vblock = b;
}

template <class T>
void copy_cols(const Mvec<T>* X, int xoff, Mvec<T>* Y, int yoff, int ncols)
{
  if (X->nrows == 0 || ncols == 0) return;
  k_copy<T, T><<<grid_for((int64_t)X->nrows * ncols), 256, 0, stream()>>>(
      X->d() + xoff, X->lda, Y->d() + yoff, Y->lda, X->nrows, ncols);
  PB_LAUNCH_CHECK();
}

// V(:,j) *= s[j] with the host coefficients passed by value (64 columns per launch)
template <class T>
void vscale_cols(Mvec<T>* V, const T* s)
{
  if (V->nrows == 0) return;
  for (int c0 = 0; c0 < V->nvec; c0 += 64) {
    const int nv = std::min(64, V->nvec - c0);
    Coef64<T> c;
    for (int j = 0; j < nv; j++) c.v[j] = s[c0 + j];
    k_vscale_v<T><<<grid_for((int64_t)V->nrows * nv), 256, 0, stream()>>>(V->d() + c0, V->lda, V->nrows, nv, c);
    PB_LAUNCH_CHECK();
  }
}

// Y(:,j) = alpha[j] X(:,j) + beta Y(:,j), coefficients passed by value
template <class T>
void vadd_cols(const T* alpha, const Mvec<T>* X, T beta, Mvec<T>* Y)
{
  if (Y->nrows == 0) return;
  for (int c0 = 0; c0 < Y->nvec; c0 += 64) {
    const int nv = std::min(64, Y->nvec - c0);
    Coef64<T> c;
    for (int j = 0; j < nv; j++) c.v[j] = alpha[c0 + j];
    k_axpby_v<T><<<grid_for((int64_t)Y->nrows * nv), 256, 0, stream()>>>(X->d() + c0, X->lda, Y->d() + c0, Y->lda, Y->nrows, nv, c, beta);
    PB_LAUNCH_CHECK();
  }
}

template <class T>
void check_same_rows(const Mvec<T>* a, const Mvec<T>* b)
{
  PB_REQUIRE(a->nrows == b->nrows, PB_INVALID_INPUT, "mvecs have %d and %d rows", a->nrows,
             b->nrows);
}

// host mirror <-> device for the columns of a view
template <class T>
void mvec_upload(Mvec<T>* V)
{
  if (V->nrows == 0) return;
  T* h = V->h();
  // the host mirror is pageable: staged before the call returns (see sd_upload)
  if (V->nvec == V->lda)
    PB_CUDA(cudaMemcpyAsync(V->d(), h, sizeof(T) * (size_t)V->nrows * V->lda, cudaMemcpyHostToDevice, stream()));
  else
    PB_CUDA(cudaMemcpy2DAsync(V->d(), V->lda * sizeof(T), h, V->lda * sizeof(T),
                              V->nvec * sizeof(T), V->nrows, cudaMemcpyHostToDevice, stream()));
}
template <class T>
void mvec_download(Mvec<T>* V)
{
  if (V->nrows == 0) return;
  T* h = V->h();
  if (V->nvec == V->lda)
    PB_CUDA(cudaMemcpyAsync(h, V->d(), sizeof(T) * (size_t)V->nrows * V->lda, cudaMemcpyDeviceToHost, stream()));
  else
    PB_CUDA(cudaMemcpy2DAsync(h, V->lda * sizeof(T), V->d(), V->lda * sizeof(T),
                              V->nvec * sizeof(T), V->nrows, cudaMemcpyDeviceToHost, stream()));
  rt().sync();
}

template <class T>
void mvec_get_data(const void* vV, T* data, int32_t lda, int row_major)
{
  Mvec<T>* V = MV<T>(vV);
  PB_REQUIRE(data || V->nrows == 0, PB_BAD_CAST, "data is NULL");
  if (V->nrows == 0) return;
  if (row_major) {
    PB_REQUIRE(lda >= V->nvec, PB_INVALID_INPUT, "lda %d < nvec %d", lda, V->nvec);
    if (lda == V->nvec && V->lda == V->nvec) {
      // both sides contiguous: one linear copy (a 2D copy of n rows of a few
      // bytes each runs far below the link rate)
      PB_CUDA(cudaMemcpyAsync(data, V->d(), sizeof(T) * (size_t)V->nrows * V->nvec, cudaMemcpyDeviceToHost,
                              stream()));
    } else {
      PB_CUDA(cudaMemcpy2DAsync(data, (size_t)lda * sizeof(T), V->d(), V->lda * sizeof(T),
                                V->nvec * sizeof(T), V->nrows, cudaMemcpyDeviceToHost, stream()));
    }
    rt().sync();
  } else {
    PB_REQUIRE(lda >= V->nrows, PB_INVALID_INPUT, "lda %d < nrows %d", lda, V->nrows);
    // transpose on the device into scratch, then one 2D copy
    T* tmp = (T*)rt().scratch(sizeof(T) * (size_t)V->nrows * V->nvec);
    k_sd_copy<T><<<grid_for((int64_t)V->nrows * V->nvec), 256, 0, stream()>>>(
        V->d(), V->lda, tmp, V->nrows, V->nrows, V->nvec, 1);
    PB_LAUNCH_CHECK();
    PB_CUDA(cudaMemcpy2DAsync(data, (size_t)lda * sizeof(T), tmp, V->nrows * sizeof(T),
                              V->nrows * sizeof(T), V->nvec, cudaMemcpyDeviceToHost, stream()));
    rt().sync();
  }
}

template <class T>
void mvec_set_data(void* vV, const T* data, int32_t lda, int row_major)
{
  Mvec<T>* V = MV<T>(vV);
  PB_REQUIRE(data || V->nrows == 0, PB_BAD_CAST, "data is NULL");
  if (V->nrows == 0) return;
  if (row_major) {
    PB_REQUIRE(lda >= V->nvec, PB_INVALID_INPUT, "lda %d < nvec %d", lda, V->nvec);
    if (lda == V->nvec && V->lda == V->nvec) {
      PB_CUDA(cudaMemcpyAsync(V->d(), data, sizeof(T) * (size_t)V->nrows * V->nvec, cudaMemcpyHostToDevice,
                              stream()));
    } else {
      PB_CUDA(cudaMemcpy2DAsync(V->d(), V->lda * sizeof(T), data, (size_t)lda * sizeof(T),
                                V->nvec * sizeof(T), V->nrows, cudaMemcpyHostToDevice, stream()));
    }
    rt().sync();
  } else {
    PB_REQUIRE(lda >= V->nrows, PB_INVALID_INPUT, "lda %d < nrows %d", lda, V->nrows);
    T* tmp = (T*)rt().scratch(sizeof(T) * (size_t)V->nrows * V->nvec);
    PB_CUDA(cudaMemcpy2DAsync(tmp, V->nrows * sizeof(T), data, (size_t)lda * sizeof(T),
                              V->nrows * sizeof(T), V->nvec, cudaMemcpyHostToDevice, stream()));
    k_sd_copy<T><<<grid_for((int64_t)V->nrows * V->nvec), 256, 0, stream()>>>(
        tmp, V->nrows, V->d(), V->lda, V->nvec, V->nrows, 1);
    PB_LAUNCH_CHECK();
    rt().sync();
  }
}

// ======================================================================
// sdMat object model
// ======================================================================
template <class T>
void sdmat_create(void** M, int nrows, int ncols, const void* comm)
{
  ensure_init();
  PB_REQUIRE(M, PB_BAD_CAST, "M is NULL");
  PB_REQUIRE(nrows >= 0 && ncols >= 0, PB_INVALID_INPUT, "negative sdMat size");
  SdMat<T>* s = new SdMat<T>();
  s->comm = (const Comm*)comm;
  s->nrows = nrows;
  s->ncols = ncols;
  s->lda = nrows > 0 ? nrows : 1;
  s->root = s;
  size_t bytes = sizeof(T) * (size_t)s->lda * (size_t)(ncols > 0 ? ncols : 1);
  s->d_base = (T*)rt().dmalloc(bytes);
  s->h_base = (T*)calloc(1, bytes);
  PB_REQUIRE(s->h_base, PB_MEM_ALLOC_FAILED, "sdMat host allocation failed");
  PB_CUDA(cudaMemsetAsync(s->d_base, 0, bytes, stream()));
  *M = s;
}

template <class T>
void sdmat_delete(void* vM)
{
  if (!vM) return;
  SdMat<T>* s = (SdMat<T>*)vM;
  if (!s->is_view()) {
    rt().dfree(s->d_base);
    free(s->h_base);
  }
  delete s;
}

// The host copy of an sdMat is pageable memory: cudaMemcpy*Async stages it
// before returning, so the host copy may change right after this call and no
// stream drain is needed (the device copy is updated in stream order).
template <class T>
void sd_upload(SdMat<T>* M)
{
  if (M->nrows == 0 || M->ncols == 0) return;
  PB_CUDA(cudaMemcpy2DAsync(M->d(), M->lda * sizeof(T), M->h(), M->lda * sizeof(T),
                            M->nrows * sizeof(T), M->ncols, cudaMemcpyHostToDevice, stream()));
}
// Device -> host copy of an sdMat.  Small matrices (all the solvers' Gram and
// projection matrices) go through the pinned mailbox: one asynchronous DMA,
// one stream synchronisation and a host copy, instead of a pageable transfer.
template <class T>
void sd_download(SdMat<T>* M)
{
  if (M->nrows == 0 || M->ncols == 0) return;
  const size_t col = sizeof(T) * (size_t)M->nrows;
  if (col * (size_t)M->ncols <= Runtime::kMailboxResultBytes) {
    char* hb = (char*)rt().mailbox_host();
    PB_CUDA(cudaMemcpy2DAsync(hb, col, M->d(), M->lda * sizeof(T), col, M->ncols, cudaMemcpyDeviceToHost,
                              stream()));
    rt().sync();
    for (int j = 0; j < M->ncols; j++) memcpy(M->h() + (int64_t)j * M->lda, hb + col * j, col);
    return;
  }
  PB_CUDA(cudaMemcpy2DAsync(M->h(), M->lda * sizeof(T), M->d(), M->lda * sizeof(T),
                            M->nrows * sizeof(T), M->ncols, cudaMemcpyDeviceToHost, stream()));
  rt().sync();
}

// after a host-side sdMat operation: upload unless RUN_ON_HOST only
inline bool sd_host_only(int flags)
{
  return (flags & (PB_SDMAT_RUN_ON_HOST | PB_SDMAT_RUN_ON_DEVICE)) == PB_SDMAT_RUN_ON_HOST;
}
// after a device-side sdMat result: download unless RUN_ON_DEVICE only
inline bool sd_device_only(int flags)
{
  return (flags & (PB_SDMAT_RUN_ON_HOST | PB_SDMAT_RUN_ON_DEVICE)) == PB_SDMAT_RUN_ON_DEVICE;
}

template <class T>
inline T& sdh(SdMat<T>* M, int i, int j)
{
  return M->h()[i + (int64_t)j * M->lda];
}

template <class T>
void sdmat_view_block(void* vM, void** vblock, int imin, int imax, int jmin, int jmax)
{
  SdMat<T>* M = SD<T>(vM);
  PB_REQUIRE(vblock, PB_BAD_CAST, "Mblock is NULL");
  PB_REQUIRE(imin >= 0 && imax < M->nrows && jmin >= 0 && jmax < M->ncols && imin <= imax + 1 &&
                 jmin <= jmax + 1,
             PB_INVALID_INPUT, "sdMat view (%d:%d,%d:%d) out of range %dx%d", imin, imax, jmin,
             jmax, M->nrows, M->ncols);
  SdMat<T>* b = (SdMat<T>*)*vblock;
  if (b && !b->is_view()) {
    sdmat_delete<T>(b);
    b = nullptr;
  }
  if (!b) b = new SdMat<T>();
  b->comm = M->comm;
  b->nrows = imax - imin + 1;
  b->ncols = jmax - jmin + 1;
  b->lda = M->lda;
  b->root = M->root;
  b->row_off = M->row_off + imin;
  b->col_off = M->col_off + jmin;
  *vblock = b;
}

// ======================================================================
// sparse matrix construction (host CRS -> SELL-C-sigma in HBM)
// ======================================================================
template <class T>
void sell_free(SparseMat<T>* A)
{
  rt().dfree(A->d_chunk_ptr);
  rt().dfree(A->d_chunk_len);
  rt().dfree(A->d_col);
  rt().dfree(A->d_val);
  rt().dfree(A->d_perm);
  rt().dfree(A->d_iperm);
  rt().dfree(A->d_row_len);
  rt().dfree(A->d_diag);
}

template <class T>
void* upload_vec(const std::vector<T>& v)
{
  if (v.empty()) return nullptr;
  void* d = rt().dmalloc(v.size() * sizeof(T));
  PB_CUDA(cudaMemcpyAsync(d, v.data(), v.size() * sizeof(T), cudaMemcpyHostToDevice, stream()));
  return d;
}

// SELL-C-sigma layout of the CRS rows (columns sorted inside each row):
// rows stably sorted by descending length inside windows of sigma rows,
// chunks of C rows padded to the chunk's longest row, entry k of chunk row l
// at chunk_ptr + k*C + l.  Replaces any layout A had; the result of every
// SpMMV is the same in every layout (each row sums its entries in column
// order).
template <class T>
void sell_layout(SparseMat<T>* A, const std::vector<int64_t>& rp, const std::vector<int32_t>& col,
                 const std::vector<T>& val, int C, int64_t sigma)
{
  PB_REQUIRE(C >= 1 && C <= 1024, PB_INVALID_INPUT, "SELL chunk height %d out of range", C);
  const int64_t nrows = A->nrows;
  if (sigma < 1) sigma = 1;
  rt().sync();  // the old layout may still be read by enqueued kernels
  rt().dfree(A->d_chunk_ptr);
  rt().dfree(A->d_chunk_len);
  rt().dfree(A->d_col);
  rt().dfree(A->d_val);
  rt().dfree(A->d_perm);
  rt().dfree(A->d_iperm);
  rt().dfree(A->d_row_len);
  A->d_iperm = nullptr;
  A->d_chunk_ptr = nullptr;
  A->d_chunk_len = nullptr;
  A->d_col = nullptr;
  A->d_val = nullptr;
  A->d_perm = nullptr;
  A->d_row_len = nullptr;
  A->C = C;
  A->sigma = sigma;

  // sigma permutation: stable descending row length inside windows
  std::vector<int32_t> perm(nrows);
  std::iota(perm.begin(), perm.end(), 0);
  if (sigma > 1) {
    for (int64_t w0 = 0; w0 < nrows; w0 += sigma) {
      const int64_t w1 = std::min(nrows, w0 + sigma);
      std::stable_sort(perm.begin() + w0, perm.begin() + w1, [&](int32_t a, int32_t b) {
        return (rp[a + 1] - rp[a]) > (rp[b + 1] - rp[b]);
      });
    }
  }
  bool ident = true;
  for (int64_t r = 0; r < nrows; r++)
    if (perm[r] != r) { ident = false; break; }

  A->nchunks = ceil_div(nrows, C);
  std::vector<int32_t> clen(A->nchunks, 0);
  std::vector<int64_t> cptr(A->nchunks + 1, 0);
  std::vector<int32_t> rlen(A->nchunks * C, 0);
  int maxlen = 0;
  for (int64_t r = 0; r < nrows; r++) {
    const int len = (int)(rp[perm[r] + 1] - rp[perm[r]]);
    rlen[r] = len;
    clen[r / C] = std::max(clen[r / C], len);
    maxlen = std::max(maxlen, len);
  }
  for (int64_t c = 0; c < A->nchunks; c++) cptr[c + 1] = cptr[c] + (int64_t)clen[c] * C;
  A->nnz_padded = cptr[A->nchunks];
  A->max_row_len = maxlen;
  std::vector<int32_t> scol(A->nnz_padded > 0 ? A->nnz_padded : 1, 0);
  std::vector<T> sval(A->nnz_padded > 0 ? A->nnz_padded : 1, T(0));
  for (int64_t r = 0; r < A->nchunks * C; r++) {
    const int64_t ch = r / C, l = r - ch * C;
    const int64_t base = cptr[ch] + l;
    if (r < nrows) {
      const int64_t i = perm[r];
      const int64_t p0 = rp[i];
      const int len = rlen[r];
      const int32_t padc = len > 0 ? col[p0] : 0;
      for (int k = 0; k < clen[ch]; k++) {
        if (k < len) {
          scol[base + (int64_t)k * C] = col[p0 + k];
          sval[base + (int64_t)k * C] = val[p0 + k];
        } else {
          scol[base + (int64_t)k * C] = padc;
        }
      }
    }
  }
  A->d_chunk_ptr = (int64_t*)upload_vec(cptr);
  A->d_chunk_len = (int32_t*)upload_vec(clen);
  A->d_col = (int32_t*)upload_vec(scol);
  A->d_val = (T*)upload_vec(sval);
  A->d_perm = ident ? nullptr : (int32_t*)upload_vec(perm);
  if (!ident) {
    std::vector<int32_t> iperm(nrows);
    for (int64_t r = 0; r < nrows; r++) iperm[perm[r]] = (int32_t)r;
    A->d_iperm = (int32_t*)upload_vec(iperm);
  }
  A->d_row_len = (int32_t*)upload_vec(rlen);
  A->h_perm = std::move(perm);
  rt().sync();
}

// rows stably sorted by column inside each row (the builtin's
// sort_global_cols, crsmat_module.F90:484-516), then laid out as SELL-C-sigma
template <class T>
SparseMat<T>* build_sparse(const Comm* comm, int64_t nrows, int64_t ncols,
                           std::vector<int64_t>&& rp, std::vector<int32_t>&& col,
                           std::vector<T>&& val, int flags)
{
  ensure_init();
  PB_REQUIRE(nrows >= 0 && nrows < (int64_t(1) << 31) && ncols >= 0 && ncols < (int64_t(1) << 31),
             PB_INTEGER_OVERFLOW, "matrix dimensions %lld x %lld exceed 32-bit local indices",
             (long long)nrows, (long long)ncols);
  const int64_t nnz = rp[nrows];
  // sort columns inside rows (stable)
  {
    std::vector<int64_t> idx;
    std::vector<int32_t> c2;
    std::vector<T> v2;
    for (int64_t i = 0; i < nrows; i++) {
      const int64_t p0 = rp[i], p1 = rp[i + 1], len = p1 - p0;
      bool sorted = true;
      for (int64_t p = p0 + 1; p < p1; p++)
        if (col[p] < col[p - 1]) { sorted = false; break; }
      if (sorted) continue;
      idx.resize(len);
      std::iota(idx.begin(), idx.end(), p0);
      std::stable_sort(idx.begin(), idx.end(), [&](int64_t a, int64_t b) { return col[a] < col[b]; });
      c2.resize(len);
      v2.resize(len);
      for (int64_t q = 0; q < len; q++) { c2[q] = col[idx[q]]; v2[q] = val[idx[q]]; }
      for (int64_t q = 0; q < len; q++) { col[p0 + q] = c2[q]; val[p0 + q] = v2[q]; }
    }
  }
  for (int64_t p = 0; p < nnz; p++)
    PB_REQUIRE(col[p] >= 0 && col[p] < ncols, PB_INVALID_INPUT,
               "column index %d out of range [0,%lld)", col[p], (long long)ncols);

  SparseMat<T>* A = new SparseMat<T>();
  A->comm = comm;
  A->nrows = nrows;
  A->ncols = ncols;
  A->nnz = nnz;
  const int64_t sigma = (flags & (PB_SPARSEMAT_PERM_LOCAL | PB_SPARSEMAT_PERM_GLOBAL)) ? rt().sell_sigma_default : 1;
  sell_layout(A, rp, col, val, rt().sell_C, sigma);
  {
    std::vector<T> diag(nrows, T(0));
    for (int64_t i = 0; i < nrows; i++)
      for (int64_t p = rp[i]; p < rp[i + 1]; p++)
        if (col[p] == i) diag[i] = val[p];
    A->d_diag = (T*)upload_vec(diag);
  }
  rt().sync();

  A->row_map = new Map();
  A->row_map->comm = comm;
  A->row_map->nglob = nrows;
  A->row_map->nloc = (int32_t)nrows;
  if (ncols == nrows) {
    A->dom_map = A->row_map;
  } else {
    A->dom_map = new Map();
    A->dom_map->comm = comm;
    A->dom_map->nglob = ncols;
    A->dom_map->nloc = (int32_t)ncols;
  }
  A->ctx = new Context();
  A->ctx->row_map = A->row_map;
  A->ctx->col_map = A->dom_map;
  A->ctx->range_map = A->row_map;
  A->ctx->domain_map = A->dom_map;
  A->h_row_ptr = std::move(rp);
  A->h_col = std::move(col);
  A->h_val = std::move(val);
  // the uploads ran on the creating thread's lane: drain it, so that the
  // (read-only) matrix can be used from any thread's lane right away
  rt().sync();
  return A;
}

template <class T>
void sparse_delete(void* vA)
{
  if (!vA) return;
  SparseMat<T>* A = (SparseMat<T>*)vA;
  sell_free(A);
  if (A->dom_map != A->row_map) delete A->dom_map;
  delete A->row_map;
  delete A->ctx;
  delete A;
}

typedef int (*RowFunc)(int64_t, int32_t*, int64_t*, void*, void*);
typedef int (*RowFuncCtor)(void*, void**);

template <class T>
void create_from_rowfunc(void** vA, const void* comm, int64_t nrows, int64_t ncols, int32_t maxnne,
                         RowFunc f, RowFuncCtor ctor, void* arg, int flags)
{
  PB_REQUIRE(vA && f, PB_BAD_CAST, "NULL argument");  // comm NULL: the single process
  PB_REQUIRE(maxnne >= 0, PB_INVALID_INPUT, "maxnne < 0");
  std::vector<int64_t> rp(nrows + 1, 0);
  std::vector<int32_t> col;
  std::vector<T> val;
  col.reserve((size_t)nrows * (maxnne > 0 ? maxnne : 1));
  val.reserve((size_t)nrows * (maxnne > 0 ? maxnne : 1));
  std::vector<int64_t> cbuf(maxnne > 0 ? maxnne : 1);
  std::vector<T> vbuf(maxnne > 0 ? maxnne : 1);
  void* work = arg;
  if (ctor) {
    work = nullptr;
    PB_REQUIRE(ctor(arg, &work) == 0, PB_FUNCTIONAL_ERROR, "row function constructor failed");
  }
  for (int64_t i = 0; i < nrows; i++) {
    int32_t len = 0;
    int err = f(i, &len, cbuf.data(), vbuf.data(), work);
    PB_REQUIRE(err == 0, PB_FUNCTIONAL_ERROR, "row function returned %d for row %lld", err,
               (long long)i);
    PB_REQUIRE(len >= 0 && len <= maxnne, PB_INVALID_INPUT, "row %lld has %d > maxnne=%d entries",
               (long long)i, len, maxnne);
    for (int q = 0; q < len; q++) {
      col.push_back((int32_t)cbuf[q]);
      val.push_back(vbuf[q]);
    }
    rp[i + 1] = (int64_t)col.size();
  }
  if (ctor) ctor(arg, &work);
  *vA = build_sparse<T>((const Comm*)comm, nrows, ncols, std::move(rp), std::move(col),
                        std::move(val), flags);
}

template <class T>
void read_mm(void** vA, const void* comm, const char* fn, int flags)
{
  PB_REQUIRE(vA && fn, PB_BAD_CAST, "NULL argument");
  FILE* f = fopen(fn, "r");
  PB_REQUIRE(f, PB_INVALID_INPUT, "cannot open %s", fn);
  char line[1024];
  bool symmetric = false, skew = false, pattern = false;
  if (!fgets(line, sizeof line, f)) { fclose(f); PB_THROW(PB_INVALID_INPUT, "empty file %s", fn); }
  std::string hdr(line);
  for (auto& ch : hdr) ch = (char)tolower(ch);
  if (hdr.find("complex") != std::string::npos) { fclose(f); PB_THROW(PB_NOT_IMPLEMENTED, "complex MatrixMarket not supported"); }
  symmetric = hdr.find("symmetric") != std::string::npos && hdr.find("skew") == std::string::npos;
  skew = hdr.find("skew-symmetric") != std::string::npos;
  pattern = hdr.find("pattern") != std::string::npos;
  do {
    if (!fgets(line, sizeof line, f)) { fclose(f); PB_THROW(PB_INVALID_INPUT, "truncated %s", fn); }
  } while (line[0] == '%');
  long long nr, nc, nz;
  PB_REQUIRE(sscanf(line, "%lld %lld %lld", &nr, &nc, &nz) == 3, PB_INVALID_INPUT, "bad size line");
  std::vector<int64_t> ri, ci;
  std::vector<T> vv;
  for (long long q = 0; q < nz; q++) {
    long long i, j;
    double v = 1.0;
    if (!fgets(line, sizeof line, f)) break;
    int got = pattern ? sscanf(line, "%lld %lld", &i, &j) : sscanf(line, "%lld %lld %lf", &i, &j, &v);
    if (got < 2) { q--; continue; }
    ri.push_back(i - 1); ci.push_back(j - 1); vv.push_back(T(v));
    if ((symmetric || skew) && i != j) {
      ri.push_back(j - 1); ci.push_back(i - 1); vv.push_back(T(skew ? -v : v));
    }
  }
  fclose(f);
  std::vector<int64_t> rp(nr + 1, 0);
  for (auto r : ri) rp[r + 1]++;
  for (long long r = 0; r < nr; r++) rp[r + 1] += rp[r];
  std::vector<int32_t> col(ri.size());
  std::vector<T> val(ri.size());
  std::vector<int64_t> fill(rp.begin(), rp.end() - 1);
  for (size_t q = 0; q < ri.size(); q++) {  // file order kept inside a row
    const int64_t p = fill[ri[q]]++;
    col[p] = (int32_t)ci[q];
    val[p] = vv[q];
  }
  *vA = build_sparse<T>((const Comm*)comm, nr, nc, std::move(rp), std::move(col), std::move(val), flags);
}

// ======================================================================
// SpMMV launches
// ======================================================================
template <class T>
SellDev<T> sell_dev(const SparseMat<T>* A)
{
  SellDev<T> s;
  s.nrows = A->nrows;
  s.nchunks = A->nchunks;
  s.C = A->C;
  s.chunk_ptr = A->d_chunk_ptr;
  s.chunk_len = A->d_chunk_len;
  s.col = A->d_col;
  s.val = A->d_val;
  s.perm = A->d_perm;
  return s;
}

struct SpmvOut {
  bool wdw = false, vdw = false;
};

// one instantiation family per (block width NV, threads per row TPR): the
// fully unrolled short-row kernel when the matrix has C=32 chunks of at most
// 8 entries, the general kernel otherwise
template <class T, int NV, int TPR>
void launch_spmv_nv(const SparseMat<T>* A, const SellDev<T>& S, SpmvArgs<T>& p, bool vec)
{
  constexpr int RPB = SPMV_BS / TPR;
  const int64_t npad = A->nchunks * (int64_t)A->C;
  int grid = (int)ceil_div(npad > 0 ? npad : 1, RPB);
  if (p.want_wdw || p.want_vdw) {
    // fused dots: a bounded grid walks the row tiles, so few partial vectors
    grid = std::min(grid, rt().num_sms() * 8);
    p.part = (T*)rt().scratch(sizeof(T) * (size_t)grid * 2 * NV);
    p.counter = rt().counters();
  }
  constexpr int LG = NV == 1 ? 0 : NV == 2 ? 1 : NV == 4 ? 2 : NV == 8 ? 3 : NV == 16 ? 4 : 5;
  const bool unroll = A->tune_unroll[LG] >= 0 ? A->tune_unroll[LG] != 0 : rt().spmv_unroll;
  const bool fast = unroll && A->C == 32 && A->max_row_len <= 8;
  const bool dots = p.want_wdw || p.want_vdw;
  if constexpr (NV >= 8 && NV <= 32) {
    // wide block vectors: X rows staged in shared memory by cp.async
    const bool staged = A->tune_staged[LG] >= 0 ? A->tune_staged[LG] != 0 : NV >= rt().spmv_staged_min_nvec;
    if (fast && vec && !dots && !p.u && staged) {
      const size_t smem = StagedSmem<T, NV>::bytes;
      const int bps = std::max(1, std::min(8, (int)((200 * 1024) / smem)));
      const int sgrid = (int)std::min<int64_t>(A->nchunks > 0 ? A->nchunks : 1, (int64_t)rt().num_sms() * bps);
      auto kern = k_sell_spmmv_staged<T, NV>;
      set_smem(kern, smem);
      kern<<<sgrid, 256, smem, stream()>>>(S, p);
      PB_LAUNCH_CHECK();
      return;
    }
  }
  if (fast && !dots && !p.u && rt().spmv_pf && (vec || (NV == 1 && p.nvec == 1))) {
    // resident grid, next tile's entries prefetched into shared memory
    constexpr int NT = TPR == 1 ? 128 : (TPR == 16 ? 512 : 256);
    constexpr int RPBp = NT / TPR;
    // resident blocks per SM of each form, taken once
    auto resident = [](auto kern, std::atomic<int>& occ) {
      if (occ.load() == 0) {
        int o = 0;
        PB_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&o, kern, NT, 0));
        occ.store(std::max(1, o));
      }
      return occ.load();
    };
    const int64_t ntiles = ceil_div(A->nchunks, RPBp / 32);
    // 32-byte row segments: at least 32 bytes per thread, rows on 32-byte
    // boundaries (vec already holds for 16 bytes)
    constexpr int V32 = 32 / (int)sizeof(T);
    const bool v256 = (NV / TPR) * (int)sizeof(T) >= 32 && vec && rt().spmv_v256 &&
                      ((uintptr_t)(p.x + p.col0) & 31u) == 0 && ((uintptr_t)(p.y + p.col0) & 31u) == 0 &&
                      p.ldx % V32 == 0 && p.ldy % V32 == 0;
    if constexpr ((NV / TPR) * sizeof(T) >= 32) {
      if (v256) {
        static std::atomic<int> occ32{0};
        auto kern = pf_kernel<T, NV, TPR, NT, false, 32>();
        const int pgrid = (int)std::max<int64_t>(1, std::min<int64_t>(ntiles, (int64_t)rt().num_sms() * resident(kern, occ32)));
        kern<<<pgrid, NT, 0, stream()>>>(S, p);
        PB_LAUNCH_CHECK();
        return;
      }
    }
    static std::atomic<int> occ{0};
    auto kern = pf_kernel<T, NV, TPR, NT>();
    const int pgrid = (int)std::max<int64_t>(1, std::min<int64_t>(ntiles, (int64_t)rt().num_sms() * resident(kern, occ)));
    kern<<<pgrid, NT, 0, stream()>>>(S, p);
    PB_LAUNCH_CHECK();
    return;
  }
#define PB_SPMV(VECv, KMAXv, CCv)                                                         \
  if (dots)                                                                             \
    k_sell_spmmv<T, NV, TPR, VECv, KMAXv, CCv, true><<<grid, SPMV_BS, 0, stream()>>>(S, p); \
  else                                                                                  \
    k_sell_spmmv<T, NV, TPR, VECv, KMAXv, CCv, false><<<grid, SPMV_BS, 0, stream()>>>(S, p);
  if (fast) {
    if (vec) { PB_SPMV(true, 8, 32) } else { PB_SPMV(false, 8, 32) }
  } else {
    if (vec) { PB_SPMV(true, 0, 0) } else { PB_SPMV(false, 0, 0) }
  }
#undef PB_SPMV
  PB_LAUNCH_CHECK();
}

template <class T>
bool aligned16(const void* p)
{
  return ((uintptr_t)p & 15u) == 0;
}

// Y(:,col0:col0+nv) = alpha*(A+diag(sh))X + beta*Y, nv <= 32, epilogues on
template <class T>
void spmv_tile(const SparseMat<T>* A, SpmvArgs<T>& p, int nv)
{
  const SellDev<T> S = sell_dev(A);
  p.nvec = nv;
  const int NV = nv <= 1 ? 1 : nv <= 2 ? 2 : nv <= 4 ? 4 : nv <= 8 ? 8 : nv <= 16 ? 16 : 32;
  const int lg = NV == 1 ? 0 : NV == 2 ? 1 : NV == 4 ? 2 : NV == 8 ? 3 : NV == 16 ? 4 : 5;
  // vector path: the tile width is exactly NV and every row segment that a
  // thread touches starts on a 16-byte boundary
  const int vw = 16 / (int)sizeof(T);
  bool vec = (nv == NV) && NV >= 2;
  if (vec) {
    vec = aligned16<T>(p.x + p.col0) && aligned16<T>(p.y + p.col0) && (p.ldx % vw == 0) &&
          (p.ldy % vw == 0) && (!p.u || (aligned16<T>(p.u + p.col0) && p.ldu % vw == 0));
    if (sizeof(T) == 4 && NV == 2) vec = false;
  }
  const int tpr = A->tune_tpr[lg] > 0 ? A->tune_tpr[lg] : rt().spmv_tpr[lg];
  switch (NV) {
    case 1: launch_spmv_nv<T, 1, 1>(A, S, p, false); break;
    case 2: launch_spmv_nv<T, 2, 1>(A, S, p, vec); break;
    case 4:
      if (tpr == 2) launch_spmv_nv<T, 4, 2>(A, S, p, vec);
      else launch_spmv_nv<T, 4, 1>(A, S, p, vec);
      break;
    case 8:
      if (tpr == 4) launch_spmv_nv<T, 8, 4>(A, S, p, vec);
      else if (tpr == 1) launch_spmv_nv<T, 8, 1>(A, S, p, vec);
      else launch_spmv_nv<T, 8, 2>(A, S, p, vec);
      break;
    case 16:
      if (tpr == 8) launch_spmv_nv<T, 16, 8>(A, S, p, vec);
      else if (tpr == 2) launch_spmv_nv<T, 16, 2>(A, S, p, vec);
      else launch_spmv_nv<T, 16, 4>(A, S, p, vec);
      break;
    default:
      if (tpr == 16) launch_spmv_nv<T, 32, 16>(A, S, p, vec);
      else if (tpr == 4) launch_spmv_nv<T, 32, 4>(A, S, p, vec);
      else launch_spmv_nv<T, 32, 8>(A, S, p, vec);
      break;
  }
}

// W = alpha*A*V + beta*W with W'W (Gw) and V'W (Gv) formed in the same pass
// by the prefetching kernel (fused_spmv_mvTmv).  W may be NULL (beta = 0,
// W not stored).  False when the single pass does not apply (width not a
// power of two <= 16, unaligned or strided blocks, long rows, SELL C != 32):
// the caller then runs SpMMV and the products as separate passes.
template <class T, int NV, int TPR>
void launch_spmv_gram_nv(const SparseMat<T>* A, SpmvArgs<T>& p, SdMat<T>* Gw, SdMat<T>* Gv)
{
  constexpr int NT = TPR == 1 ? 128 : 256;
  constexpr int RPB = NT / TPR;
  auto kern = pf_kernel<T, NV, TPR, NT, true>();
  static std::atomic<int> occ{0};
  if (occ.load() == 0) {
    int o = 0;
    PB_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&o, kern, NT, 0));
    occ.store(std::max(1, o));
  }
  const int64_t ntiles = ceil_div(A->nchunks, RPB / 32);
  const int grid = (int)std::max<int64_t>(1, std::min<int64_t>(ntiles, (int64_t)rt().num_sms() * occ.load()));
  T* part = (T*)rt().scratch(sizeof(T) * 2 * (size_t)grid * NV * NV);
  p.gram_w = Gw ? part : nullptr;
  p.gram_v = Gv ? part + (size_t)grid * NV * NV : nullptr;
  kern<<<grid, NT, 0, stream()>>>(sell_dev(A), p);
  PB_LAUNCH_CHECK();
  const int rb = (int)ceil_div(NV * NV, 32);
  if (Gw) {
    k_reduce_partials<T><<<rb, 256, 0, stream()>>>(p.gram_w, grid, NV * NV, Gw->d(), NV, Gw->lda, T(1), T(0));
    PB_LAUNCH_CHECK();
  }
  if (Gv) {
    k_reduce_partials<T><<<rb, 256, 0, stream()>>>(p.gram_v, grid, NV * NV, Gv->d(), NV, Gv->lda, T(1), T(0));
    PB_LAUNCH_CHECK();
  }
}

template <class T>
bool spmv_gram_fused(T alpha, const SparseMat<T>* A, const Mvec<T>* V, T beta, Mvec<T>* W, SdMat<T>* Gw,
                     SdMat<T>* Gv)
{
  const int nv = V->nvec;
  // widths 1..16; at 32 the products (2*32*32 FMAs per row on the FP64
  // tensor cores) make the single pass slower than SpMMV plus two Gram
  // passes on the benchmark matrix (826 us against about 670 us)
  const int NV = nv <= 1 ? 1 : nv <= 2 ? 2 : nv <= 4 ? 4 : nv <= 8 ? 8 : nv <= 16 ? 16 : 0;
  if (NV != nv || alpha == T(0) || A->nnz == 0 || !rt().spmv_pf) return false;
  if (!(A->C == 32 && A->max_row_len <= 8)) return false;
  const int vw = 16 / (int)sizeof(T);
  if (NV >= 2 && (!aligned16<T>(V->d()) || V->lda % vw != 0)) return false;
  if (NV >= 2 && W && (!aligned16<T>(W->d()) || W->lda % vw != 0)) return false;
  if (sizeof(T) == 4 && NV == 2) return false;
  SpmvArgs<T> p;
  memset(&p, 0, sizeof(p));
  p.alpha = alpha;
  p.beta = W ? beta : T(0);
  p.x = V->d();
  p.ldx = V->lda;
  p.y = W ? W->d() : nullptr;
  p.ldy = W ? W->lda : 0;
  p.nvec = nv;
  p.no_store = W ? 0 : 1;
  switch (NV) {
    case 1: launch_spmv_gram_nv<T, 1, 1>(A, p, Gw, Gv); break;
    case 2: launch_spmv_gram_nv<T, 2, 1>(A, p, Gw, Gv); break;
    case 4: launch_spmv_gram_nv<T, 4, 1>(A, p, Gw, Gv); break;
    case 8: launch_spmv_gram_nv<T, 8, 2>(A, p, Gw, Gv); break;
    default: launch_spmv_gram_nv<T, 16, 4>(A, p, Gw, Gv); break;
  }
  return true;
}

// general entry: tiles of <= 32 columns; dots returned to host arrays
template <class T>
void spmv_general(T alpha, const SparseMat<T>* A, const T* shifts, const Mvec<T>* X, T beta,
                  Mvec<T>* Y, T* WdotW, T* VdotW, T gamma, T delta, Mvec<T>* U)
{
  PB_REQUIRE(X->nvec == Y->nvec, PB_INVALID_INPUT, "X has %d columns, Y %d", X->nvec, Y->nvec);
  PB_REQUIRE(X->nrows == A->ncols && Y->nrows == A->nrows, PB_INVALID_INPUT,
             "shape mismatch: A %lldx%lld, X %d rows, Y %d rows", (long long)A->nrows,
             (long long)A->ncols, X->nrows, Y->nrows);
  if (U) {
    PB_REQUIRE(U->nvec == Y->nvec && U->nrows == Y->nrows, PB_INVALID_INPUT, "U shape mismatch");
  }
  const int nvec = X->nvec;
  if (alpha == T(0) || A->nnz == 0) {
    // crsmat_module.F90:1508-1511: only scale Y; the fused extras still apply
    if (Y->nrows > 0) {
      k_scale_rows<T><<<grid_for((int64_t)Y->nrows * nvec), 256, 0, stream()>>>(Y->d(), Y->lda, Y->nrows, nvec, beta);
      PB_LAUNCH_CHECK();
    }
    if (!WdotW && !VdotW && !U) return;
    // fall through with alpha = 0: the kernel computes y = beta*y once more
    // from the scaled values would be wrong, so do the extras explicitly
    if (U) {
      k_axpby<T><<<grid_for((int64_t)Y->nrows * nvec), 256, 0, stream()>>>(Y->d(), Y->lda, U->d(), U->lda, Y->nrows, nvec, gamma, nullptr, delta);
      PB_LAUNCH_CHECK();
    }
    // dots written by the final reduction straight into the mapped mailbox
    T* dd = (T*)rt().mailbox_dev();
    const T* hbox = (const T*)rt().mailbox_host();
    for (int c0 = 0; c0 < nvec; c0 += 64) {
      const int nv = std::min(64, nvec - c0);
      auto dotk = [&](const Mvec<T>* P, int poff, T* out) {
        const int grid = std::min(grid_for(P->nrows), rt().num_sms() * 4);
        T* part = (T*)rt().scratch(sizeof(T) * (size_t)grid * 64);
        k_coldot<T, 64><<<grid, 256, 0, stream()>>>(P->d() + poff, P->lda, Y->d() + c0, Y->lda, Y->nrows, nv, part, rt().counters(), dd);
        PB_LAUNCH_CHECK();
        rt().sync();
        for (int j = 0; j < nv; j++) out[c0 + j] = hbox[j];
      };
      if (WdotW) dotk(Y, c0, WdotW);
      if (VdotW) dotk(X, c0, VdotW);
    }
    return;
  }
  // fused dots: the kernel's final reduction writes into the mapped mailbox
  T* dots_dev = (WdotW || VdotW) ? (T*)rt().mailbox_dev() : nullptr;
  const T* hd = (const T*)rt().mailbox_host();
  for (int c0 = 0; c0 < nvec; c0 += 32) {
    const int nv = std::min(32, nvec - c0);
    SpmvArgs<T> p;
    memset(&p, 0, sizeof(p));
    p.alpha = alpha;
    p.beta = beta;
    p.x = X->d();
    p.ldx = X->lda;
    p.y = Y->d();
    p.ldy = Y->lda;
    p.col0 = c0;
    p.want_wdw = WdotW != nullptr;
    p.want_vdw = VdotW != nullptr;
    p.dots_out = dots_dev;
    p.gamma = gamma;
    p.delta = delta;
    p.u = U ? U->d() : nullptr;
    p.ldu = U ? U->lda : 0;
    if (shifts) {
      p.has_shift = 1;
      for (int j = 0; j < nv; j++) p.sh[j] = shifts[c0 + j];
    }
    spmv_tile<T>(A, p, nv);
    if (dots_dev) {
      const int NV = nv <= 1 ? 1 : nv <= 2 ? 2 : nv <= 4 ? 4 : nv <= 8 ? 8 : nv <= 16 ? 16 : 32;
      rt().sync();
      for (int j = 0; j < nv; j++) {
        if (WdotW) WdotW[c0 + j] = hd[j];
        if (VdotW) VdotW[c0 + j] = hd[NV + j];
      }
    }
  }
}

// ======================================================================
// block products
// ======================================================================
// cuTensorMapEncodeTiled through the runtime's driver entry point (no
// link-time dependency on libcuda)
inline PFN_cuTensorMapEncodeTiled_v12000 tmap_encoder()
{
  static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
  static std::once_flag once;
  std::call_once(once, [] {
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = (PFN_cuTensorMapEncodeTiled_v12000)p;
    else
      cudaGetLastError();
  });
  return fn;
}

// 2D tensor map of a row-major block (nrows x ncols, leading dimension ld)
// with boxes of box_rows x box_cols (columns past ncols read as zero).
// False where TMA cannot describe the block: base not 16-byte aligned, row
// stride not a multiple of 16 bytes, or a box beyond the hardware limits.
template <class T>
bool make_rows_tmap(CUtensorMap* map, const T* base, int64_t nrows, int ncols, int64_t ld, int box_cols,
                    int box_rows)
{
  auto fn = tmap_encoder();
  if (!fn || nrows < 1 || ncols < 1 || nrows >= (int64_t(1) << 31)) return false;
  if ((((uintptr_t)base) & 15u) != 0 || ((size_t)ld * sizeof(T)) % 16 != 0) return false;
  if (box_cols > 256 || box_rows > 256 || ((size_t)box_cols * sizeof(T)) % 16 != 0) return false;
  cuuint64_t dims[2] = {(cuuint64_t)ncols, (cuuint64_t)nrows};
  cuuint64_t strides[1] = {(cuuint64_t)((size_t)ld * sizeof(T))};
  cuuint32_t box[2] = {(cuuint32_t)box_cols, (cuuint32_t)box_rows};
  cuuint32_t estr[2] = {1, 1};
  const CUresult r = fn(map, sizeof(T) == 8 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT64 : CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 2,
                        (void*)base, dims, strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
                        CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                        CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  return r == CUDA_SUCCESS;
}

inline int pad_width5(int w) { return w <= 4 ? 4 : w <= 8 ? 8 : w <= 16 ? 16 : w <= 32 ? 32 : 64; }

// k_mvtmv_async launch for padded widths BM x BK: micro-tile TT by output
// size; R rows per stage sized for about 32 KiB of staged rows, 3 stages,
// two blocks per SM (the reduction buffer may need more shared memory for
// the widest tiles, which are compute-bound anyway)
template <class T, int BM, int BK>
void mvtmv_async_launch(MvTmvArgs<T>& a, int64_t n)
{
  constexpr int TT = (BM * BK <= 64) ? 2 : (BM * BK <= 1024) ? 4 : 8;
  constexpr int VWd = 16 / (int)sizeof(T);
  constexpr int PV = BM + VWd, PW = BK + VWd;
  constexpr int RR = ((32768 / (int)sizeof(T)) / (PV + PW)) / 16 * 16;
  constexpr int R = RR < 16 ? 16 : RR;
  constexpr int S = 3;
  constexpr int NT = (BM / TT) * (BK / TT), RG = 256 / NT;
  const size_t stage = sizeof(T) * (size_t)S * R * (PV + PW);
  const size_t red = sizeof(T) * (size_t)RG * BM * BK;
  const size_t smem = std::max(stage, red);
  const int grid = (int)std::min<int64_t>(ceil_div(n > 0 ? n : 1, R), (int64_t)rt().num_sms() * 2);
  a.part = (T*)rt().scratch(sizeof(T) * (size_t)grid * a.m * a.k);
  a.counter = rt().counters();
  a.R = R;
  // many outputs: the cross-block sum as a second, GPU-wide pass
  const int nout = a.m * a.k;
  a.ext_reduce = (nout >= 64 && grid > 1) ? 1 : 0;
  // FP64 on the tensor cores (DMMA) for widths that are multiples of 8
  if constexpr (std::is_same<T, double>::value && BM >= 8 && BK >= 8) {
    constexpr int DPV = BM + 4, DPW = BK + 4;
    constexpr int DR0 = (4096 / (DPV + DPW)) / 32 * 32;
    constexpr int DR = DR0 < 32 ? 32 : DR0 > 256 ? 256 : DR0;
    CUtensorMap mV, mW;
    if (rt().use_tma && rt().use_dmma && make_rows_tmap<T>(&mV, a.V, n, a.m, a.ldv, DPV, DR) &&
        make_rows_tmap<T>(&mW, a.W, n, a.k, a.ldw, DPW, DR)) {
      const size_t dsmem = sizeof(T) * (size_t)S * DR * (DPV + DPW) + 8 * S;
      const int dgrid = (int)std::min<int64_t>(ceil_div(n, DR), (int64_t)rt().num_sms() * 2);
      a.part = (T*)rt().scratch(sizeof(T) * (size_t)dgrid * a.m * a.k);
      a.ext_reduce = (nout >= 64 && dgrid > 1) ? 1 : 0;
      a.R = DR;
      auto kd = k_mvtmv_dmma<BM, BK, DR, S>;
      set_smem(kd, dsmem);
      kd<<<dgrid, BLK_BS, dsmem, stream()>>>(a, mV, mW, rt().device_error_word());
      if (a.ext_reduce) {
        PB_LAUNCH_CHECK();
        k_reduce_partials<T><<<(nout + 31) / 32, 256, 0, stream()>>>(a.part, dgrid, nout, a.Cd, a.m, a.ldc,
                                                                      a.alpha, a.beta);
      }
      return;
    }
  }
  // TMA staging where both blocks can be described by tensor maps
  constexpr int RT = R > 256 ? 256 : R;
  CUtensorMap mapV, mapW;
  if (rt().use_tma && make_rows_tmap<T>(&mapV, a.V, n, a.m, a.ldv, PV, RT) &&
      make_rows_tmap<T>(&mapW, a.W, n, a.k, a.ldw, PW, RT)) {
    const size_t tstage = sizeof(T) * (size_t)S * RT * (PV + PW) + 8 * S;
    const size_t tsmem = std::max(tstage, red);
    const int tgrid = (int)std::min<int64_t>(ceil_div(n, RT), (int64_t)rt().num_sms() * 2);
    a.part = (T*)rt().scratch(sizeof(T) * (size_t)tgrid * a.m * a.k);
    a.ext_reduce = (nout >= 64 && tgrid > 1) ? 1 : 0;
    a.R = RT;
    auto kern = k_mvtmv_tma<T, BM, BK, TT, RT, S>;
    set_smem(kern, tsmem);
    kern<<<tgrid, BLK_BS, tsmem, stream()>>>(a, mapV, mapW, rt().device_error_word());
    if (a.ext_reduce) {
      PB_LAUNCH_CHECK();
      k_reduce_partials<T><<<(nout + 31) / 32, 256, 0, stream()>>>(a.part, tgrid, nout, a.Cd, a.m, a.ldc, a.alpha,
                                                                    a.beta);
    }
    return;
  }
  auto kern = k_mvtmv_async<T, BM, BK, TT, R, S>;
  set_smem(kern, smem);
  kern<<<grid, BLK_BS, smem, stream()>>>(a);
  if (a.ext_reduce) {
    PB_LAUNCH_CHECK();
    k_reduce_partials<T><<<(nout + 31) / 32, 256, 0, stream()>>>(a.part, grid, nout, a.Cd, a.m, a.ldc, a.alpha,
                                                                  a.beta);
  }
}

template <class T, int BM>
void mvtmv_async_bk(MvTmvArgs<T>& a, int64_t n, int BK)
{
  switch (BK) {
    case 4: mvtmv_async_launch<T, BM, 4>(a, n); break;
    case 8: mvtmv_async_launch<T, BM, 8>(a, n); break;
    case 16: mvtmv_async_launch<T, BM, 16>(a, n); break;
    case 32: mvtmv_async_launch<T, BM, 32>(a, n); break;
    default: mvtmv_async_launch<T, BM, 64>(a, n); break;
  }
}

template <class T>
void mvtmv_async(MvTmvArgs<T>& a, int64_t n, int BM, int BK)
{
  switch (BM) {
    case 4: mvtmv_async_bk<T, 4>(a, n, BK); break;
    case 8: mvtmv_async_bk<T, 8>(a, n, BK); break;
    case 16: mvtmv_async_bk<T, 16>(a, n, BK); break;
    case 32: mvtmv_async_bk<T, 32>(a, n, BK); break;
    default: mvtmv_async_bk<T, 64>(a, n, BK); break;
  }
}

// C = alpha*V'W + beta*C with compensated (double-double) sums, for
// PHIST_ROBUST_REDUCTIONS (pb_prec.cuh); result blocks of at most 64 x 64
inline void launch_mvTmv_prec(int64_t n, int m, int k, double alpha, const double* V, int64_t ldv,
                              const double* W, int64_t ldw, double beta, double* Cd, int64_t ldc)
{
  for (int r0 = 0; r0 < m; r0 += 64)
    for (int j0 = 0; j0 < k; j0 += 64) {
      MvTmvPrecArgs a;
      a.n = n;
      a.m = std::min(64, m - r0);
      a.k = std::min(64, k - j0);
      a.V = V + r0; a.ldv = ldv;
      a.W = W + j0; a.ldw = ldw;
      a.alpha = alpha; a.beta = beta;
      a.C = Cd + r0 + (int64_t)j0 * ldc; a.ldc = ldc;
      const int nout = a.m * a.k;
      const int nq = (int)ceil_div(nout, PREC_BS);
      const int64_t ntiles = ceil_div(n, PREC_R);
      const int grid = (int)std::max<int64_t>(1, std::min<int64_t>(ntiles, 2 * (int64_t)rt().num_sms()));
      a.part = (double*)rt().scratch(sizeof(double) * 2 * (size_t)grid * nout);
      a.counter = rt().counters();
      if (nq <= 1) k_mvTmv_prec<1><<<grid, PREC_BS, 0, stream()>>>(a);
      else if (nq <= 2) k_mvTmv_prec<2><<<grid, PREC_BS, 0, stream()>>>(a);
      else if (nq <= 4) k_mvTmv_prec<4><<<grid, PREC_BS, 0, stream()>>>(a);
      else if (nq <= 8) k_mvTmv_prec<8><<<grid, PREC_BS, 0, stream()>>>(a);
      else k_mvTmv_prec<16><<<grid, PREC_BS, 0, stream()>>>(a);
      PB_LAUNCH_CHECK();
    }
}

// the Gram product a caller asked for: compensated sums when the caller sets
// PHIST_ROBUST_REDUCTIONS in FP64 (PHIST's builtin has no FP32 robust
// kernels either: its S/C/Z types are not implemented, builtin/kernels.cpp:270-283)
template <class T>
bool robust_requested(int flags_in)
{
  return (flags_in & PB_ROBUST_REDUCTIONS) && std::is_same<T, double>::value;
}

template <class T>
void launch_mvTmv(int64_t n, int m, int k, T alpha, const T* V, int64_t ldv, const T* W,
                  int64_t ldw, T beta, T* Cd, int64_t ldc)
{
  MvTmvArgs<T> a;
  a.n = n; a.m = m; a.k = k; a.V = V; a.ldv = ldv; a.W = W; a.ldw = ldw;
  a.alpha = alpha; a.beta = beta; a.Cd = Cd; a.ldc = ldc;
  if constexpr (std::is_same<T, double>::value) {
    // FP64 blocks of exactly 4 columns on 32-byte row boundaries: thread per
    // row with 256-bit loads (n = 2,097,152: 38.9 us against 51.7 us for
    // the staged tile kernel; at 8 columns the tile kernel stays faster,
    // 68.9 against 71.8 us)
    const bool a32 = ((uintptr_t)V & 31u) == 0 && ((uintptr_t)W & 31u) == 0 && ldv % 4 == 0 && ldw % 4 == 0;
    if (rt().spmv_v256 && a32 && m == 4 && k == 4 && n > 0) {
      static std::atomic<int> occ[1];
      auto run = [&](auto kern, std::atomic<int>& o) {
        if (o.load() == 0) {
          int b = 0;
          PB_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, kern, 256, 0));
          o.store(std::max(1, b));
        }
        const int grid = (int)std::max<int64_t>(1, std::min<int64_t>(ceil_div(n, 256), (int64_t)rt().num_sms() * o.load()));
        a.part = (T*)rt().scratch(sizeof(T) * (size_t)grid * m * k);
        a.counter = rt().counters();
        a.R = 0;
        kern<<<grid, 256, 0, stream()>>>(a);
        PB_LAUNCH_CHECK();
      };
      run(k_mvTmv_v4<4, 4, 4>, occ[0]);
      return;
    }
  }
  if (m <= 64 && k <= 64 && vec_ok(V, ldv, m) && vec_ok(W, ldw, k)) {
    // multi-stage asynchronously staged row tiles, widths padded to 4..64
    mvtmv_async<T>(a, n, pad_width5(m), pad_width5(k));
    PB_LAUNCH_CHECK();
    return;
  }
  if (m <= 8 && k <= 8) {
    // register kernel (odd or unaligned widths): padded widths M (4|8) and K (1|4|8)
    const int M = m <= 4 ? 4 : 8, K = k == 1 ? 1 : k <= 4 ? 4 : 8;
    const int grid = std::max(1, std::min(grid_for(n), rt().num_sms() * 4));
    a.part = (T*)rt().scratch(sizeof(T) * (size_t)grid * M * K);
    a.counter = rt().counters();
    a.R = 0;
#define PB_MVR(Mv, Kv) k_mvTmv_reg<T, Mv, Kv><<<grid, 256, 0, stream()>>>(a)
    if (M == 4) {
      if (K == 1) PB_MVR(4, 1); else if (K == 4) PB_MVR(4, 4); else PB_MVR(4, 8);
    } else {
      if (K == 1) PB_MVR(8, 1); else if (K == 4) PB_MVR(8, 4); else PB_MVR(8, 8);
    }
#undef PB_MVR
    PB_LAUNCH_CHECK();
    return;
  }
  const bool big = (int64_t)m * k >= 256;
  const int TM = big ? 8 : 4, TK = big ? 8 : 4;
  const int mp = ceil_div(m, TM) * TM, kp = ceil_div(k, TK) * TK;
  const int nt = (mp / TM) * (kp / TK);
  PB_REQUIRE(nt <= BLK_BS, PB_NOT_IMPLEMENTED, "mvecT_times_mvec with %dx%d result exceeds one block's tiles", m, k);
  const int RG = BLK_BS / nt;
  a.R = std::max(32, ((RG * 4 + 31) / 32) * 32);
  a.R = std::min(a.R, 128);
  size_t smem = sizeof(T) * (size_t)a.R * (mp + kp);
  const size_t red = sizeof(T) * (size_t)RG * mp * kp;
  if (red > smem) smem = red;
  const int64_t ntiles = ceil_div(n > 0 ? n : 1, a.R);
  const int grid = (int)std::min<int64_t>(ntiles, (int64_t)rt().num_sms() * 2);
  a.part = (T*)rt().scratch(sizeof(T) * (size_t)grid * m * k);
  a.counter = rt().counters();
  if (big) {
    auto kern = k_mvTmv<T, 8, 8>;
    set_smem(kern, smem);
    kern<<<grid, BLK_BS, smem, stream()>>>(a);
  } else {
    auto kern = k_mvTmv<T, 4, 4>;
    set_smem(kern, smem);
    kern<<<grid, BLK_BS, smem, stream()>>>(a);
  }
  PB_LAUNCH_CHECK();
}

// k_mvsd_async launch for padded widths BM x BK: TC output columns per
// thread (TX = BK/TC threads per row), TR rows per thread, sized for about
// 24 KiB of staged input rows per stage; 4 stages (3 where a stage is
// larger), two blocks per SM
template <class T, int BM, int BK>
void mvsd_async_launch(RowGemmArgs<T>& a)
{
  constexpr int TC = BK >= 16 ? 4 : BK / 4;
  constexpr int TX = BK / TC, TY = 256 / TX;
  constexpr int AP = BM + 16 / (int)sizeof(T);
  constexpr int TR0 = 24576 / (TY * AP * (int)sizeof(T));
  constexpr int TR = TR0 < 1 ? 1 : TR0 > 8 ? 8 : TR0;
  constexpr int R = TY * TR;
  constexpr int S = (R * AP * (int)sizeof(T) > 30000) ? 3 : 4;
  const size_t smem = sizeof(T) * ((size_t)BM * BK + (size_t)S * R * AP);
  const int grid = (int)std::min<int64_t>(ceil_div(a.n > 0 ? a.n : 1, R), (int64_t)rt().num_sms() * 2);
  if constexpr (std::is_same<T, double>::value && BM >= 8 && BK >= 8) {
    // FP64 on the tensor cores (DMMA), rows staged by TMA
    constexpr int DAP = BM + 4, DCP = BK + 4;
    constexpr int DR = (DAP * 8 * 128 <= 24576) ? 128 : 64;
    constexpr int DS = (DR * DAP * 8 > 30000) ? 3 : 4;
    constexpr int DCSZ = (BM * DCP * 8 + 127) / 128 * 128 / 8;
    const T* A = (a.mode == RM_MVSDI) ? (const T*)a.W : a.V;
    const int64_t lda = (a.mode == RM_MVSDI) ? a.ldw : a.ldv;
    CUtensorMap mA;
    if (rt().use_tma && rt().use_dmma && make_rows_tmap<T>(&mA, A, a.n, a.m, lda, DAP, DR)) {
      const size_t dsmem = sizeof(T) * ((size_t)DCSZ + (size_t)DS * DR * DAP) + 8 * DS;
      const int dgrid = (int)std::min<int64_t>(ceil_div(a.n, DR), (int64_t)rt().num_sms() * 2);
      auto kd = k_mvsd_dmma<BM, BK, DR, DS>;
      set_smem(kd, dsmem);
      kd<<<dgrid, BLK_BS, dsmem, stream()>>>(a, mA, rt().device_error_word());
      return;
    }
  }
  {
    // TMA staging of the input rows where a tensor map describes them
    constexpr int TRT = (TY * TR > 256) ? 256 / TY : TR;
    constexpr int RT = TY * TRT;
    const T* A = (a.mode == RM_MVSDI) ? (const T*)a.W : a.V;
    const int64_t lda = (a.mode == RM_MVSDI) ? a.ldw : a.ldv;
    CUtensorMap mapA;
    if (rt().use_tma && make_rows_tmap<T>(&mapA, A, a.n, a.m, lda, AP, RT)) {
      constexpr int CSZ = (BM * BK * (int)sizeof(T) + 127) / 128 * 128 / (int)sizeof(T);
      const size_t tsmem = sizeof(T) * ((size_t)CSZ + (size_t)S * RT * AP) + 8 * S;
      const int tgrid = (int)std::min<int64_t>(ceil_div(a.n, RT), (int64_t)rt().num_sms() * 2);
      auto kt = k_mvsd_tma<T, BM, BK, TRT, TC, S>;
      set_smem(kt, tsmem);
      kt<<<tgrid, BLK_BS, tsmem, stream()>>>(a, mapA, rt().device_error_word());
      return;
    }
  }
  auto kern = k_mvsd_async<T, BM, BK, TR, TC, S>;
  set_smem(kern, smem);
  kern<<<grid, BLK_BS, smem, stream()>>>(a);
}

template <class T, int BM>
void mvsd_async_bk(RowGemmArgs<T>& a, int BK)
{
  switch (BK) {
    case 4: mvsd_async_launch<T, BM, 4>(a); break;
    case 8: mvsd_async_launch<T, BM, 8>(a); break;
    case 16: mvsd_async_launch<T, BM, 16>(a); break;
    case 32: mvsd_async_launch<T, BM, 32>(a); break;
    default: mvsd_async_launch<T, BM, 64>(a); break;
  }
}

template <class T>
void mvsd_async(RowGemmArgs<T>& a, int BM, int BK)
{
  switch (BM) {
    case 4: mvsd_async_bk<T, 4>(a, BK); break;
    case 8: mvsd_async_bk<T, 8>(a, BK); break;
    case 16: mvsd_async_bk<T, 16>(a, BK); break;
    case 32: mvsd_async_bk<T, 32>(a, BK); break;
    default: mvsd_async_bk<T, 64>(a, BK); break;
  }
}

// fused V*C + Gram on the tensor cores (FP64, widths 8..64 in steps of 8)
template <int BM, int BK, int MV, int GM>
bool mvsd_gram_dmma_launch(RowGemmArgs<double>& a)
{
  constexpr int R = (BK >= 32 || MV >= 32) ? 64 : 128;
  constexpr int AP = BM + 4, CP = BK + 4, PT = BK + 4, PVG = MV + 4;
  constexpr int CSZ = (BM * CP * 8 + 127) / 128 * 128 / 8;
  constexpr int VSZ = (GM == GM_VW) ? R * PVG : 0;
  constexpr size_t BYTES3 = 8 * ((size_t)CSZ + 3 * (size_t)R * AP + 3 * (size_t)VSZ + (size_t)R * PT) + 24;
  constexpr int S = BYTES3 <= 200 * 1024 ? 3 : 2;
  const double* A = (a.mode == RM_MVSDI) ? (const double*)a.W : a.V;
  const int64_t lda = (a.mode == RM_MVSDI) ? a.ldw : a.ldv;
  CUtensorMap mA, mV;
  if (!make_rows_tmap<double>(&mA, A, a.n, a.m, lda, AP, R)) return false;
  if (GM == GM_VW) {
    if (!make_rows_tmap<double>(&mV, a.Vg, a.n, a.mv, a.ldvg, PVG, R)) return false;
  } else {
    mV = mA;
  }
  const size_t smem = 8 * ((size_t)CSZ + (size_t)S * R * AP + (size_t)S * VSZ + (size_t)R * PT) + 8 * S;
  // one wave of as many blocks as fit an SM (shared memory allows 4 at
  // width 8, 2 from width 16 on)
  auto kern = k_mvsd_gram_dmma<BM, BK, MV, R, S, GM>;
  set_smem(kern, smem);
  static std::atomic<int> occ{0};
  if (occ.load() == 0) {
    int o = 0;
    PB_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&o, kern, BLK_BS, smem));
    occ.store(std::max(1, o));
  }
  const int grid = (int)std::min<int64_t>(ceil_div(a.n, R), (int64_t)rt().num_sms() * occ.load());
  const int gm = (GM == GM_WW) ? a.k : a.mv;
  const int nout = gm * a.k;
  a.part = (double*)rt().scratch(sizeof(double) * (size_t)grid * nout);
  a.counter = rt().counters();
  const bool ext = nout >= 64 && grid > 1;
  a.R = ext ? -1 : R;
  kern<<<grid, BLK_BS, smem, stream()>>>(a, mA, mV, rt().device_error_word());
  PB_LAUNCH_CHECK();
  if (ext) {
    k_reduce_partials<double><<<(nout + 31) / 32, 256, 0, stream()>>>(a.part, grid, nout, a.Gd, gm, a.ldg, a.galpha,
                                                                      a.gbeta);
    PB_LAUNCH_CHECK();
  }
  return true;
}

template <int BM, int BK, int GM>
bool mvsd_gram_dmma_mv(RowGemmArgs<double>& a, int MV)
{
  switch (MV) {
    case 8: return mvsd_gram_dmma_launch<BM, BK, 8, GM>(a);
    case 16: return mvsd_gram_dmma_launch<BM, BK, 16, GM>(a);
    case 32: return mvsd_gram_dmma_launch<BM, BK, 32, GM>(a);
    default: return mvsd_gram_dmma_launch<BM, BK, 64, GM>(a);
  }
}

// true if the fused tensor-core kernel took the product
inline bool mvsd_gram_dmma(RowGemmArgs<double>& a)
{
  if (!rt().use_tma || !rt().use_dmma || a.mode == RM_VCWD || a.gram == GM_NONE) return false;
  if (a.m > 64 || a.k > 64 || a.m < 5 || a.k < 5) return false;  // widths <= 4: register kernel
  const int BM = pad_width5(a.m), BK = pad_width5(a.k);
  if (a.gram == GM_WW) {
    switch (BM * 100 + BK) {
#define PB_GW(bm, bk) \
  case bm * 100 + bk: return mvsd_gram_dmma_launch<bm, bk, bk, GM_WW>(a);
      PB_GW(8, 8) PB_GW(8, 16) PB_GW(8, 32) PB_GW(8, 64) PB_GW(16, 8) PB_GW(16, 16) PB_GW(16, 32) PB_GW(16, 64)
      PB_GW(32, 8) PB_GW(32, 16) PB_GW(32, 32) PB_GW(32, 64) PB_GW(64, 8) PB_GW(64, 16) PB_GW(64, 32)
      PB_GW(64, 64)
#undef PB_GW
      default: return false;
    }
  }
  // V'W with the in-place product: square blocks only (BM == BK)
  if (a.mv < 5 || a.mv > 64 || BM != BK) return false;
  const int MV = pad_width5(a.mv);
  switch (BM) {
    case 8: return mvsd_gram_dmma_mv<8, 8, GM_VW>(a, MV);
    case 16: return mvsd_gram_dmma_mv<16, 16, GM_VW>(a, MV);
    case 32: return mvsd_gram_dmma_mv<32, 32, GM_VW>(a, MV);
    default: return mvsd_gram_dmma_mv<64, 64, GM_VW>(a, MV);
  }
}
inline bool mvsd_gram_dmma(RowGemmArgs<float>&) { return false; }

template <class T>
void launch_rowgemm(RowGemmArgs<T>& a)
{
  // fused V*C + Gram in one pass on the tensor cores
  if (mvsd_gram_dmma(a)) return;
  {
    // gram-free V*C and in-place W*C on aligned widths: multi-stage staged tiles
    const T* A = (a.mode == RM_MVSDI) ? (const T*)a.W : a.V;
    const int64_t lda = (a.mode == RM_MVSDI) ? a.ldw : a.ldv;
    if (a.gram == GM_NONE && a.mode != RM_VCWD && a.m <= 64 && a.k <= 64 && vec_ok(A, lda, a.m)) {
      mvsd_async<T>(a, pad_width5(a.m), pad_width5(a.k));
      PB_LAUNCH_CHECK();
      return;
    }
  }
  if (a.m <= 8 && a.k <= 8 && (a.gram != GM_VW || a.mv <= 8)) {
    // register kernel: padded widths M (4|8), K (1|4|8), MV (1, or 8 for V'W)
    const int M = a.m <= 4 ? 4 : 8, K = a.k == 1 ? 1 : a.k <= 4 ? 4 : 8;
    const int grid = std::max(1, std::min(grid_for(a.n), rt().num_sms() * 4));
    if (a.gram != GM_NONE) {
      a.part = (T*)rt().scratch(sizeof(T) * (size_t)grid * 64);
      a.counter = rt().counters();
    }
#define PB_RGR(Mv, Kv, MVv) k_rowgemm_reg<T, Mv, Kv, MVv><<<grid, 256, 0, stream()>>>(a)
#define PB_RGR_K(Mv, MVv)                                   \
  if (K == 1) PB_RGR(Mv, 1, MVv);                           \
  else if (K == 4) PB_RGR(Mv, 4, MVv);                      \
  else PB_RGR(Mv, 8, MVv);
    if (a.gram == GM_VW) {
      if (M == 4) { PB_RGR_K(4, 8) } else { PB_RGR_K(8, 8) }
    } else {
      if (M == 4) { PB_RGR_K(4, 1) } else { PB_RGR_K(8, 1) }
    }
#undef PB_RGR_K
#undef PB_RGR
    PB_LAUNCH_CHECK();
    return;
  }
  {
    const T* A = (a.mode == RM_MVSDI) ? (const T*)a.W : a.V;
    const int64_t lda = (a.mode == RM_MVSDI) ? a.ldw : a.ldv;
    const bool gram_ok = a.gram == GM_NONE || (vec_ok((const T*)a.W, a.ldw, a.k) &&
                                               (a.gram == GM_WW || (a.mv <= 64 && vec_ok(a.Vg, a.ldvg, a.mv))));
    if (gram_ok && a.mode != RM_VCWD && a.m <= 64 && a.k <= 64 && vec_ok(A, lda, a.m)) {
      // multi-stage staged row tiles, widths padded to 4..64
      mvsd_async<T>(a, pad_width5(a.m), pad_width5(a.k));
      PB_LAUNCH_CHECK();
      // fused Gram at these widths: a second pass over the new W with the
      // staged Gram kernel (the register kernels above fuse it into one pass)
      if (a.gram == GM_WW)
        launch_mvTmv<T>(a.n, a.k, a.k, T(1), a.W, a.ldw, a.W, a.ldw, T(0), a.Gd, a.ldg);
      else if (a.gram == GM_VW)
        launch_mvTmv<T>(a.n, a.mv, a.k, a.galpha, a.Vg, a.ldvg, a.W, a.ldw, a.gbeta, a.Gd, a.ldg);
      return;
    }
  }
  // micro-tile: TK columns per thread, TR rows
  const int TK = a.k >= 32 ? 8 : a.k >= 8 ? 4 : a.k >= 2 ? 2 : 1;
  const int kp = ceil_div(a.k, TK) * TK;
  const int ntk = kp / TK;
  const int ntr = BLK_BS / ntk;
  const int TR = (a.k >= 32) ? 4 : 1;
  a.R = ntr * TR;
  const int ap = a.m + (a.m & 1);
  const int mvp = a.mv + (a.mv & 1);
  size_t smem = sizeof(T) * ((size_t)a.R * ap + (size_t)a.R * kp + (size_t)ap * kp +
                             (a.mode == RM_VCWD ? (size_t)kp * kp : 0) +
                             (a.gram == GM_VW ? (size_t)a.R * mvp : 0));
  // (plus the reduction's static shared buffer, 8 KiB)
  PB_REQUIRE(smem + 9 * 1024 <= 227 * 1024, PB_NOT_IMPLEMENTED, "block product too wide for one tile (%zu bytes of shared memory)", smem);
  const int gm = (a.gram == GM_WW) ? a.k : a.mv;
  PB_REQUIRE(a.gram == GM_NONE || gm * a.k <= 16 * BLK_BS, PB_NOT_IMPLEMENTED, "fused Gram matrix larger than 64x64");
  const int64_t ntiles = ceil_div(a.n > 0 ? a.n : 1, a.R);
  const int grid = (int)std::min<int64_t>(ntiles, (int64_t)rt().num_sms() * 4);
  if (a.gram != GM_NONE) {
    a.part = (T*)rt().scratch(sizeof(T) * (size_t)grid * gm * a.k);
    a.counter = rt().counters();
  }
#define PB_RG_LAUNCH(TRv, TKv)                                                                 \
  {                                                                                            \
    auto kern = k_rowgemm<T, TRv, TKv>;                                                        \
    set_smem(kern, smem); \
    kern<<<grid, BLK_BS, smem, stream()>>>(a);                                                 \
  }
  if (TK == 8) PB_RG_LAUNCH(4, 8)
  else if (TK == 4) PB_RG_LAUNCH(1, 4)
  else if (TK == 2) PB_RG_LAUNCH(1, 2)
  else PB_RG_LAUNCH(1, 1)
#undef PB_RG_LAUNCH
  PB_LAUNCH_CHECK();
}

template <class T>
RowGemmArgs<T> rowgemm_args()
{
  RowGemmArgs<T> a;
  memset(&a, 0, sizeof(a));
  a.alpha = T(1);
  a.galpha = T(1);
  return a;
}

// ======================================================================
// CARP
// ======================================================================
// Block-coloured layout (pb_carp_blocks.hpp): blocks of at most R rows
// whose footprint has at most 1.25 R rows of X (at least 16; the shared
// memory of every thread block is sized for the largest footprint, and
// compact blocks of the benchmark matrices stay well below it) and whose
// pattern at most 16R entries; R is the runtime carp_block_rows, or, when
// that is 0, 128 for sweeps of up to 8 columns and 64 beyond (width: the
// number of columns the sweeps are expected to have).  False when the matrix has
// rows too long for that, or a block needs more than 64 steps; the caller
// then uses the row colouring.
template <class T>
bool carp_build_blocks(const SparseMat<T>* A, const std::vector<int64_t>& prp, const std::vector<int32_t>& pcol,
                       int width, CarpWork<T>* w)
{
  const int64_t n = A->nrows;
  CarpBlocks B;
  const int R = rt().carp_block_rows > 0 ? rt().carp_block_rows : width <= 8 ? 128 : 64;
  if (!carp_block_partition(n, prp, pcol, R, std::max(16, R + R / 4), std::max(16, 16 * R), B)) return false;
  if (!carp_block_color(n, prp, pcol, B)) return false;
  CarpBlockLayout<T> L;
  carp_block_layout<T>(B, n, A->h_row_ptr.data(), A->h_col.data(), A->h_val.data(), L);
  w->blocks = true;
  w->nbcolors = B.ncolors;
  w->h_bcolor_ptr = B.color_ptr;
  w->max_fp = B.max_fp;
  w->max_rows = B.max_rows;
  w->seg_stride = L.stride;
  {
    // rows without a repeated column let the sweep update gathered values
    std::vector<int64_t> seen(n, -1);
    w->distinct = true;
    for (int64_t i = 0; i < n && w->distinct; i++)
      for (int64_t p = A->h_row_ptr[i]; p < A->h_row_ptr[i + 1]; p++) {
        if (seen[A->h_col[p]] == i) {
          w->distinct = false;
          break;
        }
        seen[A->h_col[p]] = i;
      }
  }
  w->h_rows = B.seq_rows;
  w->h_color_ptr = B.seq_ptr;
  w->ncolors = (int)B.seq_ptr.size() - 1;
  w->d_bseg = (unsigned char*)upload_vec(L.seg);
  return true;
}

template <class T>
CarpWork<T>* carp_build(const SparseMat<T>* A, int nshifts, const T* sr, const T* si, int width = 0)
{
  PB_REQUIRE(A->nrows == A->ncols, PB_INVALID_INPUT, "CARP needs a square matrix");
  CarpWork<T>* w = new CarpWork<T>();
  w->nshifts = nshifts;
  w->sigma_r.assign(sr, sr + nshifts);
  if (si) w->sigma_i.assign(si, si + nshifts);
  else w->sigma_i.assign(nshifts, T(0));
  const int64_t n = A->nrows;
  // The projection of row i also writes x_i through the shift term
  // (x_i += tmp*sigma) even where row i stores no diagonal entry, so the
  // colouring works on the pattern of A with every diagonal present.
  std::vector<int64_t> prp(n + 1, 0);
  std::vector<int32_t> pcol;
  pcol.reserve(A->nnz + n);
  for (int64_t i = 0; i < n; i++) {
    bool has_diag = false;
    for (int64_t p = A->h_row_ptr[i]; p < A->h_row_ptr[i + 1]; p++) {
      pcol.push_back(A->h_col[p]);
      has_diag |= (A->h_col[p] == i);
    }
    if (!has_diag) pcol.push_back((int32_t)i);
    prp[i + 1] = (int64_t)pcol.size();
  }
  w->nrows = n;
  if (rt().carp_blocks && n > 0 && carp_build_blocks(A, prp, pcol, width > 0 ? width : nshifts, w)) {
    rt().sync();
    return w;
  }
  std::vector<int32_t> color;
  w->ncolors = dist2_color(n, A->ncols, prp, pcol, color);
  w->h_color_ptr.assign(w->ncolors + 1, 0);
  for (int64_t i = 0; i < n; i++) w->h_color_ptr[color[i] + 1]++;
  for (int c = 0; c < w->ncolors; c++) w->h_color_ptr[c + 1] += w->h_color_ptr[c];
  std::vector<int32_t> rows(n);
  {
    std::vector<int64_t> fill(w->h_color_ptr.begin(), w->h_color_ptr.end() - 1);
    for (int64_t i = 0; i < n; i++) rows[fill[color[i]]++] = (int32_t)i;
  }
  std::vector<int64_t> rp(n + 1, 0);
  std::vector<int32_t> col;
  std::vector<T> val, nrm(n), dg(n);
  col.reserve(A->nnz);
  val.reserve(A->nnz);
  for (int64_t q = 0; q < n; q++) {
    const int64_t i = rows[q];
    T s = T(0), d = T(0);
    for (int64_t p = A->h_row_ptr[i]; p < A->h_row_ptr[i + 1]; p++) {
      col.push_back(A->h_col[p]);
      val.push_back(A->h_val[p]);
      s += A->h_val[p] * A->h_val[p];
      if (A->h_col[p] == i) d = A->h_val[p];
    }
    nrm[q] = s;
    dg[q] = d;
    rp[q + 1] = (int64_t)col.size();
  }
  w->h_rows = rows;
  w->d_rows = (int32_t*)upload_vec(rows);
  w->d_rp = (int64_t*)upload_vec(rp);
  w->d_col = (int32_t*)upload_vec(col);
  w->d_val = (T*)upload_vec(val);
  w->d_nrm = (T*)upload_vec(nrm);
  w->d_diag = (T*)upload_vec(dg);
  rt().sync();
  return w;
}

template <class T>
void carp_free(CarpWork<T>* w)
{
  if (!w) return;
  rt().dfree(w->d_rows);
  rt().dfree(w->d_rp);
  rt().dfree(w->d_col);
  rt().dfree(w->d_val);
  rt().dfree(w->d_nrm);
  rt().dfree(w->d_diag);
  rt().dfree(w->d_bseg);
  delete w;
}

template <class T, bool RC>
void carp_run_blocks(const CarpWork<T>* w, int nvec, const T* sr, const T* si, const Mvec<T>* B, Mvec<T>* Xr,
                     Mvec<T>* Xi, const T* omega)
{
  for (int c0 = 0; c0 < nvec; c0 += 32) {
    const int nv = std::min(32, nvec - c0);
    KaczBlockArgs<T> a;
    memset(&a, 0, sizeof(a));
    a.seg = w->d_bseg;
    a.nvec = nv;
    a.max_fp = w->max_fp; a.max_rows = w->max_rows; a.seg_stride = w->seg_stride;
    a.distinct = w->distinct ? 1 : 0;
    for (int j = 0; j < nv; j++) {
      a.sig_r[j] = sr[c0 + j];
      a.sig_i[j] = si ? si[c0 + j] : T(0);
      a.omega[j] = omega[c0 + j];
    }
    a.b = B ? B->d() + c0 : nullptr;
    a.ldb = B ? B->lda : 0;
    a.xr = Xr->d() + c0;
    a.ldxr = Xr->lda;
    a.xi = Xi ? Xi->d() + c0 : nullptr;
    a.ldxi = Xi ? Xi->lda : 0;
    // TPR = nv rounded up to a power of two
    const int TPR = nv <= 1 ? 1 : nv <= 2 ? 2 : nv <= 4 ? 4 : nv <= 8 ? 8 : nv <= 16 ? 16 : 32;
    // X and B copied in 16-byte pieces where every row of both starts on a
    // 16-byte boundary and the columns fill whole pieces
    constexpr int WV = 16 / (int)sizeof(T);
    auto al16 = [](const void* p) { return ((uintptr_t)p & 15) == 0; };
    const bool wide = nv % WV == 0 && al16(a.xr) && a.ldxr % WV == 0 && (!RC || (al16(a.xi) && a.ldxi % WV == 0)) &&
                      (!a.b || (al16(a.b) && a.ldb % WV == 0));
    const CarpSmem L =
        carp_smem_layout(w->max_fp, w->max_rows, w->seg_stride, TPR, (int)sizeof(T), RC, a.b != nullptr);
    PB_REQUIRE(L.total <= 227 * 1024, PB_NOT_IMPLEMENTED, "CARP block needs %d bytes of shared memory", L.total);
    auto one = [&](int color, int dir) {
      a.blk0 = w->h_bcolor_ptr[color];
      const int64_t cnt = w->h_bcolor_ptr[color + 1] - a.blk0;
      if (cnt <= 0) return;
      a.dir = dir;
      // one thread block per row block; with a programmatic dependency on
      // the previous launch in the stream (its blocks copy their segments
      // during that launch's tail)
      auto go = [&](auto kern) {
        set_smem(kern, L.total);
        cudaLaunchConfig_t cfg;
        memset(&cfg, 0, sizeof(cfg));
        cfg.gridDim = dim3((unsigned)cnt);
        cfg.blockDim = dim3(KB_NT);
        cfg.dynamicSmemBytes = L.total;
        cfg.stream = stream();
        cudaLaunchAttribute attr[1];
        attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
        attr[0].val.programmaticStreamSerializationAllowed = 1;
        cfg.attrs = attr;
        cfg.numAttrs = rt().carp_pdl ? 1 : 0;
        PB_CUDA(cudaLaunchKernelEx(&cfg, kern, a));
      };
#define PB_KB(TPRv)                                              \
  {                                                              \
    if (wide) go(k_kacz_blocks<T, TPRv, RC, KB_NT, WV>);        \
    else go(k_kacz_blocks<T, TPRv, RC, KB_NT, 1>);              \
  }
      if (TPR == 1) PB_KB(1)
      else if (TPR == 2) PB_KB(2)
      else if (TPR == 4) PB_KB(4)
      else if (TPR == 8) PB_KB(8)
      else if (TPR == 16) PB_KB(16)
      else PB_KB(32)
#undef PB_KB
      PB_LAUNCH_CHECK();
    };
    // forward over the colours, the last colour forward and straight back,
    // then backward over the others
    const int C = w->nbcolors;
    for (int c = 0; c < C - 1; c++) one(c, 1);
    if (C > 0) one(C - 1, 3);
    for (int c = C - 2; c >= 0; c--) one(c, 2);
  }
}

template <class T, bool RC>
void carp_run(const CarpWork<T>* w, int nvec, const T* sr, const T* si, const Mvec<T>* B,
              Mvec<T>* Xr, Mvec<T>* Xi, const T* omega)
{
  if (w->blocks) {
    carp_run_blocks<T, RC>(w, nvec, sr, si, B, Xr, Xi, omega);
    return;
  }
  for (int c0 = 0; c0 < nvec; c0 += 32) {
    const int nv = std::min(32, nvec - c0);
    KaczArgs<T> a;
    memset(&a, 0, sizeof(a));
    a.rows = w->d_rows; a.rp = w->d_rp; a.col = w->d_col; a.val = w->d_val;
    a.nrm = w->d_nrm; a.diag = w->d_diag;
    a.nvec = nv;
    for (int j = 0; j < nv; j++) {
      a.sig_r[j] = sr[c0 + j];
      a.sig_i[j] = si ? si[c0 + j] : T(0);
      a.omega[j] = omega[c0 + j];
    }
    a.b = B ? B->d() + c0 : nullptr;
    a.ldb = B ? B->lda : 0;
    a.xr = Xr->d() + c0;
    a.ldxr = Xr->lda;
    a.xi = Xi ? Xi->d() + c0 : nullptr;
    a.ldxi = Xi ? Xi->lda : 0;
    auto one = [&](int color) {
      a.q0 = w->h_color_ptr[color];
      a.q1 = w->h_color_ptr[color + 1];
      const int64_t cnt = a.q1 - a.q0;
      if (cnt <= 0) return;
      // one thread per (row, column): TPR = nv rounded up to a power of two
      const int TPR = nv <= 1 ? 1 : nv <= 2 ? 2 : nv <= 4 ? 4 : nv <= 8 ? 8 : nv <= 16 ? 16 : 32;
      const int grid = (int)ceil_div(cnt * TPR, 256);
#define PB_KZ(TPRv)                                                       \
  k_kacz_color_cols<T, TPRv, RC><<<grid, 256, 0, stream()>>>(a);
      if (TPR == 1) PB_KZ(1)
      else if (TPR == 2) PB_KZ(2)
      else if (TPR == 4) PB_KZ(4)
      else if (TPR == 8) PB_KZ(8)
      else if (TPR == 16) PB_KZ(16)
      else PB_KZ(32)
#undef PB_KZ
      PB_LAUNCH_CHECK();
    };
    for (int c = 0; c < w->ncolors; c++) one(c);        // forward
    for (int c = w->ncolors - 1; c >= 0; c--) one(c);   // backward
  }
}

}  // namespace pb
