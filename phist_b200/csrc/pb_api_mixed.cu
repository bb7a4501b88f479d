// pb_api_mixed.cu -- precision conversion helpers of the mixed-precision form
// (library extensions; PHIST itself has no mixed-type kernels)
#include "pb_api.cuh"

using namespace pb;

extern "C" {

void phist_b200_mvec_DtoS(const void* vX, void* vY, int* iflag)
{
  PB_API_BEGIN(iflag);
  const Mvec<double>* X = MV<double>(vX);
  Mvec<float>* Y = MV<float>(vY);
  PB_REQUIRE(X->nrows == Y->nrows && X->nvec == Y->nvec, PB_INVALID_INPUT, "mvec shapes differ");
  if (X->nrows > 0) {
    k_copy<double, float><<<grid_for((int64_t)X->nrows * X->nvec), 256, 0, stream()>>>(
        X->d(), X->lda, Y->d(), Y->lda, X->nrows, X->nvec);
    PB_LAUNCH_CHECK();
  }
  PB_API_END(iflag);
}

void phist_b200_mvec_StoD(const void* vX, void* vY, int* iflag)
{
  PB_API_BEGIN(iflag);
  const Mvec<float>* X = MV<float>(vX);
  Mvec<double>* Y = MV<double>(vY);
  PB_REQUIRE(X->nrows == Y->nrows && X->nvec == Y->nvec, PB_INVALID_INPUT, "mvec shapes differ");
  if (X->nrows > 0) {
    k_copy<float, double><<<grid_for((int64_t)X->nrows * X->nvec), 256, 0, stream()>>>(
        X->d(), X->lda, Y->d(), Y->lda, X->nrows, X->nvec);
    PB_LAUNCH_CHECK();
  }
  PB_API_END(iflag);
}

// FP32 copy of a double matrix: same rows, same sigma permutation and chunks
void phist_b200_sparseMat_DtoS(const void* vA, void** vAs, int* iflag)
{
  PB_API_BEGIN(iflag);
  const SparseMat<double>* A = SP<double>(vA);
  PB_REQUIRE(vAs, PB_BAD_CAST, "output handle is NULL");
  std::vector<int64_t> rp(A->h_row_ptr);
  std::vector<int32_t> col(A->h_col);
  std::vector<float> val(A->h_val.size());
  for (size_t p = 0; p < val.size(); p++) val[p] = (float)A->h_val[p];
  const int saveC = rt().sell_C;
  const int64_t saveS = rt().sell_sigma_default;
  rt().sell_C = A->C;
  rt().sell_sigma_default = A->sigma;
  try {
    *vAs = build_sparse<float>(A->comm, A->nrows, A->ncols, std::move(rp), std::move(col),
                               std::move(val), A->sigma > 1 ? PB_SPARSEMAT_PERM_LOCAL : 0);
  } catch (...) {
    rt().sell_C = saveC;
    rt().sell_sigma_default = saveS;
    throw;
  }
  rt().sell_C = saveC;
  rt().sell_sigma_default = saveS;
  PB_API_END(iflag);
}

}  // extern "C"
